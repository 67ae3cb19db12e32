import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", os.path.join("hyteg-vara_b200", "python")):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O

    O.build()
    return O


def _write_gmsh(path, coords, tets, seed, permute_cells=False):
    """A Gmsh 2.2 ASCII file of the mesh with scattered node ids, shuffled node and element
    order, and the lower-dimensional elements (points, edges, triangles) a Gmsh export holds.
    With permute_cells the vertices of each tetrahedron are listed in a random order."""
    rng = np.random.default_rng(seed)
    ids = np.sort(rng.choice(np.arange(1, 10 * len(coords) + 10), len(coords), replace=False))
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(len(coords))]
    for i in rng.permutation(len(coords)):
        lines.append("%d %.17g %.17g %.17g" % (ids[i], *coords[i]))
    lines += ["$EndNodes", "$Elements"]
    elems = [(15, [ids[0]]), (1, [ids[0], ids[1]]), (2, [ids[0], ids[1], ids[2]])]
    for t in tets:
        t = rng.permutation(t) if permute_cells else t
        elems.append((4, [ids[v] for v in t]))
    order = rng.permutation(len(elems))
    lines.append(str(len(elems)))
    for k, e in enumerate(order):
        typ, nodes = elems[e]
        lines.append(" ".join(map(str, [k + 1, typ, 2, 7, 3] + list(nodes))))
    lines.append("$EndElements")
    path.write_text("\n".join(lines) + "\n")


@pytest.fixture(scope="session")
def write_gmsh():
    return _write_gmsh
