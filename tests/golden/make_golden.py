"""Generate the golden fixtures that pin the CPU oracle to the reference.

Run with HYTEG_REFERENCE_ROOT naming the reference source tree. It compiles the reference's own generated macro-cell kernels
and its FEniCS P1 diffusion form, unchanged, into oracle/_ref/ (oracle/Makefile
target "ref"), runs them on seeded inputs and writes tests/golden/*.npz.
The tests then compare the oracle against these files; neither the tests nor
the GPU runs need the reference tree.

Reference pieces exercised (paths relative to the reference project root):
  src/hyteg/forms/form_fenics_generated/p1_tet_diffusion.h           element stiffness
  src/hyteg/p1functionspace/P1Elements.hpp:93-302, 464-526           stencil assembly recipe
  src/hyteg/p1functionspace/generatedKernels/apply_3D_macrocell_*    cell apply
  src/hyteg/p1functionspace/generatedKernels/sor_3D_macrocell_P1*    cell SOR (forward/backward)
  src/hyteg/gridtransferoperators/generatedKernels/prolongate_3D_macrocell_P1_push_additive.cpp
  src/hyteg/gridtransferoperators/generatedKernels/restrict_3D_macrocell_P1_pull_additive.cpp
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# Stencil-direction names -> logical offsets (VertexDoFIndexing.cpp:484-525)
DIR = {"C": (0, 0, 0), "W": (-1, 0, 0), "E": (1, 0, 0), "N": (0, 1, 0), "S": (0, -1, 0), "NW": (-1, 1, 0),
       "SE": (1, -1, 0), "TC": (0, 0, 1), "TW": (-1, 0, 1), "TS": (0, -1, 1), "TSE": (1, -1, 1), "BC": (0, 0, -1),
       "BN": (0, 1, -1), "BE": (1, 0, -1), "BNW": (-1, 1, -1)}
# The 24 micro-cells at an inner micro-vertex, as listed in P1Elements.hpp:93-143
# (white up/down, blue up/down, green up/down; first entry is always the centre).
CELLS_AT_INNER_VERTEX = [
    ("C", "BC", "BE", "BN"), ("C", "S", "SE", "TS"), ("C", "W", "NW", "TW"), ("C", "N", "E", "TC"),
    ("C", "W", "BC", "S"), ("C", "E", "SE", "BE"), ("C", "N", "NW", "BN"), ("C", "TS", "TC", "TW"),
    ("C", "BC", "BN", "BNW"), ("C", "W", "S", "TS"), ("C", "E", "SE", "TSE"), ("C", "NW", "N", "TC"),
    ("C", "BC", "S", "SE"), ("C", "W", "NW", "BNW"), ("C", "E", "BN", "N"), ("C", "TC", "TS", "TSE"),
    ("C", "W", "BC", "BNW"), ("C", "E", "BE", "BN"), ("C", "TC", "TW", "NW"), ("C", "SE", "TS", "TSE"),
    ("C", "BC", "BE", "SE"), ("C", "BN", "BNW", "NW"), ("C", "E", "TSE", "TC"), ("C", "W", "TS", "TW"),
]
OFFS = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (-1, 1, 0), (1, -1, 0),
        (-1, 0, 1), (1, 0, -1), (0, -1, 1), (0, 1, -1), (-1, 1, -1), (1, -1, 1)]


def tet_size(w):
    return (w + 2) * (w + 1) * w // 6


def cell_idx(width, x, y, z):
    wms = width - z
    return tet_size(width) - tet_size(wms) + y * (wms + 1) - ((y + 1) * y) // 2 + x


def micro_coord(V, N, idx):
    v0, v1, v2, v3 = V
    return v0 + (v1 - v0) / N * idx[0] + (v2 - v0) / N * idx[1] + (v3 - v0) / N * idx[2]


def ref_inner_stencil(R, V, level):
    """calculateStencilInMacroCellForm_new at an inner vertex, with the FEniCS form row 0."""
    N = 1 << level
    centre = np.array([2, 2, 2])  # any inner point: the stencil is translation invariant
    st = np.zeros(15)
    A = np.zeros(16)
    for cell in CELLS_AT_INNER_VERTEX:
        idxs = [centre + np.array(DIR[d]) for d in cell]
        X = np.concatenate([micro_coord(V, N, i) for i in idxs])
        R.ref_p1_tet_diffusion(O._p(X), O._p(A))
        for k, d in enumerate(cell):
            st[OFFS.index(DIR[d])] += A[k]  # row 0 (A is symmetric)
    return st


def cell_neighbour_counts(tets):
    """#cells at each local edge (0..5), face (0..3), vertex (0..3) of every cell, in the
    reference's local numbering (SetupPrimitiveStorage.cpp:259-292)."""
    from collections import Counter
    ec, fc, vc = Counter(), Counter(), Counter()
    for t in tets:
        for a in range(4):
            vc[t[a]] += 1
            for b in range(a + 1, 4):
                ec[tuple(sorted((t[a], t[b])))] += 1
        for f in [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]:
            fc[tuple(sorted(t[i] for i in f))] += 1
    out = []
    for t in tets:
        edges = [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3)]
        faces = [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)]
        row = [ec[tuple(sorted((t[a], t[b])))] for a, b in edges]
        row += [fc[tuple(sorted(t[i] for i in f))] for f in faces]
        row += [vc[t[a]] for a in range(4)]
        out.append(row)
    return np.array(out, np.float64)


def main():
    if not O.reference_root():
        sys.exit("set HYTEG_REFERENCE_ROOT to the reference checkout")
    O.build(ref=True)
    R = O.ref_lib()
    assert R is not None, "reference kernels not built"
    rng = np.random.default_rng(0)

    # 1) element stiffness of random tetrahedra
    X = rng.uniform(-1, 1, size=(8, 12))
    K = np.zeros((8, 16))
    for i in range(8):
        R.ref_p1_tet_diffusion(O._p(X[i].copy()), O._p(K[i]))
    np.savez(os.path.join(HERE, "fenics_p1_tet_diffusion.npz"), coords=X, K=K)

    # 2) inner stencils of the six cuboid macro-tets (levels 2..4)
    coords, tets = O.mesh_cuboid(1, 1, 1)
    st = np.zeros((3, len(tets), 15))
    for li, level in enumerate((2, 3, 4)):
        for c, t in enumerate(tets):
            st[li, c] = ref_inner_stencil(R, coords[t], level)
    np.savez(os.path.join(HERE, "stencils_cube1.npz"), levels=np.array([2, 3, 4]), stencils=st, coords=coords,
             tets=tets)

    # 3) generated cell kernels on one macro-cell closure (cell 0 of the cube mesh, level 4)
    level = 4
    N = 1 << level
    S = tet_size(N + 1)
    src = rng.uniform(-1, 1, S)
    rhs = rng.uniform(-1, 1, S)
    dst0 = rng.uniform(-1, 1, S)
    stencil = st[2, 0]
    out = {}
    d = dst0.copy()
    R.ref_apply_cell(O._p(d), O._p(src), level, O._p(stencil), 0)
    out["apply_replace"] = d
    d = dst0.copy()
    R.ref_apply_cell(O._p(d), O._p(src), level, O._p(stencil), 1)
    out["apply_add"] = d
    for relax in (1.0, 0.8):
        for bw in (0, 1):
            x = src.copy()
            R.ref_sor_cell(O._p(x), O._p(rhs), level, O._p(stencil), relax, bw)
            out[f"sor_relax{relax}_bw{bw}"] = x
    np.savez(os.path.join(HERE, "cell_kernels_L4.npz"), level=level, src=src, rhs=rhs, dst0=dst0, stencil=stencil,
             **out)

    # 4) generated transfer kernels on all six cells of the cube mesh, coarse level 3.
    #    Global (consistent) vectors are gathered into each cell's closure with the
    #    oracle's closure map; the per-cell kernel outputs are stored in closure layout.
    cl = 3
    nbr = cell_neighbour_counts(tets)
    orc = O.Oracle(coords, tets, cl + 1)
    coarse = rng.uniform(-1, 1, orc.n(cl))
    fine = rng.uniform(-1, 1, orc.n(cl + 1))
    Sc, Sf = tet_size((1 << cl) + 1), tet_size((1 << (cl + 1)) + 1)
    pro, res = np.zeros((len(tets), Sf)), np.zeros((len(tets), Sc))
    for c in range(len(tets)):
        f = np.zeros(Sf)
        R.ref_prolongate_cell(O._p(coarse[orc.closure_map(cl, c)].copy()), O._p(f), cl, O._p(nbr[c].copy()))
        pro[c] = f
        r = np.zeros(Sc)
        R.ref_restrict_cell(O._p(r), O._p(fine[orc.closure_map(cl + 1, c)].copy()), cl, O._p(nbr[c].copy()))
        res[c] = r
    np.savez(os.path.join(HERE, "transfer_cube1_L3.npz"), coarse_level=cl, nbr=nbr, coarse=coarse, fine=fine,
             prolongated=pro, restricted=res)
    # 5) the reference test meshes used by the ported known-answer tests, parsed from the
    #    Gmsh files the reference's tests load (data/meshes/3D/*.msh; MeshGenFromGmshFile.cpp:
    #    node ids as given, tetrahedra (element type 4) keyed by their vertex-id vectors)
    meshes = {}
    for name in ("regular_octahedron_8el", "tet_1el", "pyramid_4el", "cube_6el"):
        path = os.path.join(REF_ROOT, "data", "meshes", "3D", name + ".msh")
        if os.path.exists(path):
            c, t = read_gmsh(path)
            meshes[name + "_coords"] = c
            meshes[name + "_tets"] = t
    np.savez(os.path.join(HERE, "reference_meshes.npz"), **meshes)
    print("golden fixtures written to", HERE)


REF_ROOT = os.environ.get("HYTEG_REFERENCE_ROOT")


def read_gmsh(path):
    """Gmsh 2.2 ASCII: nodes (id x y z) and tetrahedra (type 4), ids made 0-based, cells in
    the lexicographic order of their vertex-id vectors (the reference's std::map order)."""
    lines = open(path).read().split("\n")
    i = lines.index("$Nodes")
    n = int(lines[i + 1])
    ids, xyz = [], []
    for k in range(n):
        f = lines[i + 2 + k].split()
        ids.append(int(f[0]))
        xyz.append([float(v) for v in f[1:4]])
    order = np.argsort(ids)
    remap = {ids[j]: r for r, j in enumerate(order)}
    coords = np.array(xyz)[order]
    i = lines.index("$Elements")
    n = int(lines[i + 1])
    tets = set()
    for k in range(n):
        f = [int(v) for v in lines[i + 2 + k].split()]
        if f[1] == 4:
            ntags = f[2]
            tets.add(tuple(remap[v] for v in f[3 + ntags:3 + ntags + 4]))
    return coords, np.array(sorted(tets), np.int64)


if __name__ == "__main__":
    main()
