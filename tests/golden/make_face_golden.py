"""Generate tests/golden/face_kernels_cube1.npz: the reference's macro-face rows.

Run with HYTEG_REFERENCE_ROOT naming the reference source tree. It compiles the reference's
generated macro-face kernels unchanged (oracle/Makefile target "ref",
oracle/ref_face_abi.cpp) and writes, for the six-tet unit cube:

* partial stencils at macro-face, -edge and -vertex points of every cell (levels 2..4):
  calculateStencilInMacroCellForm_new (src/hyteg/p1functionspace/P1Elements.hpp:464-516)
  summed over the micro-cells getNeighboringElements returns (P1Elements.hpp:215-290): the
  allCellsAtFace tables for a face point, the intersection of two of them for an edge point,
  the single micro-cell for a vertex point. The tables are read from P1Elements.hpp itself;
  the element rows come from the compiled FEniCS form (p1_tet_diffusion.h).
* at levels 3 and 4, for seeded inputs x, b: every face's apply
  (apply_3D_macroface_one_sided_vertexdof_to_vertexdof_{replace,add}, one call per neighbour
  cell as P1ConstantOperator.cpp:208-306 makes them), its SOR sweep
  (sor_3D_macroface_P1{,_one_sided}{,_backwards}, dispatched as P1ConstantOperator.cpp:372-534)
  with the ghost layers filled by communicate_directly_vertexdof_cell_to_face, and the
  index map of communicate_directly_vertexdof_face_to_cell (which face point lands on which
  cell-closure point).

Faces are the sorted vertex triples in ascending order (the face-local vertex order of a
mesh-built face), neighbour cells ascend by index. The tests compare the oracle's apply,
its face SOR stage and its cell closure maps with these arrays; neither they nor the GPU
runs need the reference tree.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import oracle as O  # noqa: E402
from make_golden import CELLS_AT_INNER_VERTEX, DIR, OFFS, cell_idx, micro_coord, tet_size  # noqa: E402

LEVELS_STENCIL = (2, 3, 4)
LEVELS_KERNEL = (3, 4)
SOR_CASES = ((1.0, 0), (0.8, 0), (0.8, 1), (1.0, 1))
# point masks: bit k set iff barycentric coordinate b_k is zero
MASKS = [8, 4, 2, 1,                       # faces 0..3: z = 0, y = 0, x = 0, x+y+z = N
         12, 10, 6, 9, 5, 3,               # edges: two zero barycentrics
         14, 13, 11, 7]                    # vertices 0..3: three zero barycentrics


def tables(ref_root):
    """allCellsAtFace0..3 and the single micro-cell at each cell vertex, from P1Elements.hpp."""
    src = open(os.path.join(ref_root, "src", "hyteg", "p1functionspace", "P1Elements.hpp")).read()
    faces = []
    for k in range(4):
        m = re.search(r"allCellsAtFace%d\s*=\s*\{(.*?)\}\s*\};" % k, src, re.S)
        toks = re.findall(r"VERTEX_(\w+)", m.group(1))
        assert len(toks) == 48, (k, len(toks))
        faces.append([tuple(toks[i:i + 4]) for i in range(0, 48, 4)])
    m = re.search(r"const auto singleMicroCell = \[localVertexID\] \{(.*?)\}\(\);", src, re.S)
    toks = re.findall(r"VERTEX_(\w+)", m.group(1))
    assert len(toks) == 16
    verts = [tuple(toks[i:i + 4]) for i in range(0, 16, 4)]
    return faces, verts


def bary_delta(d):
    """Change of the barycentric coordinates (b0..b3) along a logical offset."""
    x, y, z = DIR[d]
    return (-(x + y + z), x, y, z)


def half_space_rule(cells, zero_bary):
    """The micro-cells whose vertices all keep the barycentric coordinates in `zero_bary` >= 0."""
    return [c for c in cells if all(bary_delta(d)[k] >= 0 for d in c for k in zero_bary)]


def elements_at(mask, faces, verts):
    """getNeighboringElements for a point whose zero barycentrics are the bits of `mask`."""
    zero = [k for k in range(4) if mask >> k & 1]
    # local face id of barycentric b_k = 0: face 0 is z = 0 (b3), 1 is y = 0 (b2), 2 is x = 0 (b1), 3 is b0
    face_of = {3: 0, 2: 1, 1: 2, 0: 3}
    if len(zero) == 1:
        return faces[face_of[zero[0]]]
    if len(zero) == 2:
        a, b = (faces[face_of[k]] for k in zero)
        return [c for c in a if c in b]
    # the vertex whose barycentric coordinate is the non-zero one
    v = [k for k in range(4) if k not in zero][0]
    return [verts[v]]


def partial_stencil(R, V, level, mask, faces, verts):
    N = 1 << level
    zero = [k for k in range(4) if mask >> k & 1]
    # a point with exactly these barycentric coordinates zero (all others >= 1)
    free = [k for k in range(4) if k not in zero]
    b = [0] * 4
    for k in free:
        b[k] = 1
    b[free[0]] += N - sum(b)
    p = np.array(b[1:])
    st = np.zeros(15)
    A = np.zeros(16)
    for cell in elements_at(mask, faces, verts):
        X = np.concatenate([micro_coord(V, N, p + np.array(DIR[d])) for d in cell])
        R.ref_p1_tet_diffusion(O._p(X), O._p(A))
        for k, d in enumerate(cell):
            st[OFFS.index(DIR[d])] += A[k]
    return st


def mesh_faces(tets):
    fs = set()
    for t in tets:
        for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            fs.add(tuple(sorted(int(t[i]) for i in f)))
    return sorted(fs)


def face_cells(tets, f):
    return [c for c, t in enumerate(tets) if all(v in list(t) for v in f)]


def local_ids(t, f):
    return [list(t).index(v) for v in f]


def tri_idx(width, i, j):
    return i + j * (width + 1) - j * (j + 1) // 2


def face_layout(cm, t, f, N):
    """Closure indices of the face-layout triangle (width N + 1) of face f seen from a cell
    with vertex tuple t."""
    ids = local_ids(t, f)
    opp = [k for k in range(4) if k not in ids][0]
    out = np.zeros((N + 1) * (N + 2) // 2, np.int64)
    for j in range(N + 1):
        for i in range(N + 1 - j):
            b = [0] * 4
            b[ids[0]], b[ids[1]], b[ids[2]], b[opp] = N - i - j, i, j, 0
            out[tri_idx(N + 1, i, j)] = cm[cell_idx(N + 1, b[1], b[2], b[3])]
    return out


def main():
    root = O.reference_root()
    if not root:
        sys.exit("set HYTEG_REFERENCE_ROOT to the reference checkout")
    O.build(ref=True)
    R, RF = O.ref_lib(), O.ref_face_lib()
    assert R is not None and RF is not None, "reference kernels not built"
    faces_tab, verts_tab = tables(root)
    # the tables are the half-space rule: 12 micro-cells per face, one per vertex
    for k, zb in enumerate((3, 2, 1, 0)):
        assert sorted(faces_tab[k]) == sorted(half_space_rule(CELLS_AT_INNER_VERTEX, [zb])), k
    for v in range(4):
        assert [verts_tab[v]] == half_space_rule(CELLS_AT_INNER_VERTEX, [k for k in range(4) if k != v]), v

    coords, tets = O.mesh_cuboid(1, 1, 1)
    out = {"coords": coords, "tets": tets, "masks": np.array(MASKS), "levels_stencil": np.array(LEVELS_STENCIL),
           "levels_kernel": np.array(LEVELS_KERNEL), "sor_cases": np.array(SOR_CASES)}
    st = np.zeros((len(LEVELS_STENCIL), len(tets), len(MASKS), 15))
    for li, L in enumerate(LEVELS_STENCIL):
        for c, t in enumerate(tets):
            for mi, mask in enumerate(MASKS):
                st[li, c, mi] = partial_stencil(R, coords[t], L, mask, faces_tab, verts_tab)
    out["partial_stencils"] = st

    fl = mesh_faces(tets)
    rng = np.random.default_rng(11)
    for L in LEVELS_KERNEL:
        N = 1 << L
        o = O.Oracle(coords, tets, L)
        n = o.n(L)
        x = rng.uniform(-1, 1, n)
        b = rng.uniform(-1, 1, n)
        out[f"x_L{L}"], out[f"b_L{L}"] = x, b
        li = LEVELS_STENCIL.index(L)
        cms = [o.closure_map(L, c) for c in range(len(tets))]
        apply_out, sor_out, f2c = [], {cs: [] for cs in SOR_CASES}, []
        for f in fl:
            cs = face_cells(tets, f)
            ids = [np.array(local_ids(tets[c], f), np.int32) for c in cs]
            opp = [[k for k in range(4) if k not in list(i)][0] for i in ids]
            sts = [st[li, c, MASKS.index(1 << k)].copy() for c, k in zip(cs, opp)]
            gls = []
            for c, i in zip(cs, ids):
                gl = np.zeros(N * (N + 1) // 2)
                RF.ref_cell_to_face(O._p(np.ascontiguousarray(x[cms[c]])), O._p(gl), L, O._p(i))
                gls.append(gl)
            fmap = face_layout(cms[cs[0]], tets[cs[0]], f, N)
            src = np.ascontiguousarray(x[fmap])
            dst = np.zeros_like(src)
            for k, (gl, i, s) in enumerate(zip(gls, ids, sts)):
                RF.ref_face_apply(O._p(dst), O._p(src), O._p(gl), L, O._p(i), O._p(s), int(k > 0))
            apply_out.append(dst)
            rhs = np.ascontiguousarray(b[fmap])
            two = len(cs) == 2
            for relax, bw in SOR_CASES:
                fc = src.copy()
                g = [gl.copy() for gl in gls]
                RF.ref_face_sor(O._p(fc), O._p(g[0]), O._p(g[1]) if two else None, O._p(rhs), L, O._p(ids[0]),
                                O._p(ids[1]) if two else None, relax, O._p(sts[0]), O._p(sts[1]) if two else None, bw)
                sor_out[(relax, bw)].append(fc)
            # face -> cell: which face-layout point lands on which closure point of each cell
            for c, i in zip(cs, ids):
                cell = np.full(tet_size(N + 1), -1.0)
                RF.ref_face_to_cell(O._p(cell), O._p(np.arange(len(src), dtype=np.float64)), L, O._p(i))
                f2c.append(cell.astype(np.int32))
        out[f"apply_L{L}"] = np.array(apply_out)
        for (relax, bw), v in sor_out.items():
            out[f"sor_L{L}_relax{relax}_bw{bw}"] = np.array(v)
        out[f"face_to_cell_L{L}"] = np.array(f2c)
    np.savez_compressed(os.path.join(HERE, "face_kernels_cube1.npz"), **out)
    print("wrote face_kernels_cube1.npz:", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
