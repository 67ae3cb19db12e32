"""Pin the oracle's macro-face, -edge and -vertex rows to the reference.

tests/golden/face_kernels_cube1.npz (tests/golden/make_face_golden.py) holds what the
reference's own code computes on the six-tet unit cube:

* the partial stencils of every cell at face, edge and vertex points
  (calculateStencilInMacroCellForm_new over getNeighboringElements, P1Elements.hpp:215-516,
  with the compiled FEniCS form);
* every face's apply and SOR sweep through the generated macro-face kernels
  (apply_3D_macroface_one_sided_vertexdof_to_vertexdof_*, sor_3D_macroface_P1*), the ghost
  layers filled by communicate_directly_vertexdof_cell_to_face;
* where communicate_directly_vertexdof_face_to_cell puts each face point in each
  neighbour cell's closure.

The face-layout DoFs below come from the canonical numbering alone (hyteg_oracle.h), not
from the oracle's closure maps, so the face-to-cell check pins those maps independently.
"""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "face_kernels_cube1.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def tri_idx(width, i, j):
    return i + j * (width + 1) - j * (j + 1) // 2


def mesh_prims(tets):
    es, fs = set(), set()
    for t in tets:
        t = [int(v) for v in t]
        for a in range(4):
            for b in range(a + 1, 4):
                es.add(tuple(sorted((t[a], t[b]))))
        for f in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
            fs.add(tuple(sorted(t[i] for i in f)))
    return sorted(es), sorted(fs)


def face_dofs(nv, edges, faces, f, N):
    """Canonical DoF of every point of face f's closure, in the face layout (width N + 1,
    face vertex 0 at the origin, i towards vertex 1, j towards vertex 2)."""
    eid = {e: k for k, e in enumerate(edges)}
    fid = faces.index(f)
    offE = nv
    offF = offE + len(edges) * (N - 1)
    nIntFace = (N - 1) * (N - 2) // 2
    out = np.zeros((N + 1) * (N + 2) // 2, np.int64)
    for j in range(N + 1):
        for i in range(N + 1 - j):
            w = {f[0]: N - i - j, f[1]: i, f[2]: j}
            nz = sorted(v for v in f if w[v] > 0)
            if len(nz) == 1:
                d = nz[0]
            elif len(nz) == 2:
                d = offE + eid[tuple(nz)] * (N - 1) + w[nz[1]] - 1
            else:
                d = offF + fid * nIntFace + (j - 1) * (N - 1) - (j - 1) * j // 2 + (i - 1)
            out[tri_idx(N + 1, i, j)] = d
    return out


def inner_points(N):
    return [tri_idx(N + 1, i, j) for j in range(1, N - 1) for i in range(1, N - j)]


def face_cells(tets, f):
    return [c for c, t in enumerate(tets) if all(v in [int(u) for u in t] for v in f)]


def test_partial_stencils_match_reference_assembly(oracle_mod, gold):
    """Face/edge/vertex stencils of each cell = the reference's element-list recipe."""
    O = oracle_mod
    o = O.Oracle(gold["coords"], gold["tets"], int(gold["levels_stencil"].max()))
    for li, L in enumerate(gold["levels_stencil"]):
        for c in range(len(gold["tets"])):
            for mi, mask in enumerate(gold["masks"]):
                ref = gold["partial_stencils"][li, c, mi]
                got = o.cell_stencil(int(L), c, int(mask))
                np.testing.assert_allclose(got, ref, rtol=0, atol=1e-13 * np.abs(ref).max(),
                                           err_msg=f"level {L} cell {c} mask {mask}")


@pytest.mark.parametrize("level", [3, 4])
def test_closure_maps_match_face_to_cell_kernel(oracle_mod, gold, level):
    """communicate_directly_vertexdof_face_to_cell puts face point p at closure point q of
    each neighbour cell; the oracle's closure map must name the same DoF at q."""
    O = oracle_mod
    tets = gold["tets"]
    N = 1 << level
    o = O.Oracle(gold["coords"], tets, level)
    edges, faces = mesh_prims(tets)
    f2c = gold[f"face_to_cell_L{level}"]
    k = 0
    for f in faces:
        fd = face_dofs(len(gold["coords"]), edges, faces, f, N)
        for c in face_cells(tets, f):
            cm = o.closure_map(level, c)
            g = f2c[k]
            k += 1
            pos = np.nonzero(g >= 0)[0]
            assert len(pos) == len(fd)  # every face point lands on a distinct closure point
            np.testing.assert_array_equal(cm[pos], fd[g[pos]], err_msg=f"face {f} cell {c}")
    assert k == len(f2c)


@pytest.mark.parametrize("level", [3, 4])
def test_face_apply_matches_generated_face_kernels(oracle_mod, gold, level):
    O = oracle_mod
    tets = gold["tets"]
    N = 1 << level
    o = O.Oracle(gold["coords"], tets, level)
    edges, faces = mesh_prims(tets)
    x = gold[f"x_L{level}"]
    assert len(x) == o.n(level)
    y = o.apply(x, level, flag=O.ALL)
    ref = gold[f"apply_L{level}"]
    ip = inner_points(N)
    for fi, f in enumerate(faces):
        fd = face_dofs(len(gold["coords"]), edges, faces, f, N)
        r = ref[fi][ip]
        np.testing.assert_allclose(y[fd[ip]], r, rtol=0, atol=1e-12 * (1 + np.abs(r).max()),
                                   err_msg=f"face {f} ({len(face_cells(tets, f))} cells)")


@pytest.mark.parametrize("level", [3, 4])
def test_face_sor_stage_matches_generated_face_kernels(oracle_mod, gold, level):
    """The face stage of the reference-order SOR (one- and two-sided faces, forward and
    backward, relax 1 and 0.8) against sor_3D_macroface_P1*; nothing but face interiors moves."""
    O = oracle_mod
    tets = gold["tets"]
    N = 1 << level
    o = O.Oracle(gold["coords"], tets, level)
    edges, faces = mesh_prims(tets)
    x0, b = gold[f"x_L{level}"], gold[f"b_L{level}"]
    ip = inner_points(N)
    fds = [face_dofs(len(gold["coords"]), edges, faces, f, N) for f in faces]
    moved = np.zeros(len(x0), bool)
    for fd in fds:
        moved[fd[ip]] = True
    for relax, bw in gold["sor_cases"]:
        xs = x0.copy()
        o.sor_ref(xs, b, level, relax=float(relax), flag=O.ALL, backwards=bool(bw), stages=4)
        np.testing.assert_array_equal(xs[~moved], x0[~moved])
        ref = gold[f"sor_L{level}_relax{float(relax)}_bw{int(bw)}"]
        for fi, f in enumerate(faces):
            r = ref[fi][ip]
            assert not np.allclose(r, x0[fds[fi][ip]])  # the kernel did run on this face
            np.testing.assert_allclose(xs[fds[fi][ip]], r, rtol=0, atol=1e-12 * (1 + np.abs(r).max()),
                                       err_msg=f"face {f} relax {relax} backwards {bw}")


def test_apply_rows_equals_apply(oracle_mod, gold):
    """The oracle's row spot check (used on levels too large for a full oracle apply) is the
    full apply restricted to the listed DoFs."""
    O = oracle_mod
    o = O.Oracle(gold["coords"], gold["tets"], 4)
    x = gold["x_L4"]
    dofs = np.arange(o.n(4))[::7]
    np.testing.assert_array_equal(o.apply_rows(x, 4, dofs), o.apply(x, 4, flag=O.ALL)[dofs])
