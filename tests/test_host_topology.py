"""Host-side numbering, tables and index maps of the product against the reference fixtures."""

import numpy as np
import pytest

from oracle import q1_mhm as o
from pymhm_b200 import topology as tp
from tests._cases import face_space, CASES, load


def product_case(name):
    margs, face, ref, *_ = CASES[name]
    mesh = tp.CartesianMacroMesh(*margs)
    sk = tp.SkeletonSpace(mesh, (face_space(tp.FaceSpace, face),) * len(mesh.faces))
    return mesh, sk, ref


@pytest.mark.parametrize("name", list(CASES))
def test_numbering_bit_exact(name):
    g = load(name)
    mesh, sk, _ = product_case(name)
    for key in ("cell_faces", "signs", "faces", "face_cells"):
        assert np.array_equal(getattr(mesh, key), g[key]), key
    assert np.array_equal(sk.offsets, g["offsets"])
    assert np.array_equal(sk.cell_dof_array, g["cell_dofs"])


@pytest.mark.parametrize("n", [(1, 1), (5, 3), (2, 7), (64, 64)])
def test_vectorised_mesh_equals_first_encounter_definition(n):
    mine = tp.CartesianMacroMesh(*n)
    ref = o.cartesian_mesh(*n)
    for key in ("cells", "faces", "cell_faces", "signs", "face_cells"):
        assert np.array_equal(getattr(mine, key), getattr(ref, key)), key


@pytest.mark.parametrize("name", list(CASES))
def test_coupling_tables_reproduce_trace_coupling(name):
    """Per-side tables x cell signs equal the reference trace coupling B (quadrilateral.py:256-298)."""
    g = load(name)
    mesh, sk, (rx, ry) = product_case(name)
    sh, sv = sk.uniform_by_orientation()
    hx, hy = mesh.spacing
    table = tp.coupling_tables(sh, sv, rx, ry, hx, hy)
    orient = tp.side_orientation(mesh)
    nnx, nny = rx + 1, ry + 1
    for c in g["keep_cells"]:
        B = np.zeros((nnx * nny, 2 * (sh.size + sv.size)))
        off = 0
        for s in range(4):
            kind = s % 2
            size = sh.size if kind == 0 else sv.size
            length = nnx if kind == 0 else nny
            nodes = [k, k * nnx + nnx - 1, (nny - 1) * nnx + k, k * nnx] if False else None
            for k in range(length):
                node = (k, k * nnx + nnx - 1, (nny - 1) * nnx + k, k * nnx)[s]
                B[node, off: off + size] += mesh.signs[c, s] * table[kind, orient[c, s], k, :size]
            off += size
        assert np.allclose(B, g[f"cell{c}_B"], rtol=0, atol=1e-15 * np.abs(g[f"cell{c}_B"]).max())


@pytest.mark.parametrize("n,deg,sub", [((8,), 1, 1), ((5, 3, (0, 2, 0, 1)), 2, 1), ((4, 6), 1, 2)])
def test_sine_transform_diagonalises_geometric_coarse_operator(n, deg, sub):
    mesh = tp.CartesianMacroMesh(*n)
    sk = tp.SkeletonSpace(mesh, (tp.FaceSpace.uniform(deg, sub),) * len(mesh.faces))
    sh, sv = sk.uniform_by_orientation()
    g0 = tp.geometric_constraint(mesh, sh, sv)
    G = np.zeros((sk.size, len(mesh.cells)))
    for c in range(len(mesh.cells)):
        G[sk.cell_dof_array[c], c] += g0[c]
    GG = G.T @ G
    qx, qy = tp.sine_transform(mesh.nx), tp.sine_transform(mesh.ny)
    eig = tp.coarse_eigenvalues(mesh, sh, sv)
    # apply Q (diag) Q to unit vectors: V[iy, ix]
    inv = np.zeros_like(GG)
    for c in range(len(mesh.cells)):
        v = np.zeros((mesh.ny, mesh.nx))
        v.flat[c] = 1.0
        w = (qy @ v @ qx) / eig
        inv[:, c] = (qy @ w @ qx).ravel()
    assert np.allclose(inv @ GG, np.eye(len(mesh.cells)), atol=1e-10)


@pytest.mark.parametrize("name", list(CASES))
def test_geometric_constraint_is_coupling_times_one(name):
    g = load(name)
    mesh, sk, _ = product_case(name)
    sh, sv = sk.uniform_by_orientation()
    g0 = tp.geometric_constraint(mesh, sh, sv)
    for c in g["keep_cells"]:
        assert np.allclose(g0[c], g[f"cell{c}_B"].sum(axis=0), rtol=0, atol=1e-15)


@pytest.mark.parametrize("name", list(CASES))
def test_pattern_maps_reproduce_oracle_assembly(name):
    """The contributor lists sum blocks in cell order exactly like assemble_hybrid_contributions."""
    mesh, sk, ref = product_case(name)
    g = load(name)
    cd = sk.cell_dof_array
    pat = tp.skeleton_pattern(cd, sk.size)
    rng = np.random.default_rng(5)
    t1 = cd.shape[1] + 1
    blocks = rng.normal(size=(len(cd), t1, t1))
    loads = rng.normal(size=(len(cd), t1))
    vals = np.array([blocks.ravel()[pat.contrib[a:b]].sum() for a, b in zip(pat.slot_ptr[:-1], pat.slot_ptr[1:])])
    contribs = [(np.r_[cd[c], sk.size + c], blocks[c], loads[c]) for c in range(len(cd))]
    boundary = rng.normal(size=sk.size)
    A, rhs, scale = o.assemble_global(contribs, sk.size, boundary)
    ours = np.zeros(pat.size)
    sc = np.zeros(pat.size)
    for r in range(pat.size):
        seg = loads.ravel()[pat.load_contrib[pat.load_ptr[r]:pat.load_ptr[r + 1]]]
        acc = 0.0
        for v in seg:
            acc += v
        ours[r] = acc - (boundary[r] if r < sk.size else 0.0)
        sc[r] = np.abs(seg).sum() + (abs(boundary[r]) if r < sk.size else 0.0)
    assert np.array_equal(ours, rhs)
    assert np.allclose(sc, scale, rtol=1e-15)
    dense = A.toarray()
    rows = np.repeat(np.arange(pat.size), np.diff(pat.indptr))
    assert np.array_equal(dense[rows, pat.indices], vals)
    assert np.all(pat.indices[pat.indptr[1]:pat.indptr[2]][:-1] < pat.indices[pat.indptr[1]:pat.indptr[2]][1:])
    del g, ref


@pytest.mark.parametrize("name", list(CASES))
def test_boundary_load_matches_reference(name):
    g = load(name)
    mesh, sk, _ = product_case(name)
    dr = CASES[name][5]
    b = tp.boundary_data(sk, dr, 4)
    assert np.allclose(b, g["boundary"], rtol=0, atol=1e-15 * max(1.0, np.abs(g["boundary"]).max()))


def test_dof_cell_maps():
    mesh = tp.CartesianMacroMesh(3, 2)
    sk = tp.SkeletonSpace(mesh, (tp.FaceSpace.uniform(2),) * len(mesh.faces))
    dc, ds = tp.dof_cell_maps(sk.cell_dof_array, sk.size)
    for dof in range(sk.size):
        for k in range(2):
            c = dc[dof, k]
            if c >= 0:
                assert sk.cell_dof_array[c, ds[dof, k]] == dof
    assert np.all((dc[:, 0] >= 0))
    assert np.all((dc[:, 1] == -1) | (dc[:, 1] > dc[:, 0]))
