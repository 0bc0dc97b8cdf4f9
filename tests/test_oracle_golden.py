"""The oracle against fixtures written by the reference itself (tests/golden/make_golden.py)."""

import numpy as np
import pytest
from scipy import sparse

from oracle import q1_mhm as o
from tests._cases import face_space, CASES, load, rel

# Cases whose fine cells are cut by pixel lines: the reference evaluates the Q1 basis at
# per-cell intersection points through its tabulation backend, so operator entries agree
# to rounding, and an entry that cancels to exactly zero on one side (then dropped by
# eliminate_zeros) may be a rounding residue on the other.
ROUNDED_PATTERN = ("darcy_4x4_r8_p1_cut20",)


def oracle_case(name):
    g = load(name)
    margs, face, ref, perm, src, dr = CASES[name]
    mesh = o.cartesian_mesh(*margs)
    sk = o.Skeleton(mesh, (face_space(o.FaceSpace, face),) * len(mesh.faces))
    p = perm(g)
    if hasattr(p, "values"):
        p = o.PixelField(p.values, p.spacing, p.origin)
    return g, mesh, sk, ref, p, src, dr


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_reference(name):
    g, mesh, sk, ref, perm, src, dr = oracle_case(name)
    assert np.array_equal(mesh.cell_faces, g["cell_faces"])
    assert np.array_equal(mesh.signs, g["signs"])
    assert np.array_equal(mesh.faces, g["faces"])
    assert np.array_equal(sk.offsets, g["offsets"])
    sol = o.solve_darcy_q1(mesh, sk, ref, perm, src, dr, keep_responses=True)
    if name in ROUNDED_PATTERN:
        tol = 1e-13
        n = sk.size + len(mesh.cells)
        dense = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n)).toarray()
        mine = sol.matrix.toarray()
        scale = np.max(np.abs(dense))
        assert np.max(np.abs(mine - dense)) <= tol * scale
        # pattern differences are entries that vanish to rounding
        diff = (mine != 0) != (dense != 0)
        assert np.all(np.abs(mine[diff]) <= 1e-15 * scale) and np.all(np.abs(dense[diff]) <= 1e-15 * scale)
    else:
        # bit-exact sparsity after the reference's eliminate_zeros
        assert np.array_equal(sol.matrix.indptr, g["indptr"])
        assert np.array_equal(sol.matrix.indices, g["indices"])
        # values: identical arithmetic except the breakpoint-split trace integrals (1e-16 level)
        tol = 0.0 if name != "affine_3x2_rect_r4x5_p1s2" else 1e-13
        assert np.max(np.abs(sol.matrix.data - g["data"])) <= tol * np.max(np.abs(g["data"]))
    for key, val in (("trace", sol.trace), ("coarse", sol.coarse), ("fields", sol.fields), ("flux", sol.flux),
                     ("rhs", sol.rhs)):
        assert rel(val, g[key]) <= max(tol, 0.0) * 100, key
    assert np.array_equal(sol.corrected, g["corrected"])
    for c in g["keep_cells"]:
        r = sol.responses[c]
        idx, block, ld = o.contribution(r, sk.size + c)
        assert rel(r.lifts, g[f"cell{c}_lifts"]) <= tol * 100
        assert rel(block, g[f"cell{c}_block"]) <= tol * 100
        assert rel(ld, g[f"cell{c}_load"]) <= max(tol * 100, 1e-12)


@pytest.mark.parametrize("name", list(CASES))
def test_structural_pattern_covers_reference(name):
    """Reference nonzeros = structural pattern minus entries that sum to exactly zero."""
    from pymhm_b200.topology import skeleton_pattern

    g, mesh, sk, ref, perm, src, dr = oracle_case(name)
    cell_dofs = np.array([sk.cell_dofs(c) for c in range(len(mesh.cells))])
    pat = skeleton_pattern(cell_dofs, sk.size)
    N = pat.size
    struct = sparse.csr_matrix((np.ones(len(pat.indices)), pat.indices, pat.indptr), shape=(N, N))
    ref_m = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N)).tocsr()
    ref_m.sort_indices()
    ones = ref_m.copy()
    ones.data[:] = 1.0
    assert (ones - ones.multiply(struct)).nnz == 0  # reference pattern inside the structural one
    # the oracle's own pre-elimination assembly is zero exactly on the difference
    contribs = []
    for c in range(len(mesh.cells)):
        _, prob = o.local_problem(mesh, sk, c, ref, perm, src)
        contribs.append(o.contribution(o.condense(prob), sk.size + c))
    rows = np.concatenate([np.repeat(i, len(i)) for i, _, _ in contribs])
    cols = np.concatenate([np.tile(i, len(i)) for i, _, _ in contribs])
    vals = np.concatenate([b.ravel() for _, b, _ in contribs])
    full = sparse.coo_matrix((vals, (rows, cols)), shape=(N, N)).tocsr()
    full.sum_duplicates()
    missing = struct - ones.multiply(struct)
    r, cc = missing.nonzero()
    bound = 0.0 if name not in ROUNDED_PATTERN else 1e-15 * np.max(np.abs(g["data"]))
    if len(r):
        assert np.all(np.abs(np.asarray(full[r, cc]).ravel()) <= bound)
    assert len(pat.indices) - len(g["indices"]) == len(r)


def test_full_size_topology_digests():
    from pymhm_b200.workloads import digest

    g = load("darcy_64x64_r16_p2_lognormal")
    mesh = o.cartesian_mesh(64)
    sk = o.Skeleton(mesh, (o.FaceSpace.uniform(2),) * len(mesh.faces))
    cell_dofs = np.array([sk.cell_dofs(c) for c in range(len(mesh.cells))])
    assert digest(mesh.cell_faces) == str(g["cell_faces_sha256"])
    assert digest(mesh.signs) == str(g["signs_sha256"])
    assert digest(mesh.faces) == str(g["faces_sha256"])
    assert digest(cell_dofs) == str(g["cell_dofs_sha256"])


def test_oracle_condensation_matches_monolithic_solve():
    """The reference's algebraic check (tests/test_hybrid.py:28-42) on a Q1 cell."""
    g = load("poisson_8x8_r4_p1")
    aug, rhs = g["cell0_aug"], g["cell0_rhs"]
    x = np.linalg.solve(aug, rhs)
    n = len(g["cell0_source"])
    assert np.allclose(x[:n, 0], g["cell0_source"], atol=1e-13)
    assert np.allclose(x[:n, 1:1 + g["cell0_lifts"].shape[1]], g["cell0_lifts"], atol=1e-13)


def test_full_size_oracle_is_the_reference():
    """At 64x64 x 16x16 the oracle's parallel solve reproduces the reference: the
    skeleton matrix's SHA-256 digests (indptr, indices, data after eliminate_zeros),
    its trace and coarse unknowns exactly, and the norms and kept cells of the fields
    and fluxes.  This pins the oracle as the checker of the full-size GPU solve."""
    from pymhm_b200.workloads import digest
    from tests._full_size import oracle_solution

    g = load("darcy_64x64_r16_p2_lognormal")
    sol = oracle_solution()
    m = sol["matrix"]
    assert digest(m.indptr) == str(g["indptr_sha256"])
    assert digest(m.indices) == str(g["indices_sha256"])
    assert digest(m.data) == str(g["data_sha256"])
    assert np.array_equal(sol["trace"], g["trace"])
    assert np.array_equal(sol["coarse"], g["coarse"])
    assert np.array_equal(sol["rhs"], g["rhs"])
    assert np.linalg.norm(sol["fields"]) == pytest.approx(float(g["fields_norm"]), rel=1e-15)
    assert np.linalg.norm(sol["flux"]) == pytest.approx(float(g["flux_norm"]), rel=1e-15)
    keep = list(g["keep_cells"])
    assert rel(sol["fields"][keep], g["fields_cells"]) <= 1e-15
    # the gradient's differences amplify the reconstruction's rounding
    assert rel(sol["flux"][keep], g["flux_cells"]) <= 1e-13


def test_vectorised_flux_equals_cell_flux():
    """``cartesian_flux`` (all cells at once) is ``cell_flux`` cell by cell, bit for bit."""
    mesh = o.cartesian_mesh(3, 2, (-1.0, 2.0, -2.0, 2.0))
    rng = np.random.default_rng(3)
    fields = rng.normal(size=(6, 5 * 5))
    kappa = o.PixelField(np.exp(rng.normal(size=(12, 10))), (0.25, 0.4), (-1.0, -2.0))
    flux = o.cartesian_flux(mesh, 4, fields, kappa)
    for c in range(6):
        assert np.array_equal(flux[c], o.cell_flux(mesh.submesh(c, 4), fields[c], kappa))
