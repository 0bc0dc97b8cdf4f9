"""GPU parity of the Cartesian Q1 path against the reference fixtures and the oracle."""

import numpy as np
import pytest

from tests._cases import face_space, CASES, load, rel

pytestmark = pytest.mark.gpu

# tolerances on relative L2 error against the reference's FP64 SuperLU solution
TOL = {"fp64": 1e-10, "mixed": 1e-8}


def make_plan(name, precision, **kw):
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    g = load(name)
    margs, face, ref, perm, src, dr = CASES[name]
    mesh = CartesianMacroMesh(*margs)
    sk = SkeletonSpace(mesh, (face_space(FaceSpace, face),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, ref, dirichlet=dr, precision=precision, **kw)
    plan.set_coefficients(perm(g), src)
    return g, plan


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_solution_matches_reference(name, precision):
    g, plan = make_plan(name, precision)
    plan.launch()
    sol = plan.result()
    tol = TOL[precision]
    assert rel(sol.trace, g["trace"]) <= tol
    assert rel(sol.coarse, g["coarse"]) <= tol
    assert rel(sol.fields, g["fields"]) <= tol
    assert rel(sol.flux, g["flux"]) <= tol
    assert sol.residual <= 1e-12
    assert np.array_equal(sol.corrected, g["corrected"]) or name == "poisson_8x8_r4_p1"


@pytest.mark.parametrize("name", list(CASES))
def test_cell_responses_and_blocks(name):
    g, plan = make_plan(name, "fp64")
    plan.launch()
    plan.check()
    n = plan.n
    for c in g["keep_cells"]:
        sol = plan.solution[c].cpu().numpy()
        assert rel(sol[1:-1, :n].T, g[f"cell{c}_lifts"]) <= 1e-10
        assert rel(1.0 - sol[-1, :n], g[f"cell{c}_retained"]) <= 1e-12
        blk, ref = plan.blocks[c].cpu().numpy(), g[f"cell{c}_block"]
        assert np.max(np.abs(blk - ref)) <= 1e-10 * np.max(np.abs(ref))
        ld, refl = plan.loads[c].cpu().numpy(), g[f"cell{c}_load"]
        assert np.max(np.abs(ld - refl)) <= 1e-10 * max(np.max(np.abs(refl)), 1e-300) + 1e-18


# An entry the reference drops (exact zero after summation) that this solve keeps, or
# the other way round, must be a rounding residue on both sides: every such entry is a
# quantity that is zero in exact arithmetic (a face moment of a Legendre mode >= 1
# against the nearly constant retained column, a symmetry-zero coupling), whose
# computed value is rounding of that side's local solves.
ROUNDING = 1e-15


def assert_reference_sparsity(A, ref):
    """The exported CSC equals the reference's post-``eliminate_zeros`` matrix: the same
    index arrays where both keep the same entries; otherwise the entries kept by one
    side only are rounding residues on both sides."""
    from tests._full_size import pattern_differences

    scale = np.max(np.abs(ref.data))
    r, c, mine, theirs = pattern_differences(A, ref)
    assert np.all(mine <= ROUNDING * scale) and np.all(theirs <= ROUNDING * scale)
    if len(r) == 0:
        assert np.array_equal(A.indptr, ref.indptr) and np.array_equal(A.indices, ref.indices)
    return len(r), A.nnz, ref.nnz


@pytest.mark.parametrize("name", list(CASES))
def test_skeleton_matrix_sparsity_and_values(name):
    """The exported matrix (CSC, exact zeros dropped on the device) against the
    reference's ``indptr`` / ``indices`` / ``data`` arrays of the fixture."""
    from scipy import sparse

    g, plan = make_plan(name, "fp64")
    plan.launch()
    plan.check()
    A = plan.matrix()
    N = plan.N
    assert A.format == "csc" and A.indices.dtype == g["indices"].dtype
    ref = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    diff = (A - ref).toarray()
    assert np.max(np.abs(diff)) <= 1e-10 * np.max(np.abs(ref.data))
    assert not np.any(A.data == 0.0)
    assert np.all(np.diff(A.indptr) >= 0) and A.has_sorted_indices
    assert_reference_sparsity(A, ref)
    assert rel(plan.rhs.cpu().numpy(), g["rhs"]) <= 1e-10


def test_deterministic_bitwise():
    _, plan = make_plan("darcy_4x4_r16_p2_lognormal", "mixed")
    plan.launch()
    a = (plan.x.clone(), plan.values.clone(), plan.fields.clone())
    plan.launch()
    plan.check()
    b = (plan.x, plan.values, plan.fields)
    for u, v in zip(a, b):
        assert bool((u == v).all())


def test_full_size_workload_matches_reference():
    """64x64 macrocells x 16x16 Q1, lognormal kappa: the benchmarked workload.  Relative
    L2 errors over all 4096 cells of u and the flux against the oracle's solve (which
    reproduces the reference's matrix digests and unknowns exactly), of lambda and c
    against the reference's fixture, and the exported sparsity against the
    reference's matrix."""
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import digest
    from tests._full_size import oracle_solution, workload_kappa

    g = load("darcy_64x64_r16_p2_lognormal")
    ref = oracle_solution()
    mesh = CartesianMacroMesh(64)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    kappa = workload_kappa()
    for precision in ("fp64", "mixed"):
        plan = CartesianQ1Plan(mesh, sk, 16, precision=precision)
        plan.set_coefficients(kappa, 1.0)
        plan.launch()
        sol = plan.result()
        tol = TOL[precision]
        assert rel(sol.trace, g["trace"]) <= tol
        assert rel(sol.coarse, g["coarse"]) <= tol
        assert rel(sol.fields, ref["fields"]) <= tol
        assert rel(sol.flux, ref["flux"]) <= tol
        keep = list(g["keep_cells"])
        assert rel(sol.fields[keep], g["fields_cells"]) <= tol
        assert rel(sol.flux[keep], g["flux_cells"]) <= tol
        assert np.array_equal(sol.corrected, g["corrected"])
        if precision == "fp64":
            A = plan.matrix()
            assert digest(ref["matrix"].indptr) == str(g["indptr_sha256"])
            assert_reference_sparsity(A, ref["matrix"])


def test_exact_pressure_convergence_sanity():
    """Manufactured sine solution: the discrete pressure approximates sin(pi x) sin(pi y)."""
    from pymhm_b200.darcy import solve_darcy_quadrilateral
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import sine_source

    errs = []
    for macro in (4, 8):
        mesh = CartesianMacroMesh(macro)
        sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
        sol = solve_darcy_quadrilateral(mesh, skeleton=sk, local_refinement=8, source=sine_source)
        nodes = []
        for c in range(len(mesh.cells)):
            x0, y0 = mesh.points[mesh.cells[c, 0]]
            hx, hy = mesh.spacing
            xs = x0 + np.linspace(0, hx, 9)
            ys = y0 + np.linspace(0, hy, 9)
            X, Y = np.meshgrid(xs, ys)
            nodes.append(np.sin(np.pi * X) * np.sin(np.pi * Y))
        exact = np.array(nodes).reshape(len(mesh.cells), -1)
        errs.append(np.max(np.abs(sol.fields - exact)))
    assert errs[1] < errs[0] / 3
    assert errs[1] < 5e-3


def test_failures_are_reported_not_hidden():
    """Host-made failures: too few refinement sweeps and a capped global solve."""
    from pymhm_b200.errors import LinearSolveError

    _, plan = make_plan("darcy_4x4_r16_p2_lognormal", "mixed", max_refine=1)
    plan.launch()
    with pytest.raises(LinearSolveError, match="residual"):
        plan.check()
    _, plan = make_plan("darcy_4x4_r16_p2_lognormal", "fp64", max_inner=2)
    plan.launch()
    with pytest.raises(LinearSolveError, match="converge"):
        plan.check()
