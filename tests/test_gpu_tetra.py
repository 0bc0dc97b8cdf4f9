"""GPU parity of the 3D P1 tetrahedral path against fixtures written by the reference
(``make_tetra_golden.py``) and against the oracle on a larger mesh."""

import numpy as np
import pytest

from tests._cases import load, rel
from tests.test_oracle_tetra import TETRA_CASES, tetra_case

pytestmark = pytest.mark.gpu


def plan_for(name):
    from pymhm_b200.tetra_darcy import TetraP1Plan

    g, mesh, sk, r, field = tetra_case(name)
    plan = TetraP1Plan(mesh, sk, r)
    plan.set_coefficients(field, 1.0)
    return g, plan


@pytest.mark.parametrize("name", list(TETRA_CASES))
def test_tetra_solution_matches_reference(name):
    g, plan = plan_for(name)
    plan.launch()
    sol = plan.result()
    assert rel(sol.trace, g["trace"]) <= 1e-10
    assert rel(sol.coarse, g["coarse"]) <= 1e-10
    assert rel(sol.fields, g["fields"]) <= 1e-10
    assert sol.residual <= 1e-12
    assert np.array_equal(sol.corrected, g["corrected"])
    # per-cell responses and contributions of the kept cells
    n = plan.n
    for c in g["keep_cells"]:
        X = plan.solution[c].cpu().numpy()
        assert rel(X[:n, 1:plan.t + 1], g[f"cell{c}_lifts"]) <= 1e-10
        assert rel(1.0 - X[:n, -1], g[f"cell{c}_retained"]) <= 1e-12
        blk, ref = plan.blocks[c].cpu().numpy(), g[f"cell{c}_block"]
        assert np.max(np.abs(blk - ref)) <= 1e-10 * np.max(np.abs(ref))
        ld, refl = plan.loads[c].cpu().numpy(), g[f"cell{c}_load"]
        assert np.max(np.abs(ld - refl)) <= 1e-10 * np.max(np.abs(refl))
        assert np.allclose(plan.stiffness[c].cpu().numpy(), g[f"cell{c}_A"], rtol=0,
                           atol=1e-13 * np.max(np.abs(g[f"cell{c}_A"])))


@pytest.mark.parametrize("name", list(TETRA_CASES))
def test_tetra_matrix_against_reference(name):
    from scipy import sparse

    from tests.test_gpu_darcy import assert_reference_sparsity

    g, plan = plan_for(name)
    plan.launch()
    plan.check()
    A = plan.matrix()
    ref = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(plan.N, plan.N))
    assert np.max(np.abs((A - ref).toarray())) <= 1e-10 * np.max(np.abs(ref.data))
    assert_reference_sparsity(A, ref)
    assert rel(plan.grhs.cpu().numpy(), g["rhs"]) <= 1e-10


def test_tetra_deterministic_bitwise():
    _, plan = plan_for("tetra_cube2_r4_p1_layered")
    plan.launch()
    a = (plan.x.clone(), plan.values.clone(), plan.fields.clone())
    plan.launch()
    plan.check()
    for u, v in zip(a, (plan.x, plan.values, plan.fields)):
        assert bool((u == v).all())


def test_tetra_larger_mesh_against_oracle():
    """162 macro tetrahedra (unit cube 3^3), 35 local nodes, 8 layers: the oracle's solve."""
    from oracle import tetra_mhm as ot
    from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
    from pymhm_b200.tetra_darcy import TetraP1Plan
    from pymhm_b200.workloads import LayeredField, layered_lognormal_permeability

    mesh = TetraMesh.unit_cube(3)
    sk = TriangularSkeleton(mesh, 1)
    field = LayeredField(layered_lognormal_permeability(8, 16, sigma=3.0, ell=0.1, contrast=1e6, seed=5))
    ref = ot.solve_darcy_p1(mesh, sk, 4, field, 1.0)
    plan = TetraP1Plan(mesh, sk, 4)
    sol = plan.solve(field, 1.0)
    assert rel(sol.trace, ref["trace"]) <= 1e-10
    assert rel(sol.coarse, ref["coarse"]) <= 1e-10
    assert rel(sol.fields, ref["fields"]) <= 1e-10


def test_solve_darcy_3d_drop_in():
    from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
    from pymhm_b200.tetra_darcy import solve_darcy_3d

    g, mesh, sk, r, field = tetra_case("tetra_cube2_r4_p1_layered")
    sol = solve_darcy_3d(mesh, permeability=field, source=1.0, skeleton=sk, local_refinement=r, degree=1)
    assert rel(sol.fields, g["fields"]) <= 1e-10
    with pytest.raises(NotImplementedError):
        solve_darcy_3d(mesh, permeability=field, source=1.0, skeleton=sk, local_refinement=r, degree=2)
    with pytest.raises(NotImplementedError):
        solve_darcy_3d(TetraMesh.unit_cube(1), dirichlet=1.0, skeleton=None, degree=1)


def test_tetra_preconditioners_agree():
    """Cell-Dirichlet (the cells' D S^-1 D) and face block-Jacobi preconditioning reach
    the same solution; the cell preconditioner in fewer iterations."""
    from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
    from pymhm_b200.tetra_darcy import TetraP1Plan
    from pymhm_b200.workloads import LayeredField, layered_lognormal_permeability

    mesh = TetraMesh.unit_cube(3)
    sk = TriangularSkeleton(mesh, 1)
    field = LayeredField(layered_lognormal_permeability(8, 16, sigma=3.0, ell=0.1, contrast=1e6, seed=5))
    sols = {}
    for pc in ("cell", "face"):
        plan = TetraP1Plan(mesh, sk, 4, preconditioner=pc)
        sols[pc] = plan.solve(field, 1.0)
        assert sols[pc].residual <= 1e-12
    assert rel(sols["cell"].trace, sols["face"].trace) <= 1e-11
    assert rel(sols["cell"].fields, sols["face"].fields) <= 1e-11
    assert sols["cell"].global_iterations < sols["face"].global_iterations


def test_tetra_pivoting_variants_agree():
    """The windowed-pivot LU (default) and full partial pivoting give the same 3D
    solution to rounding."""
    from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
    from pymhm_b200.tetra_darcy import TetraP1Plan
    from pymhm_b200.workloads import LayeredField, layered_lognormal_permeability

    mesh = TetraMesh.unit_cube(3)
    sk = TriangularSkeleton(mesh, 1)
    field = LayeredField(layered_lognormal_permeability(12, 16, sigma=3.0, ell=0.1, contrast=1e6, seed=31))
    a = TetraP1Plan(mesh, sk, 4).solve(field, 1.0)
    b = TetraP1Plan(mesh, sk, 4, lu="partial").solve(field, 1.0)
    assert rel(a.trace, b.trace) <= 1e-11
    assert rel(a.fields, b.fields) <= 1e-11
