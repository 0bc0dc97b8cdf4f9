"""The global skeleton solver for macro meshes of any shape (``mhm_general_solve``),
checked on the Cartesian systems whose reference solutions the fixtures hold: the
same reduced system solved without the Cartesian coarse structure."""

import numpy as np
import pytest

from tests._cases import CASES, load, rel

pytestmark = pytest.mark.gpu


def general_for(plan):
    from pymhm_b200.general import GeneralSkeleton
    from pymhm_b200.topology import geometric_constraint

    space_h, space_v = plan.skeleton.uniform_by_orientation()
    g0 = geometric_constraint(plan.mesh, space_h, space_v)
    return GeneralSkeleton(plan.cell_dofs_h, g0, plan.skeleton.offsets, plan.T, plan.pattern.indptr,
                           plan.pattern.indices)


@pytest.mark.parametrize("name", list(CASES))
def test_general_solver_matches_reference_on_cartesian_systems(name):
    import torch

    from tests.test_gpu_darcy import make_plan

    g, plan = make_plan(name, "fp64")
    plan.launch()
    plan.check()
    gs = general_for(plan)
    x = torch.empty_like(plan.x)
    gs.launch(plan.values, plan.rhs, x)
    info, stats = gs.check()
    xh = x.cpu().numpy()
    assert stats[0] <= 1e-13
    assert rel(xh[: plan.T], g["trace"]) <= 1e-10
    assert rel(xh[plan.T:], g["coarse"]) <= 1e-10
    assert rel(xh, plan.x.cpu().numpy()) <= 1e-11
    # bitwise reproducible
    x2 = torch.empty_like(x)
    gs.launch(plan.values, plan.rhs, x2)
    gs.check()
    assert bool((x2 == x).all())


def test_general_factorization_on_the_reference_matrix():
    """``GeneralFactorization`` (LinearFactorization contract) given the reference's own
    assembled matrix (post-eliminate_zeros CSC) and right-hand side."""
    from scipy import sparse

    from pymhm_b200.general import GeneralFactorization
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace, geometric_constraint

    g = load("darcy_4x4_r16_p2_lognormal")
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    N = sk.size + len(mesh.cells)
    K = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    g0 = geometric_constraint(mesh, *sk.uniform_by_orientation())
    with GeneralFactorization(K, list(sk.cell_dof_array), list(g0), sk.offsets) as f:
        assert f.matches(K) and not f.matches(2 * K)
        x = f.solve(g["rhs"])
        both = f.solve(np.column_stack((g["rhs"], 2 * g["rhs"])))
    assert rel(x[: sk.size], g["trace"]) <= 1e-10
    assert rel(x[sk.size:], g["coarse"]) <= 1e-10
    assert rel(both[:, 1], 2 * x) <= 1e-12


def test_general_solver_full_size():
    """The 64x64 x 16x16 lognormal system: the general solver against the reference."""
    import torch

    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from tests._full_size import workload_kappa

    g = load("darcy_64x64_r16_p2_lognormal")
    mesh = CartesianMacroMesh(64)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, 16, precision="fp64")
    plan.set_coefficients(workload_kappa(), 1.0)
    plan.launch()
    plan.check()
    gs = general_for(plan)
    x = torch.empty_like(plan.x)
    gs.launch(plan.values, plan.rhs, x)
    info, stats = gs.check()
    xh = x.cpu().numpy()
    assert rel(xh[: plan.T], g["trace"]) <= 1e-10
    assert rel(xh[plan.T:], g["coarse"]) <= 1e-10
