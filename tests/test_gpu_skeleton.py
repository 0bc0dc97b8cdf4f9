"""SkeletonFactorization (LinearFactorization contract) on the oracle's assembled system."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_skeleton_factorization_solves_reference_matrix():
    from scipy import sparse

    from pymhm_b200.skeleton import SkeletonFactorization
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from tests._cases import load, rel

    g = load("darcy_4x4_r16_p2_lognormal")
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    N = sk.size + len(mesh.cells)
    A = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    with SkeletonFactorization(A, mesh, sk) as f:
        assert f.matches(A)
        B = A.copy()
        B.data[0] += 1.0
        assert not f.matches(B)
        x = f.solve(g["rhs"])
        assert rel(x[: sk.size], g["trace"]) <= 1e-10
        assert rel(x[sk.size:], g["coarse"]) <= 1e-10
        two = f.solve(np.column_stack((g["rhs"], 2 * g["rhs"])))
        assert rel(two[:, 1], 2 * x) <= 1e-12
    with pytest.raises(RuntimeError, match="closed"):
        f.solve(g["rhs"])


@pytest.mark.parametrize("cell_blocks", [False, True])
def test_solution_carried_by_coarse_unknowns_alone(cell_blocks):
    """A right-hand side whose solution has zero trace part: the projected inner
    residual starts at rounding level, and the solve must stop instead of breaking
    down (the case of an original-equation correction of a shifted field)."""
    from scipy import sparse

    from pymhm_b200.skeleton import SkeletonFactorization
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from tests._cases import load

    g = load("darcy_4x4_r16_p2_lognormal")
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    N = sk.size + len(mesh.cells)
    A = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    want = np.r_[np.zeros(sk.size), 0.002 * np.arange(1, len(mesh.cells) + 1)]
    b = A @ want
    if cell_blocks:
        from tests.test_gpu_darcy import make_plan

        _, plan = make_plan("darcy_4x4_r16_p2_lognormal", "fp64")
        plan.launch()
        plan.check()
        import torch

        plan.rhs.copy_(torch.from_numpy(b).to(plan.device))
        plan.load_scale.zero_()
        from pymhm_b200 import _lib

        P = _lib.ptr
        _lib.check(plan.lib.mhm_skeleton_solve(plan.sys, P(plan.rhs), P(plan.load_scale), P(plan.x),
                                               plan.global_rtol, plan.inner_rtol, plan.max_inner, plan.max_outer,
                                               plan.grid, P(plan.workspace), plan.workspace.numel(), P(plan.info),
                                               P(plan.stats), None), "mhm_skeleton_solve")
        plan.check()
        x = plan.x.cpu().numpy()
    else:
        with SkeletonFactorization(A, mesh, sk) as f:
            x = f.solve(b)
    assert np.max(np.abs(x - want)) <= 1e-12 * np.max(np.abs(want))
