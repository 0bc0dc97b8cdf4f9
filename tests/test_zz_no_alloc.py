"""The allocation-free global solve (mhm_skeleton_solve_static) against the regular one.

Some callers of this library cannot allocate device memory: a C or Fortran
host code that reaches it only through the C ABI without a CUDA allocator of
its own, or a serving process that reserves all device memory at start-up and
must not call cudaMalloc/cudaFree afterwards.  For them the global skeleton
solve also exists with its scratch in a fixed 4 MiB device array inside the
library.  This test calls that entry point through the C ABI, twice in a row
(the second call reuses the array with the first call's leftovers), and checks
both results against the entry point that takes caller-allocated scratch.
Collected last so a failure here never hides the other tests.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_static_scratch_solve_matches_workspace_solve():
    import torch

    from pymhm_b200 import _lib
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import lognormal_permeability

    mesh = CartesianMacroMesh(16)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, 8, precision="fp64")
    plan.set_coefficients(lognormal_permeability(128, 128, seed=11), 1.0)
    plan.launch(reconstruct=False)
    plan.check()
    reference = plan.x.cpu().numpy()
    lib = _lib.load()
    need = lib.mhm_skeleton_workspace_bytes(plan.sys, plan.grid)
    assert 0 < need <= 4 << 20
    P = _lib.ptr
    stream = _lib.stream_handle(None)
    for call in range(2):
        x = torch.full_like(plan.x, float("nan"))
        info = torch.full((4,), -1, dtype=torch.int32, device=plan.device)
        stats = torch.zeros(4, dtype=torch.float64, device=plan.device)
        rc = lib.mhm_skeleton_solve_static(plan.sys, P(plan.rhs), P(plan.load_scale), P(x), plan.global_rtol,
                                           plan.inner_rtol, plan.max_inner, plan.max_outer, plan.grid, P(info),
                                           P(stats), stream)
        assert rc == _lib.MHM_OK
        torch.cuda.synchronize()
        assert int(info[0]) == _lib.SOLVE_OK, f"call {call}: status {int(info[0])}"
        got = x.cpu().numpy()
        assert np.linalg.norm(got - reference) <= 1e-10 * np.linalg.norm(reference), f"call {call}"
        assert float(stats[1]) <= 1e-12


def test_static_scratch_rejects_oversized_systems():
    from pymhm_b200 import _lib
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    mesh = CartesianMacroMesh(128)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, 2, precision="fp64")
    lib = _lib.load()
    assert lib.mhm_skeleton_workspace_bytes(plan.sys, plan.grid) > 4 << 20
    rc = lib.mhm_skeleton_solve_static(plan.sys, _lib.ptr(plan.rhs), 0, _lib.ptr(plan.x), 1e-13, 1e-12, 10, 2,
                                       plan.grid, _lib.ptr(plan.info), _lib.ptr(plan.stats),
                                       _lib.stream_handle(None))
    assert rc == _lib.MHM_ERR_UNSUPPORTED
