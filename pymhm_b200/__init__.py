"""B200-native Primal-MHM hot path (Cartesian Q1 Darcy) behind PyMHM's provider API.

Public entry points:

* ``solve_darcy_quadrilateral`` / ``CartesianQ1Plan`` - the whole local/global solve
  on one GPU (``pymhm_b200.darcy``);
* ``BatchedFactorization``, ``condense_batched``, ``GpuLocalSolver`` - drop-ins for the
  reference's batched GPU local algebra and ``LocalLinearSolver`` protocol
  (``pymhm_b200.batched``);
* ``SkeletonFactorization`` - a ``LinearFactorization``-style global solver for
  ``HybridSystem.solve(factorization=...)`` (``pymhm_b200.skeleton``);
* ``OfflineQ1System`` - factors kept for repeated sources (``pymhm_b200.offline``);
* ``refine_hybrid`` / ``CartesianQ1Plan.refine`` - defect correction of the original
  uncondensed equations (``pymhm_b200.darcy``).

Compute runs in ``libmhm_b200.so`` (hand-written sm_100a CUDA behind a C ABI);
importing this package does not touch the GPU.
"""

from .errors import LinearSolveError, SolverUnavailableError
from .topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

__all__ = [
    "CartesianMacroMesh", "FaceSpace", "SkeletonSpace", "LinearSolveError", "SolverUnavailableError",
    "solve_darcy_quadrilateral", "CartesianQ1Plan", "BatchedFactorization", "condense_batched",
    "GpuLocalSolver", "SkeletonFactorization", "OfflineQ1System", "refine_hybrid", "HybridRefinement",
]


def __getattr__(name):
    if name in ("solve_darcy_quadrilateral", "CartesianQ1Plan", "Q1Solution", "refine_hybrid", "HybridRefinement"):
        from . import darcy

        return getattr(darcy, name)
    if name in ("BatchedFactorization", "condense_batched", "GpuLocalSolver"):
        from . import batched

        return getattr(batched, name)
    if name == "OfflineQ1System":
        from . import offline

        return offline.OfflineQ1System
    if name == "SkeletonFactorization":
        from . import skeleton

        return skeleton.SkeletonFactorization
    raise AttributeError(name)
