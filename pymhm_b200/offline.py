"""Offline / online reuse of the Cartesian Q1 path for repeated sources.

``OfflineQ1System`` is the GPU counterpart of ``OfflineHybridSystem``
(``src/pymhm/core/offline.py:148-313``) for Cartesian Q1 Darcy: it keeps every
macrocell's factor (the inverses of its line Schur complements) and the
source-independent responses (lifts and the retained response) resident in
HBM, together with the Schur blocks and the assembled skeleton matrix.  Each
online query changes the source only: the cells' source responses are solved
with the kept factors, the reduced right-hand side is rebuilt, and the global
solve runs on the unchanged skeleton matrix.

The reference's ``solve(loads)`` takes one assembled load vector per local
problem; this path assembles the loads on the GPU, so ``solve(source)`` takes
the source itself (a constant, a callable of points, or an array on the fine
grid, as ``CartesianQ1Plan.set_coefficients``).  Like the reference, online
queries may not change the material, the mesh or the spaces.
"""

from __future__ import annotations

from .darcy import CartesianQ1Plan, Q1Solution


class OfflineQ1System:
    """Prepare a fixed Cartesian Q1 discretization for many source queries."""

    def __init__(self, mesh, skeleton=None, local_refinement=4, *, permeability=1.0, source=0.0,
                 precision="fp64", **plan_options) -> None:
        self.plan = CartesianQ1Plan(mesh, skeleton, local_refinement, precision=precision, **plan_options)
        self.plan.set_coefficients(permeability, source)
        self.plan.prepare_offline()
        self.prepared = self.plan.result()
        self._closed = False

    def solve(self, source) -> Q1Solution:
        """One new source query without refactoring (``offline.py:231-307``)."""
        if self._closed:
            raise RuntimeError("offline system is closed")
        return self.plan.solve_source(source)

    def solve_many(self, sources) -> tuple[Q1Solution, ...]:
        """Evaluate source cases in order while keeping all offline resources."""
        return tuple(self.solve(case) for case in sources)

    def close(self) -> None:
        """Release the kept factors; repeated calls are safe."""
        if not self._closed:
            self._closed = True
            self.plan.factors = None

    def __enter__(self) -> "OfflineQ1System":
        if self._closed:
            raise RuntimeError("offline system is closed")
        return self

    def __exit__(self, *exc) -> None:
        self.close()
