"""Exceptions mirroring PyMHM's (``src/pymhm/linalg/linear.py:32-41``).

Messages reuse the reference wording ("singular pivot", "rank deficient",
"residual", "nonfinite", "zero row", "zero column") so callers that match on
them behave the same.
"""


class LinearSolveError(RuntimeError):
    """A factorization, iteration, or independently checked residual failed."""


class SolverUnavailableError(ImportError):
    """The CUDA library or a CUDA device is not available (there is no CPU fallback)."""
