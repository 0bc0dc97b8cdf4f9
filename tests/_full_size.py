"""The full-size Cartesian workload (64x64 macrocells x 16x16 Q1, P2 faces, lognormal
kappa) solved once per test process by the oracle, which is the checker at that size.

The fixture written by the reference keeps only digests, norms and three cells at this
size; the oracle's solve reproduces the reference's matrix bit for bit (its SHA-256
digests) and its trace and coarse unknowns exactly, so its full fields and fluxes stand
in for the reference's (pinned in ``tests/test_oracle_golden.py``).
"""

import os

import numpy as np
from scipy import sparse

_CACHE = {}


def workload_kappa():
    from pymhm_b200.workloads import lognormal_permeability

    return lognormal_permeability(1024, 1024, sigma=2.0, ell=0.05, seed=20261203)


def oracle_solution():
    """Oracle solve of the full-size workload on a spawn pool (about 15 s on 8 cores)."""
    if "sol" not in _CACHE:
        from oracle.q1_mhm import CartesianSolve

        workers = max(1, min(os.cpu_count() or 1, 32))
        with CartesianSolve(64, 16, 2, workload_kappa(), 1.0, workers=workers) as solver:
            _CACHE["sol"] = solver.solve()
    return _CACHE["sol"]


def stored_values(m, rows, cols):
    """Values of the stored entries (row, col) of a CSR matrix, 0 where none is stored."""
    out = np.zeros(len(rows))
    for k, (i, j) in enumerate(zip(rows, cols)):
        lo, hi = m.indptr[i], m.indptr[i + 1]
        p = lo + np.searchsorted(m.indices[lo:hi], j)
        if p < hi and m.indices[p] == j:
            out[k] = m.data[p]
    return out


def pattern_differences(mine, ref):
    """Entries stored by exactly one of two sparse matrices: (rows, cols, |mine|, |ref|)."""
    a = sparse.csr_matrix(mine)
    b = sparse.csr_matrix(ref)
    a.sort_indices()
    b.sort_indices()
    ones_a, ones_b = a.copy(), b.copy()
    ones_a.data[:] = 1.0
    ones_b.data[:] = 1.0
    only = (ones_a - ones_a.multiply(ones_b)) + (ones_b - ones_b.multiply(ones_a))
    r, c = only.nonzero()
    return r, c, np.abs(stored_values(a, r, c)), np.abs(stored_values(b, r, c))
