"""CPU oracle for the Cartesian Q1 Primal-MHM hot path (test infrastructure).

This package is the checker, not the product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline arm may import it.
It restates PyMHM 1.3.2's NumPy/SciPy path (each function cites the reference
file and line it follows) and is pinned against golden fixtures produced by the
reference itself (``tests/golden/make_golden.py``).
"""
