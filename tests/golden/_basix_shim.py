"""Clean-room stand-in for the two Basix tabulations the Cartesian Q1 path uses.

Fixture generation only: this module is imported by ``make_golden.py`` in a
development checkout, never by the library, the oracle or the GPU tests.

PyMHM 1.3.2 reaches Basix (``fenics-basix`` 0.11.0 pinned in the project's
``pixi.lock``) only through ``pymhm.fem.reference``.  The Cartesian Qk path
calls two of its functions:

* ``simplex_lagrange_tabulation("interval", k, bary, nodes=..., nderiv)``
  (``src/pymhm/fem/reference.py:497-540``) from ``_cardinal_values``
  (``src/pymhm/fem/scalar/quadrilateral.py:58-68``) and continuous faces;
* ``legendre_values`` / ``legendre_tabulation``
  (``src/pymhm/fem/reference.py:596-625``) from ``FaceSpace.evaluate``
  (``src/pymhm/fem/traces/interval.py:54-89``).

The P1 operator fixtures (``make_p1_golden.py``) also need the degree-one
Lagrange basis on triangles and tetrahedra (barycentric coordinates).

The tetrahedral fixtures (``make_tetra_golden.py``) need the Bernstein basis of the
triangular skeleton faces too.

The mixed RT0 fixtures (``make_polygon_rt0_golden.py``) need a basis of the lowest
Raviart-Thomas space on the reference triangle (``vector_tabulation("RT", "triangle",
1, ...)``, ``src/pymhm/fem/hdiv/reference.py:18-37``).  The reference turns whatever
candidate basis it gets into its canonical face-moment basis by exact moments
(``rt_moment_coefficients``, ``src/pymhm/fem/hdiv/rt.py:64-88``), so any basis of
RT0 = {a + b x} gives the same result up to rounding: here (x, y), (x - 1, y),
(x, y - 1), each of divergence 2.

All are restated here from their published mathematics: the nodal Lagrange
basis on the declared node order (unique polynomial interpolant, obtained by a
Legendre-Vandermonde solve) with exact Kronecker rows at literal nodes, as the
reference wrapper enforces (``reference.py:484-488``); and the conventional
Legendre polynomials ``L_j(1)=1`` by the three-term recurrence.
"""

from __future__ import annotations

import numpy as np
from numpy.polynomial import legendre as npleg


def _interval_lagrange(degree, points, nodes, nderiv):
    x = np.asarray(points, dtype=float)
    c = np.asarray(nodes, dtype=float)
    # Vandermonde in shifted Legendre polynomials on [0, 1]: V[i, j] = P_j(2 c_i - 1)
    vand = npleg.legvander(2 * c - 1, degree)
    coef = np.linalg.solve(vand, np.eye(degree + 1))  # column j: coefficients of phi_j
    vals = npleg.legvander(2 * x - 1, degree) @ coef
    ders = np.zeros_like(vals)
    if nderiv:
        for j in range(degree + 1):
            d = npleg.legder(coef[:, j]) * 2.0
            ders[:, j] = npleg.legval(2 * x - 1, d) if len(d) else 0.0
    rows, cols = np.nonzero(x[:, None] == c[None, :])
    vals[rows] = 0.0
    vals[rows, cols] = 1.0
    return vals, ders


def _simplex_p1(bary, nodes, nderiv):
    """Degree-one Lagrange basis on a triangle or tetrahedron for the declared node
    order: phi_j = sum_m bary_m C[m, j] with C the inverse of the nodes' barycentric
    matrix (phi_j(node_k) = delta_jk); gradients in the reference coordinates
    x = bary[:, 1:] are C[a + 1, j] - C[0, j]; Hessians vanish."""
    dim = nodes.shape[1] - 1
    coef = np.linalg.inv(nodes)
    vals = bary @ coef
    rows, cols = np.nonzero(np.all(bary[:, None, :] == nodes[None, :, :], axis=2))
    vals[rows] = 0.0
    vals[rows, cols] = 1.0
    grad = np.broadcast_to((coef[1:] - coef[0]).T, (len(bary), nodes.shape[0], dim)).copy()
    gradient = grad if nderiv else np.empty((*vals.shape, 0))
    hessian = np.zeros((*vals.shape, dim, dim)) if nderiv == 2 else np.empty((*vals.shape, 0, 0))
    return vals, gradient, hessian


def _triangle_lagrange(degree, bary, nodes, nderiv):
    """Degree-k nodal Lagrange basis on a triangle for the declared nodes (barycentric
    rows): the unique polynomial interpolant, from a monomial Vandermonde solve in the
    reference coordinates (x, y) = (lambda_1, lambda_2), with exact Kronecker rows at the
    nodes; gradients and Hessians in (x, y)."""
    powers = [(i, j) for i in range(degree + 1) for j in range(degree + 1 - i)]
    nx, ny = nodes[:, 1], nodes[:, 2]
    vand = np.array([[x ** i * y ** j for (i, j) in powers] for x, y in zip(nx, ny)])
    coef = np.linalg.solve(vand, np.eye(len(powers)))  # column m: coefficients of phi_m
    x, y = bary[:, 1], bary[:, 2]

    def mono(dx, dy):
        out = np.zeros((len(x), len(powers)))
        for k, (i, j) in enumerate(powers):
            if i < dx or j < dy:
                continue
            ci = np.prod(range(i - dx + 1, i + 1)) if dx else 1.0
            cj = np.prod(range(j - dy + 1, j + 1)) if dy else 1.0
            out[:, k] = ci * cj * x ** (i - dx) * y ** (j - dy)
        return out

    vals = mono(0, 0) @ coef
    rows, cols = np.nonzero(np.all(bary[:, None, :] == nodes[None, :, :], axis=2))
    vals[rows] = 0.0
    vals[rows, cols] = 1.0
    grad = np.stack((mono(1, 0) @ coef, mono(0, 1) @ coef), axis=-1) if nderiv else np.empty((*vals.shape, 0))
    if nderiv == 2:
        hess = np.empty((*vals.shape, 2, 2))
        hess[..., 0, 0] = mono(2, 0) @ coef
        hess[..., 0, 1] = hess[..., 1, 0] = mono(1, 1) @ coef
        hess[..., 1, 1] = mono(0, 2) @ coef
    else:
        hess = np.empty((*vals.shape, 0, 0))
    return vals, grad, hess


def simplex_lagrange_tabulation(cell, degree, bary, *, nodes, nderiv=2):
    bary = np.asarray(bary, dtype=float)
    nodes = np.asarray(nodes, dtype=float)
    if cell in ("triangle", "tetrahedron") and int(degree) == 1:
        return _simplex_p1(bary, nodes, nderiv)
    if cell == "triangle":
        return _triangle_lagrange(int(degree), bary, nodes, nderiv)
    if cell != "interval":
        raise NotImplementedError("the fixture shim covers intervals, triangles and degree-one tetrahedra")
    vals, ders = _interval_lagrange(int(degree), bary[:, 1], nodes[:, 1], nderiv)
    gradient = ders[:, :, None] if nderiv else np.empty((*vals.shape, 0))
    hessian = np.empty((*vals.shape, 0, 0))
    return vals, gradient, hessian


def legendre_tabulation(points, degree, nderiv=0):
    x = np.asarray(points, dtype=float)
    out = np.zeros((nderiv + 1, *x.shape, degree + 1))
    for j in range(degree + 1):
        e = np.zeros(degree + 1)
        e[j] = 1.0
        out[0, ..., j] = npleg.legval(x, e)
        for d in range(1, nderiv + 1):
            e = npleg.legder(e)
            out[d, ..., j] = npleg.legval(x, e) if len(e) else 0.0
    return out


def legendre_values(points, degree):
    return legendre_tabulation(points, degree)[0]


def bernstein_tabulation(points, exponents):
    """Simplex Bernstein polynomials B_alpha = (k! / alpha!) prod_a lambda_a^alpha_a of
    degree k = |alpha| in the declared exponent order, lambda = (1 - sum x, x) for the
    reference coordinates x; values (points, modes) and Cartesian gradients
    (points, modes, dim).  Replaces ``pymhm.fem.reference.bernstein_tabulation``
    (``reference.py:744-760``), which tabulates the same basis through Basix."""
    from math import factorial

    x = np.asarray(points, dtype=float)
    lam = np.column_stack((1 - x.sum(axis=1), x))
    dim = x.shape[1]
    vals = np.empty((len(x), len(exponents)))
    grads = np.zeros((len(x), len(exponents), dim))
    for m, alpha in enumerate(exponents):
        k = sum(alpha)
        coef = factorial(k) / np.prod([factorial(a) for a in alpha])
        vals[:, m] = coef * np.prod([lam[:, a] ** p for a, p in enumerate(alpha)], axis=0)
        # d lambda_0 / d x_i = -1, d lambda_{i+1} / d x_i = 1
        dl = np.zeros((len(x), dim + 1))
        for a, p in enumerate(alpha):
            if p == 0:
                continue
            rest = np.prod([lam[:, b] ** q for b, q in enumerate(alpha) if b != a], axis=0)
            dl[:, a] = coef * p * lam[:, a] ** (p - 1) * rest
        grads[:, m, :] = dl[:, 1:] - dl[:, :1]
    return vals, grads


def vector_tabulation(family, cell, degree, points):
    """Values (points, 3, 2) and divergence (points, 3) of a basis of RT0 on the
    reference triangle (see the module docstring); other spaces are not covered."""
    if (family, cell, int(degree)) != ("RT", "triangle", 1):
        raise NotImplementedError("the fixture shim covers the lowest Raviart-Thomas space on triangles")
    x = np.asarray(points, dtype=float)
    vals = np.empty((len(x), 3, 2))
    for k, shift in enumerate(((0.0, 0.0), (1.0, 0.0), (0.0, 1.0))):
        vals[:, k, 0] = x[:, 0] - shift[0]
        vals[:, k, 1] = x[:, 1] - shift[1]
    return vals, np.full((len(x), 3), 2.0)


def install():
    """Patch the reference modules in place (idempotent)."""
    import pymhm.fem.reference as ref
    import pymhm.fem.scalar.quadrilateral as quad

    ref.simplex_lagrange_tabulation = simplex_lagrange_tabulation
    ref.legendre_tabulation = legendre_tabulation
    ref.legendre_values = legendre_values
    ref.bernstein_tabulation = bernstein_tabulation
    quad.simplex_lagrange_tabulation = simplex_lagrange_tabulation
    import pymhm.fem.hdiv.rt as rt

    rt.vector_tabulation = vector_tabulation
    rt.legendre_values = legendre_values
    rt.rt_moment_coefficients.cache_clear()
