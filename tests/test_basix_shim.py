"""The clean-room Basix stand-in (``tests/golden/_basix_shim.py``) against the
reference's checks that do not depend on Basix itself.

The reference validates its tabulation-based Qk basis with cardinality, partition of
unity, polynomial reproduction and closed-form Q1 matrices
(``tests/test_quadrilateral.py:111-160`` of PyMHM 1.3.2).  The same properties at the
same tolerances are checked here on the shim, through the tensor product that
``qk_basis`` forms from the interval factors (``fem/scalar/quadrilateral.py:58-94``),
with the Gauss rule of ``quadrilateral_quadrature`` (``:25-32``).  Legendre
tabulation and the degree-one simplex basis get their defining properties.
"""

import numpy as np
import pytest
from numpy.polynomial.legendre import leggauss
from numpy.testing import assert_allclose

from tests.golden import _basix_shim as shim


def cardinal(degree, x):
    """``_cardinal_values``: interval Pk in increasing equispaced nodal order."""
    nodes = np.linspace(0, 1, degree + 1)
    values, derivatives, _ = shim.simplex_lagrange_tabulation(
        "interval", degree, np.column_stack((1 - x, x)), nodes=np.column_stack((1 - nodes, nodes)), nderiv=1)
    return values, derivatives[..., 0]


def qk(degree, points):
    x, dx = cardinal(degree, points[:, 0])
    y, dy = cardinal(degree, points[:, 1])
    basis = np.einsum("qi,qj->qij", y, x).reshape(len(points), (degree + 1) ** 2)
    grad = np.stack((np.einsum("qi,qj->qij", y, dx), np.einsum("qi,qj->qij", dy, x)), axis=-1)
    return basis, grad.reshape(len(points), (degree + 1) ** 2, 2)


def gauss_square(order):
    p, w = leggauss(order)
    p, w = (p + 1) / 2, w / 2
    return np.array([(x, y) for y in p for x in p]), np.array([wx * wy for wy in w for wx in w])


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 5, 6])
def test_cardinality_partition_and_polynomial_derivatives(degree):
    nodes = np.array([(x, y) for y in np.linspace(0, 1, degree + 1) for x in np.linspace(0, 1, degree + 1)])
    values, _ = qk(degree, nodes)
    assert_allclose(values, np.eye(len(nodes)), atol=6e-14)
    ref, weights = gauss_square(6)
    values, grads = qk(degree, ref)
    assert_allclose(values.sum(axis=1), 1, atol=6e-14)
    assert_allclose(grads.sum(axis=1), 0, atol=3e-13)
    nodal = nodes[:, 0] ** degree * nodes[:, 1] ** degree
    assert_allclose(values @ nodal, ref[:, 0] ** degree * ref[:, 1] ** degree, atol=3e-14)
    want = degree * np.column_stack((ref[:, 0] ** (degree - 1) * ref[:, 1] ** degree,
                                     ref[:, 0] ** degree * ref[:, 1] ** (degree - 1)))
    assert_allclose(np.einsum("qia,i->qa", grads, nodal), want, atol=3e-13)
    assert_allclose(weights @ (values @ nodal), 1 / (degree + 1) ** 2, atol=1e-14)


def test_q1_tensor_product_matrices_independently():
    """Q1 stiffness, mass and load of the rectangle (-2, 0) x (-1, 2) with diffusion
    diag(2, 3) and source 4, by quadrature of the shim's basis, equal the closed forms."""
    lx, ly = 2.0, 3.0
    k = np.diag([2.0, 3.0])
    ref, weights = gauss_square(4)
    values, grads = qk(1, ref)
    phys = grads / np.array([lx, ly])
    area = lx * ly
    matrix = area * np.einsum("q,qia,ab,qjb->ij", weights, phys, k, phys)
    mass = area * np.einsum("q,qi,qj->ij", weights, values, values)
    load = area * 4 * weights @ values
    m1 = np.array([[2.0, 1.0], [1.0, 2.0]]) / 6
    a1 = np.array([[1.0, -1.0], [-1.0, 1.0]])
    expected = 2 * 3 / 2 * np.kron(m1, a1) + 3 * 2 / 3 * np.kron(a1, m1)
    assert_allclose(matrix, expected, atol=1e-14)
    assert_allclose(mass, 6 * np.kron(m1, m1), atol=1e-14)
    assert_allclose(load, 6, atol=1e-14)
    assert_allclose(matrix @ np.ones(4), 0, atol=1e-14)
    assert np.linalg.eigvalsh(matrix)[1] > 0


@pytest.mark.parametrize("degree", [0, 1, 2, 3, 4])
def test_legendre_convention(degree):
    """Conventional Legendre polynomials: L_j(1) = 1, L_j(-1) = (-1)^j, and squared mass
    2 / (2j + 1) on [-1, 1] (a face of length L: L / (2j + 1))."""
    end = shim.legendre_values(np.array([1.0, -1.0]), degree)
    assert_allclose(end[0], 1, atol=1e-15)
    assert_allclose(end[1], (-1.0) ** np.arange(degree + 1), atol=1e-15)
    p, w = leggauss(degree + 2)
    v = shim.legendre_values(p, degree)
    assert_allclose(v.T @ (w[:, None] * v), np.diag(2 / (2 * np.arange(degree + 1) + 1)), atol=1e-14)
    d = shim.legendre_tabulation(p, degree, nderiv=1)
    if degree >= 1:
        assert_allclose(d[1][:, 1], 1, atol=1e-15)


@pytest.mark.parametrize("dim", [2, 3])
def test_simplex_p1_kronecker_partition_and_gradients(dim):
    rng = np.random.default_rng(dim)
    nodes = np.eye(dim + 1)[rng.permutation(dim + 1)]
    bary = rng.dirichlet(np.ones(dim + 1), size=7)
    vals, grad, hess = shim.simplex_lagrange_tabulation("triangle" if dim == 2 else "tetrahedron", 1,
                                                        np.vstack((nodes, bary)), nodes=nodes, nderiv=2)
    assert_allclose(vals[: dim + 1], np.eye(dim + 1), atol=1e-15)
    assert_allclose(vals.sum(axis=1), 1, atol=1e-14)
    assert_allclose(grad.sum(axis=1), 0, atol=1e-14)
    # the gradient of the basis function at node k in the reference coordinates
    # x = bary[:, 1:] reproduces x itself
    x = np.vstack((nodes, bary))[:, 1:]
    coords = nodes[:, 1:]
    assert_allclose(vals @ coords, x, atol=1e-14)
    assert_allclose(np.einsum("qia,ib->qab", grad, coords), np.broadcast_to(np.eye(dim), (len(x), dim, dim)),
                    atol=1e-14)
    assert np.all(hess == 0)
