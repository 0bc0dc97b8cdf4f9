"""Dense batched P1 simplex assembly on the GPU (``assemble_p1_batch``,
execution/cuda.py:27-105) against the oracle and PyMHM's own CPU operators."""

from math import factorial

import numpy as np
import pytest

from tests._cases import load

pytestmark = pytest.mark.gpu


def gpu(points, cells, **kw):
    from pymhm_b200.batched import assemble_p1_batch

    return tuple(t.cpu().numpy() for t in assemble_p1_batch(points, cells, **kw))


def structured(dimension, n):
    """A structured simplex mesh of the unit square / cube (2 triangles or 6 tetrahedra
    per box), node-numbered x-fastest."""
    axes = [np.linspace(0.0, 1.0, n + 1)] * dimension
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, dimension)
    idx = np.arange((n + 1) ** dimension).reshape((n + 1,) * dimension)
    cells = []
    if dimension == 2:
        for i in range(n):
            for j in range(n):
                a, b, c, d = idx[i, j], idx[i + 1, j], idx[i, j + 1], idx[i + 1, j + 1]
                cells += [[a, b, d], [a, d, c]]
    else:
        from itertools import permutations

        for i in range(n):
            for j in range(n):
                for k in range(n):
                    base = np.array([i, j, k])
                    for perm in permutations(range(3)):
                        path = [base.copy()]
                        for axis in perm:
                            path.append(path[-1] + np.eye(3, dtype=int)[axis])
                        cells.append([idx[tuple(p)] for p in path])
    return grid, np.array(cells, dtype=np.int64)


@pytest.mark.parametrize("dimension", [2, 3])
def test_matches_oracle_on_perturbed_batches(dimension):
    from oracle.p1_batch import assemble_p1_batch as host

    rng = np.random.default_rng(dimension)
    pts, cells = structured(dimension, 4 if dimension == 2 else 2)
    batch = 5
    coords = np.stack([pts + 0.03 * rng.standard_normal(pts.shape) for _ in range(batch)])
    m = rng.standard_normal((batch, len(cells), dimension, dimension))
    tensors = np.einsum("btij,btkj->btik", m, m) + 0.5 * np.eye(dimension)
    source = rng.uniform(0.5, 2.0, (batch, len(cells)))
    want = host(coords, cells, diffusion=tensors, source=source)
    got = gpu(coords, cells, diffusion=tensors, source=source)
    for w, g in zip(want, got):
        assert np.max(np.abs(g - w)) <= 1e-13 * np.max(np.abs(w))
    # broadcast coefficients: one tensor for all, one source per cell
    want = host(coords, cells, diffusion=tensors[0, 0], source=source[0])
    got = gpu(coords, cells, diffusion=tensors[0, 0], source=source[0])
    for w, g in zip(want, got):
        assert np.max(np.abs(g - w)) <= 1e-13 * np.max(np.abs(w))
    again = gpu(coords, cells, diffusion=tensors[0, 0], source=source[0])
    for g, h in zip(got, again):
        assert np.array_equal(g, h)  # fixed summation order: identical bits


@pytest.mark.parametrize("kind", ["tri", "tet"])
def test_matches_reference_operators(kind):
    g = load("p1_operators")
    pts = np.stack([g[f"{kind}_points"]] * 3)
    a, m, f = gpu(pts, g[f"{kind}_cells"], diffusion=g[f"{kind}_tensor"], source=float(g[f"{kind}_source"]))
    for b in range(3):
        np.testing.assert_allclose(a[b], g[f"{kind}_A"], atol=1e-13)
        np.testing.assert_allclose(m[b], g[f"{kind}_M"], atol=1e-14)
        np.testing.assert_allclose(f[b], g[f"{kind}_f"], atol=1e-14)


def test_config4_local_mesh_matches_reference():
    """One macro tetrahedron refined with submesh(cell, 8) (165 P1 nodes, the local mesh
    of the 3-D configuration): 32 affinely mapped copies, each against the reference's
    operators mapped the same way (stiffness and mass scale with the map)."""
    g = load("p1_operators")
    pts, cells = g["tet8_points"], g["tet8_cells"]
    rng = np.random.default_rng(8)
    scales = rng.uniform(0.5, 2.0, 32)
    shifts = rng.normal(size=(32, 3))
    coords = np.stack([s * pts + t for s, t in zip(scales, shifts)])
    a, m, f = gpu(coords, cells, diffusion=g["tet_tensor"], source=float(g["tet_source"]))
    for b, sc in enumerate(scales):
        # uniform scaling by sc: stiffness * sc, mass * sc^3, load * sc^3 in three dimensions
        np.testing.assert_allclose(a[b], sc * g["tet8_A"], atol=1e-12 * sc * np.abs(g["tet8_A"]).max())
        np.testing.assert_allclose(m[b], sc**3 * g["tet8_M"], atol=1e-14 * sc**3 * np.abs(g["tet8_M"]).max() + 1e-300)
        np.testing.assert_allclose(f[b], sc**3 * g["tet8_f"], atol=1e-13 * sc**3 * np.abs(g["tet8_f"]).max())


@pytest.mark.parametrize("dimension", [2, 3])
def test_simplex_moments(dimension):
    points = np.vstack((np.zeros(dimension), np.eye(dimension)))
    coordinates = np.stack((points, points * 2 + 0.3))
    cells = np.arange(dimension + 1)[None]
    tensor = np.diag(np.arange(1.0, dimension + 1))
    stiffness, mass, f = gpu(coordinates, cells, diffusion=tensor, source=3.0)
    for index, length in enumerate((1.0, 2.0)):
        volume = length**dimension / factorial(dimension)
        gradient = np.vstack((-np.ones(dimension), np.eye(dimension))) / length
        np.testing.assert_allclose(stiffness[index], volume * gradient @ tensor @ gradient.T, atol=1e-14)
        np.testing.assert_allclose(mass[index].sum(), volume)
        np.testing.assert_allclose(f[index], volume * 3 / (dimension + 1))
    a, _, _ = gpu(coordinates, cells)
    np.testing.assert_allclose(a.sum(axis=-1), 0, atol=1e-14)


@pytest.mark.parametrize(
    ("points", "cells", "kwargs", "message"),
    [
        ([[0.0, 0.0]], [[0, 1, 2]], {}, "points"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0, 1]], {}, "cells"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0.0, 1.0, 2.0]], {}, "cells"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0, 1, 3]], {}, "cells"),
        ([[[0.0, 0.0], [1.0, 0.0], [2.0, 0.0]]], [[0, 1, 2]], {}, "degenerate"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0, 1, 2]], {"diffusion": -1.0}, "diffusion"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0, 1, 2]], {"diffusion": [[1.0, 2.0], [0.0, 1.0]]}, "diffusion"),
        ([[[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]]], [[0, 1, 2]], {"source": np.nan}, "source"),
        ([[[0.0, np.inf], [1.0, 0.0], [0.0, 1.0]]], [[0, 1, 2]], {}, "points"),
    ],
)
def test_invalid_contracts(points, cells, kwargs, message):
    """The reference's invalid-contract cases, with the same messages."""
    from pymhm_b200.batched import assemble_p1_batch

    with pytest.raises(ValueError, match=message):
        assemble_p1_batch(points, cells, **kwargs)
