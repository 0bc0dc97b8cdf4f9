"""The P1 batch-assembly oracle against PyMHM's own CPU operators
(tests/golden/make_p1_golden.py) and closed-form simplex moments."""

from math import factorial

import numpy as np
import pytest

from oracle.p1_batch import assemble_p1_batch
from tests._cases import load


@pytest.mark.parametrize("kind", ["tri", "tet", "tet8"])
def test_oracle_matches_reference_operators(kind):
    g = load("p1_operators")
    pts = np.stack([g[f"{kind}_points"]] * 2)
    coef = "tet" if kind == "tet8" else kind
    a, m, f = assemble_p1_batch(pts, g[f"{kind}_cells"], diffusion=g[f"{coef}_tensor"],
                                source=float(g[f"{coef}_source"]))
    for b in range(2):
        np.testing.assert_allclose(a[b], g[f"{kind}_A"], atol=1e-13)
        np.testing.assert_allclose(m[b], g[f"{kind}_M"], atol=1e-14)
        np.testing.assert_allclose(f[b], g[f"{kind}_f"], atol=1e-14)


@pytest.mark.parametrize("dimension", [2, 3])
def test_oracle_simplex_moments(dimension):
    """The reference's closed-form check (tests/test_gpu_batch.py, resident moments)."""
    points = np.vstack((np.zeros(dimension), np.eye(dimension)))
    coordinates = np.stack((points, points * 2 + 0.3))
    cells = np.arange(dimension + 1)[None]
    tensor = np.diag(np.arange(1.0, dimension + 1))
    stiffness, mass, f = assemble_p1_batch(coordinates, cells, diffusion=tensor, source=3.0)
    for index, length in enumerate((1.0, 2.0)):
        volume = length**dimension / factorial(dimension)
        gradient = np.vstack((-np.ones(dimension), np.eye(dimension))) / length
        np.testing.assert_allclose(stiffness[index], volume * gradient @ tensor @ gradient.T, atol=1e-14)
        np.testing.assert_allclose(mass[index].sum(), volume)
        np.testing.assert_allclose(f[index], volume * 3 / (dimension + 1))
