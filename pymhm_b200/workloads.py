"""Seeded synthetic inputs for the Cartesian Darcy workloads.

The reference project publishes no dataset for these problems, so every input
is generated here deterministically from a seed:

* ``lognormal_permeability``: log-kappa is a stationary Gaussian field with
  exponential covariance ``sigma^2 exp(-|r|/ell)`` sampled on the fine-cell
  centres of a regular grid by circulant embedding on a doubled periodic grid
  (NumPy PCG64 generator, float64 FFTs).  Negative embedding eigenvalues, if
  any, are clipped to zero and reported.
* ``sine_source``: ``f = 2 pi^2 sin(pi x) sin(pi y)``, the manufactured source
  whose exact pressure is ``sin(pi x) sin(pi y)`` with homogeneous Dirichlet data.

Arrays follow the reference's pixel-field layout: ``values[ix, iy]`` with the
first axis along x (``materials/cartesian.py:14-72`` of PyMHM).
"""

from __future__ import annotations

import hashlib

import numpy as np

DEFAULT_SEED = 20261203


def lognormal_permeability(cells_x: int, cells_y: int | None = None, *, sigma: float = 2.0,
                           ell: float = 0.05, seed: int = DEFAULT_SEED,
                           extent: tuple[float, float] = (1.0, 1.0)) -> np.ndarray:
    """Return ``exp(G)`` on a ``(cells_x, cells_y)`` grid of fine-cell centres.

    ``G`` has zero mean and covariance ``sigma^2 exp(-|x-y|/ell)``.  The
    embedding grid is ``2 cells`` per axis with the same spacing as the field.
    """
    cells_y = cells_x if cells_y is None else cells_y
    hx, hy = extent[0] / cells_x, extent[1] / cells_y
    mx, my = 2 * cells_x, 2 * cells_y
    kx = np.arange(mx)
    ky = np.arange(my)
    dx = np.minimum(kx, mx - kx) * hx
    dy = np.minimum(ky, my - ky) * hy
    r = np.sqrt(dx[:, None] ** 2 + dy[None, :] ** 2)
    cov = sigma ** 2 * np.exp(-r / ell)
    eig = np.fft.fft2(cov).real
    eig = np.maximum(eig, 0.0)
    rng = np.random.Generator(np.random.PCG64(seed))
    z = rng.standard_normal((mx, my)) + 1j * rng.standard_normal((mx, my))
    field = np.fft.fft2(np.sqrt(eig / (mx * my)) * z).real[:cells_x, :cells_y]
    return np.exp(field)


def layered_lognormal_permeability(layers: int = 40, pixels: int = 64, *, sigma: float = 3.0, ell: float = 0.1,
                                   contrast: float = 1e6, seed: int = DEFAULT_SEED) -> np.ndarray:
    """``(layers, pixels, pixels)`` permeability of a layered unit cube: layer k (of
    equal thickness along z) holds its own ``lognormal_permeability`` of the
    ``pixels`` x ``pixels`` cell centres in (x, y) (seed ``seed + k``), log-values
    clipped to +-log(contrast)/2 so that max / min <= contrast."""
    half = 0.5 * np.log(contrast)
    out = np.empty((layers, pixels, pixels))
    for k in range(layers):
        g = np.log(lognormal_permeability(pixels, pixels, sigma=sigma, ell=ell, seed=seed + k))
        out[k] = np.exp(np.clip(g, -half, half))
    return out


class LayeredField:
    """Piecewise-constant scalar permeability of the unit cube on a layered pixel
    grid: point (x, y, z) takes ``values[min(floor(z L), L-1), min(floor(x P), P-1),
    min(floor(y P), P-1)]`` (coordinates clipped to [0, 1]).  Callable on (n, 3)
    points, as the reference's material callables are."""

    def __init__(self, values: np.ndarray):
        self.values = np.ascontiguousarray(values, dtype=float)

    def index(self, points: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        L, P, Q = self.values.shape
        p = np.clip(np.asarray(points, dtype=float), 0.0, 1.0)
        k = np.minimum((p[:, 2] * L).astype(np.int64), L - 1)
        i = np.minimum((p[:, 0] * P).astype(np.int64), P - 1)
        j = np.minimum((p[:, 1] * Q).astype(np.int64), Q - 1)
        return k, i, j

    def __call__(self, points: np.ndarray) -> np.ndarray:
        return self.values[self.index(points)]


def disc_inclusions(count: int = 300, *, rmin: float = 0.01, rmax: float = 0.03,
                    seed: int = DEFAULT_SEED) -> tuple[np.ndarray, np.ndarray]:
    """``count`` discs with PCG64-uniform centres in the unit square and radii uniform
    in [rmin, rmax]: (centres (count, 2), radii (count,))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centres = rng.uniform(0.0, 1.0, size=(count, 2))
    radii = rng.uniform(rmin, rmax, size=count)
    return centres, radii


class DiscInclusions:
    """Piecewise-constant scalar permeability: ``inside`` in the union of the discs,
    ``outside`` elsewhere.  A point is inside a disc when
    (x - cx)^2 + (y - cy)^2 <= r^2, each square and the sum rounded separately.
    Callable on (n, 2) points, as the reference's material callables are."""

    def __init__(self, centres, radii, inside: float = 1e4, outside: float = 1.0):
        self.centres = np.ascontiguousarray(centres, dtype=float)
        self.radii = np.ascontiguousarray(radii, dtype=float)
        self.r2 = self.radii * self.radii
        self.inside, self.outside = float(inside), float(outside)

    def __call__(self, points: np.ndarray) -> np.ndarray:
        p = np.asarray(points, dtype=float)
        hit = np.zeros(len(p), dtype=bool)
        for (cx, cy), r2 in zip(self.centres, self.r2):
            dx = p[:, 0] - cx
            dy = p[:, 1] - cy
            hit |= (dx * dx + dy * dy) <= r2
        return np.where(hit, self.inside, self.outside)


def sine_source(points: np.ndarray) -> np.ndarray:
    """Manufactured source ``2 pi^2 sin(pi x) sin(pi y)``."""
    return 2 * np.pi ** 2 * np.sin(np.pi * points[:, 0]) * np.sin(np.pi * points[:, 1])


def sine_pressure(points: np.ndarray) -> np.ndarray:
    return np.sin(np.pi * points[:, 0]) * np.sin(np.pi * points[:, 1])


def digest(array: np.ndarray) -> str:
    """SHA-256 of an array's C-order bytes (records seeded inputs and outputs)."""
    a = np.ascontiguousarray(array)
    return hashlib.sha256(a.tobytes()).hexdigest()


# Workload descriptions used by bench.py and the parity tests.
POISSON_8x8 = dict(name="poisson-q1-8x8-r4-p1", macro=8, local=4, face_degree=1,
                   permeability="one", source="sine")
TETRA_8 = dict(name="darcy-p1-tetra-cube8-r8-p1faces-layered", cube=8, local=8, face_degree=1, layers=40,
               pixels=64, sigma=3.0, ell=0.1, contrast=1e6, seed=DEFAULT_SEED)
DARCY_64x64 = dict(name="darcy-q1-64x64-r16-p2-lognormal", macro=64, local=16, face_degree=2,
                   permeability="lognormal", source="one", sigma=2.0, ell=0.05, seed=DEFAULT_SEED)
