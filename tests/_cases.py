"""Shared definitions of the golden cases (inputs as the fixture script used them)."""

from pathlib import Path

import numpy as np

from pymhm_b200.workloads import sine_source

GOLDEN = Path(__file__).resolve().parent / "golden"


class PixelField:
    """Minimal stand-in for the reference's CartesianCellField (values, spacing, origin)."""

    def __init__(self, values, spacing, origin=(0.0, 0.0)):
        self.values, self.spacing, self.origin = np.asarray(values), tuple(spacing), tuple(origin)

    def __call__(self, pts):
        from oracle.q1_mhm import PixelField as OP

        return OP(self.values, self.spacing, self.origin)(pts)


def smooth_tensor(x):
    """The anisotropic test field of the smooth-tensor fixture (make_quadrature_golden.py):
    K = [[exp(sin 2 pi x cos 2 pi y), 0.3 sin(pi x y)], [0.3 sin(pi x y), 1 + x y]]."""
    k1 = np.exp(np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]))
    k2 = 1.0 + x[:, 0] * x[:, 1]
    k12 = 0.3 * np.sin(np.pi * x[:, 0] * x[:, 1])
    return np.stack((np.stack((k1, k12), -1), np.stack((k12, k2), -1)), -2)


def quad_source(x):
    return 1.0 + x[:, 0] * x[:, 1]


def affine_dirichlet(x):
    return 0.7 + x[:, 0] - 2 * x[:, 1]


def face_space(cls, face):
    """The face space of a case: ``cls.uniform`` of its (degree, subdivisions[, continuous])."""
    degree, subdivisions, *rest = face
    return cls.uniform(degree, subdivisions, continuous=bool(rest and rest[0]))


def load(name):
    return np.load(GOLDEN / f"{name}.npz")


# name -> (macro args, (face degree, subdivisions[, continuous]), refinement, permeability(g), source,
#          dirichlet)
CASES = {
    "poisson_8x8_r4_p1": ((8,), (1, 1), (4, 4), lambda g: 1.0, sine_source, 0.0),
    "darcy_4x4_r16_p2_lognormal": ((4,), (2, 1), (16, 16),
                                   lambda g: PixelField(g["kappa"], (1 / 64, 1 / 64)), 1.0, 0.0),
    "darcy_4x4_r8_p1_cut20": ((4,), (1, 1), (8, 8),
                              lambda g: PixelField(g["kappa"], (1 / 20, 1 / 20)), 1.0, 0.0),
    # a permeability that varies inside the fine cells (Gauss-point values, kappa mode 6)
    "darcy_4x4_r8_p1_smooth_tensor": ((4,), (1, 1), (8, 8), lambda g: smooth_tensor, 1.0, 0.0),
    # continuous piecewise-linear traces on two segments per face (3 DOFs a face)
    "darcy_4x4_r8_p1c2_lognormal": ((4,), (1, 2, True), (8, 8),
                                    lambda g: PixelField(g["kappa"], (1 / 32, 1 / 32)), 1.0, 0.0),
    "affine_3x2_rect_r4x5_p1s2": ((3, 2, (-1, 2, -2, 2)), (1, 2), (4, 5),
                                  lambda g: PixelField(g["kappa"], (0.25, 0.4), (-1, -2)), quad_source,
                                  affine_dirichlet),
}


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
