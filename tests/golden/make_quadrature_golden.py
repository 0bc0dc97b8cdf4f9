"""Write the golden fixture of a permeability that varies inside the fine cells, by
running PyMHM itself: its Cartesian Q1 path evaluates a callable permeability at the
tensor Gauss points of every fine cell (``fem/scalar/quadrilateral.py:191-253``) and the
flux at the fine-cell centres.  A smooth anisotropic tensor field on a 4x4 macro mesh of
8x8 local Q1 cells, P1 faces, a constant source.

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_quadrature_golden.py

Reuses ``make_golden.run_case`` (and its Basix shim).
"""

from __future__ import annotations

import numpy as np

from make_golden import HERE, CartesianMacroMesh, FaceSpace, run_case


def smooth_tensor(x):
    """K(x, y) = [[k1, k12], [k12, k2]] with k1 = exp(sin 2 pi x cos 2 pi y),
    k2 = 1 + x y, k12 = 0.3 sin(pi x y): positive definite everywhere."""
    k1 = np.exp(np.sin(2 * np.pi * x[:, 0]) * np.cos(2 * np.pi * x[:, 1]))
    k2 = 1.0 + x[:, 0] * x[:, 1]
    k12 = 0.3 * np.sin(np.pi * x[:, 0] * x[:, 1])
    return np.stack((np.stack((k1, k12), -1), np.stack((k12, k2), -1)), -2)


def main():
    c = run_case("darcy_4x4_r8_p1_smooth_tensor", CartesianMacroMesh(4), FaceSpace.uniform(1), (8, 8),
                 smooth_tensor, 1.0, 0.0, keep_cells=(0, 9))
    name = c.pop("name")
    np.savez_compressed(HERE / f"{name}.npz", **c)
    print(name, "assemble %.2fs solve %.2fs" % (c["assemble_seconds"], c["solve_seconds"]))


if __name__ == "__main__":
    main()
