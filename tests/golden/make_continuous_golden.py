"""Write the golden fixture of a skeleton with continuous nodal face spaces, by running
PyMHM itself (``FaceSpace(..., continuous=True)``, ``fem/traces/interval.py:13-116``):
continuous piecewise-linear traces on two segments per face, a 4x4 macro mesh of 8x8
local Q1 cells and a log-normal pixel field aligned with the fine grid.

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_continuous_golden.py

Reuses ``make_golden.run_case`` (and its Basix shim).
"""

from __future__ import annotations

import numpy as np

from make_golden import HERE, CartesianCellField, CartesianMacroMesh, FaceSpace, lognormal_permeability, run_case


def main():
    kap = lognormal_permeability(32, 32, sigma=1.5, ell=0.1, seed=41)
    field = CartesianCellField(kap, spacing=(1 / 32, 1 / 32))
    c = run_case("darcy_4x4_r8_p1c2_lognormal", CartesianMacroMesh(4), FaceSpace.uniform(1, 2, continuous=True),
                 (8, 8), field, 1.0, 0.0, keep_cells=(0, 5))
    c["kappa"] = kap
    name = c.pop("name")
    np.savez_compressed(HERE / f"{name}.npz", **c)
    print(name, "assemble %.2fs solve %.2fs" % (c["assemble_seconds"], c["solve_seconds"]))


if __name__ == "__main__":
    main()
