"""Write the golden fixture of a permeability field whose pixel lines cross the fine
cells, by running PyMHM itself: its Cartesian Q1 path then integrates each fine cell on
the exact intersections with the pixels (``fem/scalar/quadrilateral.py:136-188, 215-234``).

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_cut_golden.py

Reuses ``make_golden.run_case`` (and its Basix shim).
"""

from __future__ import annotations

import numpy as np

from make_golden import CartesianCellField, CartesianMacroMesh, FaceSpace, HERE, run_case


def main():
    rng = np.random.default_rng(20)
    kap = np.exp(rng.normal(scale=1.5, size=(20, 20)))
    m = CartesianMacroMesh(4)
    field = CartesianCellField(kap, spacing=(1 / 20, 1 / 20))
    c = run_case("darcy_4x4_r8_p1_cut20", m, FaceSpace.uniform(1), (8, 8), field, 1.0, 0.0, keep_cells=(0, 6))
    c["kappa"] = kap
    name = c.pop("name")
    np.savez_compressed(HERE / f"{name}.npz", **c)
    print(name, "assemble %.2fs solve %.2fs" % (c["assemble_seconds"], c["solve_seconds"]))


if __name__ == "__main__":
    main()
