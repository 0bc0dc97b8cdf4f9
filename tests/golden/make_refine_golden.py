"""Write golden fixtures for original-equation refinement by running PyMHM's own
``refine_hybrid`` (core/refinement.py:612-800) on two golden Cartesian Q1 cases.

Run in a development checkout where the reference sources are importable:

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_refine_golden.py

The solution of each case is perturbed the way the reference's own refinement
test does it (``tests/test_darcy_refinement.py``: every local field plus
0.002 * (1, 2, ..., n)), then refined with ``max_steps=2`` and ``rtol=1e-10``.
Each ``refine_<case>.npz`` holds the perturbed starting point, the residual
history, the right-hand-side norm, the reduced residual and the refined
trace, coarse and field values.  Basix is replaced by ``_basix_shim`` as in
``make_golden.py``.
"""

from __future__ import annotations

import os
import sys
from dataclasses import replace
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
if not os.environ.get("PYMHM_SRC"):
    sys.exit("set PYMHM_SRC to the src/ directory of a PyMHM 1.3.2 checkout")
sys.path.insert(0, os.environ["PYMHM_SRC"])
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(REPO))

import _basix_shim  # noqa: E402

_basix_shim.install()

from pymhm._legacy.models.darcy.cartesian import _assemble_quad, _QuadTask  # noqa: E402
from pymhm.core.refinement import refine_hybrid  # noqa: E402
from pymhm.core.system import HybridSystem  # noqa: E402
from pymhm.fem.scalar.operators import boundary_data  # noqa: E402
from pymhm.fem.traces.interval import FaceSpace, SkeletonSpace  # noqa: E402
from pymhm.materials.cartesian import CartesianCellField  # noqa: E402
from pymhm.meshes.cartesian import CartesianMacroMesh  # noqa: E402
from pymhm_b200.workloads import lognormal_permeability, sine_source  # noqa: E402


def run(name, mesh, face_space, refinement, permeability, source):
    sk = SkeletonSpace(mesh, (face_space,) * len(mesh.faces))
    boundary, fixed = boundary_data(sk, 0.0, None, order=4)
    assert not fixed
    tasks = [_QuadTask(mesh, c, refinement, sk, 1, permeability, source, 4) for c in range(len(mesh.cells))]
    system = HybridSystem.from_local_factory(_assemble_quad, tasks, boundary_load=boundary)
    hybrid = system.solve()
    perturbed = replace(hybrid, fields=tuple(u + 0.002 * np.arange(1, len(u) + 1) for u in hybrid.fields))
    result = refine_hybrid(system, perturbed, boundary_load=boundary, max_steps=2, rtol=1e-10)
    out = dict(
        start_fields=np.array(perturbed.fields), start_trace=perturbed.trace,
        start_coarse=np.concatenate(perturbed.coarse),
        residual_norms=np.array(result.residual_norms), rhs_norm=result.rhs_norm,
        reduced=result.solution.residual, trace=result.solution.trace,
        coarse=np.concatenate(result.solution.coarse), fields=np.array(result.solution.fields),
    )
    np.savez_compressed(HERE / f"refine_{name}.npz", **out)
    print(name, "residual history", result.residual_norms, "rhs", result.rhs_norm)


def main():
    run("poisson_8x8_r4_p1", CartesianMacroMesh(8), FaceSpace.uniform(1), (4, 4), 1.0, sine_source)
    kap = lognormal_permeability(64, 64, sigma=2.0, ell=0.05, seed=7)
    run("darcy_4x4_r16_p2_lognormal", CartesianMacroMesh(4), FaceSpace.uniform(2), (16, 16),
        CartesianCellField(kap, spacing=(1 / 64, 1 / 64)), 1.0)


if __name__ == "__main__":
    main()
