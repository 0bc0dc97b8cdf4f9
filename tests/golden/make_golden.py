"""Write golden fixtures for the Cartesian Q1 MHM path by running PyMHM itself.

Run in a development checkout where the reference sources are importable:

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_golden.py [--full]

Basix (fenics-basix 0.11.0) is not installable here, so ``_basix_shim``
replaces the two interval tabulations the Q1 path needs.  The fixtures are
small ``.npz`` files; ``--full`` adds the 64x64-macro lognormal case (about
two minutes of reference CPU time), stored as solution vectors plus digests.
"""

from __future__ import annotations

import os
import sys
import time
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
from pymhm.core.system import HybridSystem  # noqa: E402
from pymhm.fem.scalar.operators import boundary_data  # noqa: E402
from pymhm.fem.traces.interval import FaceSpace, SkeletonSpace  # noqa: E402
from pymhm.materials.cartesian import CartesianCellField  # noqa: E402
from pymhm.meshes.cartesian import CartesianMacroMesh  # noqa: E402
from pymhm.postprocessing.solutions import QuadrilateralDarcySolution  # noqa: E402

from pymhm_b200.workloads import digest, lognormal_permeability, sine_source  # noqa: E402


def affine_dirichlet(x):
    return 0.7 + x[:, 0] - 2 * x[:, 1]


def quad_source(x):
    return 1.0 + x[:, 0] * x[:, 1]


def run_case(name, mesh, face_space, refinement, permeability, source, dirichlet,
             keep_cells=(0,), full_fields=True):
    sk = SkeletonSpace(mesh, (face_space,) * len(mesh.faces))
    order = 4
    boundary, fixed = boundary_data(sk, dirichlet, None, order=order)
    assert not fixed
    tasks = [_QuadTask(mesh, c, refinement, sk, 1, permeability, source, order)
             for c in range(len(mesh.cells))]
    t0 = time.time()
    system = HybridSystem.from_local_factory(_assemble_quad, tasks, boundary_load=boundary)
    t1 = time.time()
    hybrid = system.solve()
    t2 = time.time()
    fines = [meta[0] for meta in system.local_metadata]
    sol = QuadrilateralDarcySolution(sk, tuple(fines), hybrid.fields, (), hybrid, permeability,
                                     source, 1, order)
    flux = np.array([sol.evaluate(c, f.points[f.cells].mean(axis=1))[1] for c, f in enumerate(fines)])
    A = system.matrix.tocsc()
    out = dict(
        name=name, assemble_seconds=t1 - t0, solve_seconds=t2 - t1,
        cell_faces=mesh.cell_faces, signs=mesh.signs, faces=mesh.faces, face_cells=mesh.face_cells,
        offsets=sk.offsets, cell_dofs=np.array([sk.cell_dofs(c) for c in range(len(mesh.cells))]),
        boundary=boundary, indptr=A.indptr, indices=A.indices, data=A.data, rhs=system.rhs,
        load_scale=system.load_scale, trace=hybrid.trace, coarse=np.concatenate(hybrid.coarse),
        residual=hybrid.residual,
        corrected=np.array([r.coarse_vectors is not None for r in system.responses]),
    )
    fields = np.array(hybrid.fields)
    if full_fields:
        out["fields"] = fields
        out["flux"] = flux
    else:
        out["fields_norm"] = np.linalg.norm(fields)
        out["flux_norm"] = np.linalg.norm(flux)
        out["fields_cells"] = fields[list(keep_cells)]
        out["flux_cells"] = flux[list(keep_cells)]
    out["keep_cells"] = np.array(keep_cells)
    for c in keep_cells:
        r = system.responses[c]
        p = r.problem
        aug, rhs = p.condensation_system()
        out[f"cell{c}_A"] = p.matrix.toarray()
        out[f"cell{c}_B"] = p.coupling
        out[f"cell{c}_f"] = p.load
        out[f"cell{c}_C"] = p.constraints[:, 0]
        out[f"cell{c}_aug"] = aug.toarray()
        out[f"cell{c}_rhs"] = rhs
        out[f"cell{c}_source"] = r.source
        out[f"cell{c}_lifts"] = r.lifts
        out[f"cell{c}_retained"] = r.retained_basis[:, 0]
        idx, block, load = r.global_contribution(np.array([sk.size + c]))
        out[f"cell{c}_block"] = block
        out[f"cell{c}_load"] = load
    return out


def main(full=False):
    cases = []
    m = CartesianMacroMesh(8)
    cases.append(run_case("poisson_8x8_r4_p1", m, FaceSpace.uniform(1), (4, 4), 1.0, sine_source, 0.0,
                          keep_cells=(0, 9, 63)))
    kap = lognormal_permeability(64, 64, sigma=2.0, ell=0.05, seed=7)
    m = CartesianMacroMesh(4)
    field = CartesianCellField(kap, spacing=(1 / 64, 1 / 64))
    c = run_case("darcy_4x4_r16_p2_lognormal", m, FaceSpace.uniform(2), (16, 16), field, 1.0, 0.0,
                 keep_cells=(0, 5, 15))
    c["kappa"] = kap
    cases.append(c)
    m = CartesianMacroMesh(3, 2, (-1, 2, -2, 2))
    kap = np.exp(np.random.default_rng(3).normal(size=(12, 10)))
    field = CartesianCellField(kap, spacing=(0.25, 0.4), origin=(-1, -2))
    c = run_case("affine_3x2_rect_r4x5_p1s2", m, FaceSpace.uniform(1, 2), (4, 5), field, quad_source,
                 affine_dirichlet, keep_cells=(0, 4))
    c["kappa"] = kap
    cases.append(c)
    if full:
        kap = lognormal_permeability(1024, 1024, sigma=2.0, ell=0.05, seed=20261203)
        m = CartesianMacroMesh(64)
        field = CartesianCellField(kap, spacing=(1 / 1024, 1 / 1024))
        c = run_case("darcy_64x64_r16_p2_lognormal", m, FaceSpace.uniform(2), (16, 16), field, 1.0, 0.0,
                     keep_cells=(0, 1000, 4095), full_fields=False)
        c["kappa_sha256"] = digest(kap)
        c["pattern_sha256"] = digest(np.concatenate([c["indptr"], c["indices"]]))
        for key in ("indptr", "indices", "data", "cell_faces", "signs", "faces", "face_cells",
                    "cell_dofs", "load_scale"):
            c[key + "_sha256"] = digest(c.pop(key))
        cases.append(c)
    for c in cases:
        name = c.pop("name")
        np.savez_compressed(HERE / f"{name}.npz", **c)
        print(name, "assemble %.2fs solve %.2fs" % (c["assemble_seconds"], c["solve_seconds"]))


if __name__ == "__main__":
    main(full="--full" in sys.argv)
