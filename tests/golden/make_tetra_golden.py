"""Write the 3D P1 tetrahedral fixtures by running PyMHM itself.

Usage (development checkout of PyMHM 1.3.2; Basix is replaced by ``_basix_shim``):

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_tetra_golden.py

Each case runs the reference's ``_DarcyFactory`` (``_legacy/models/darcy/
primal_3d.py:32-66``, the local factory of ``solve_darcy_3d``) through
``HybridSystem.from_local_factory`` and ``system.solve()`` with degree-one local
spaces, a ``TriangularSkeleton`` of Bernstein degree 1 (or 0) per face, homogeneous
Dirichlet data, f = 1 and a layered log-normal permeability (``LayeredField``).
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

from pymhm._legacy.models.darcy.primal_3d import _DarcyFactory  # noqa: E402
from pymhm.core.system import HybridSystem  # noqa: E402
from pymhm.fem.traces.triangle_3d import TriangularSkeleton, tetra_boundary_data  # noqa: E402
from pymhm.meshes.tetrahedron import TetraMesh  # noqa: E402

from pymhm_b200.workloads import LayeredField, digest, layered_lognormal_permeability  # noqa: E402


def run_case(name, cube, refinement, face_degree, layers, pixels, seed, keep_cells):
    mesh = TetraMesh.unit_cube(cube)
    sk = TriangularSkeleton(mesh, 1, degree=face_degree)
    values = layered_lognormal_permeability(layers, pixels, sigma=3.0, ell=0.1, contrast=1e6, seed=seed)
    field = LayeredField(values)
    order = 5
    boundary, fixed = tetra_boundary_data(sk, 0.0, {}, order)
    assert not fixed
    factory = _DarcyFactory(mesh, sk, refinement, 1, field, 1.0, order)
    t0 = time.time()
    system = HybridSystem.from_local_factory(factory, range(len(mesh.cells)), boundary_load=boundary)
    t1 = time.time()
    hybrid = system.solve()
    t2 = time.time()
    A = system.matrix.tocsc()
    out = dict(
        name=name, assemble_seconds=t1 - t0, solve_seconds=t2 - t1, kappa_sha256=digest(values),
        kappa_args=np.array([layers, pixels, seed]),
        points=mesh.points, cells=mesh.cells, faces=mesh.faces, cell_faces=mesh.cell_faces,
        face_cells=mesh.face_cells, signs=mesh.signs, areas=mesh.areas, offsets=sk.offsets,
        cell_dofs=np.array([sk.cell_dofs(c) for c in range(len(mesh.cells))]),
        boundary=boundary, indptr=A.indptr, indices=A.indices, data=A.data, rhs=system.rhs,
        trace=hybrid.trace, coarse=np.concatenate(hybrid.coarse), residual=hybrid.residual,
        fields=np.array(hybrid.fields),
        corrected=np.array([r.coarse_vectors is not None for r in system.responses]),
        keep_cells=np.array(keep_cells),
    )
    for c in keep_cells:
        r = system.responses[c]
        p = r.problem
        out[f"cell{c}_A"] = p.matrix.toarray()
        out[f"cell{c}_B"] = p.coupling
        out[f"cell{c}_f"] = p.load
        out[f"cell{c}_C"] = p.constraints[:, 0]
        out[f"cell{c}_lifts"] = r.lifts
        out[f"cell{c}_retained"] = r.retained_basis[:, 0]
        idx, block, load = r.global_contribution(np.array([sk.size + c]))
        out[f"cell{c}_block"] = block
        out[f"cell{c}_load"] = load
    return out


def main():
    cases = [
        run_case("tetra_cube2_r4_p1_layered", 2, 4, 1, 8, 16, 11, keep_cells=(0, 17, 47)),
        run_case("tetra_cube1_r8_p1_layered", 1, 8, 1, 40, 64, 12, keep_cells=(0, 5)),
        run_case("tetra_cube2_r2_p0_layered", 2, 2, 0, 4, 8, 13, keep_cells=(0,)),
    ]
    for c in cases:
        name = c.pop("name")
        np.savez_compressed(HERE / f"{name}.npz", **c)
        print(name, f"assemble {c['assemble_seconds']:.2f}s solve {c['solve_seconds']:.2f}s",
              "cells", len(c["cells"]), "N", len(c["rhs"]))


if __name__ == "__main__":
    main()
