"""Write the polygonal mixed RT0 / P0 fixtures by running PyMHM itself.

Usage (development checkout of PyMHM 1.3.2; Basix is replaced by ``_basix_shim``):

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_polygon_rt0_golden.py

Each case builds the reference's ``PolygonMesh`` from this repository's seeded Voronoi
partition (``pymhm_b200.polygon.voronoi_mesh``; the partition is input data), refines
every cell with its own subdivision count (uneven local sizes), and runs the
reference's ``_DarcyLocalFactory`` (``_legacy/models/darcy/primal.py:28-106``) with
``formulation="mixed"`` through ``HybridSystem`` and ``system.solve()``: RT0 fluxes,
P0 pressures and boundary multipliers per cell, a degree-zero ``FaceSpace`` per edge
(one or two segments, aligned with the fine edges), homogeneous Dirichlet data (the
mixed boundary load, minus the primal one, is zero), f = 1 and a disc-inclusion
permeability (``DiscInclusions``).
"""

from __future__ import annotations

import os
import sys
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

from pymhm._legacy.models.darcy.primal import _DarcyLocalFactory  # noqa: E402
from pymhm.core.system import HybridSystem  # noqa: E402
from pymhm.fem.scalar.operators import boundary_data  # noqa: E402
from pymhm.fem.traces.interval import FaceSpace, SkeletonSpace  # noqa: E402
from pymhm.meshes.polygonal import PolygonMesh  # noqa: E402

from pymhm_b200.polygon import voronoi_mesh  # noqa: E402
from pymhm_b200.workloads import DiscInclusions, disc_inclusions  # noqa: E402


def run_case(name, count, seed, choices, segments, discs, keep_cells):
    poly = voronoi_mesh(count, seed)
    mesh = PolygonMesh(poly.points, tuple(poly.cells), local_triangulation="boundary")
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(0, segments),) * len(mesh.faces))
    rs = np.random.Generator(np.random.PCG64(seed + 1)).choice(np.asarray(choices), size=count)
    fines = tuple(mesh.submesh(c, int(rs[c])) for c in range(count))
    centres, radii = disc_inclusions(discs, rmin=0.04, rmax=0.09, seed=seed + 2)
    field = DiscInclusions(centres, radii)
    order = 4
    boundary, fixed = boundary_data(sk, 0.0, None, order=order)
    assert not fixed and not np.any(boundary)
    # the factory's alignment check reads local_refinement; the supplied meshes carry
    # each cell's own count, all multiples of the segment count
    factory = _DarcyLocalFactory(mesh, sk, field, 1.0, tuple(np.zeros((0, 3)) for _ in range(count)), segments,
                                 fines, 1, "mixed", order)
    assemblies = [factory(c) for c in range(count)]
    system = HybridSystem([a.problem for a in assemblies], boundary_load=-boundary)
    hybrid = system.solve()
    A = system.matrix.tocsc()
    fields = [np.asarray(f) for f in hybrid.fields]
    out = dict(
        count=count, seed=seed, refinements=rs, discs=np.array([discs]), segments=np.array([segments]),
        indptr=A.indptr, indices=A.indices, data=A.data, rhs=system.rhs,
        trace=hybrid.trace, coarse=np.concatenate(hybrid.coarse), residual=hybrid.residual,
        field_ptr=np.r_[0, np.cumsum([len(f) for f in fields])], fields=np.concatenate(fields),
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
        out[f"cell{c}_Z"] = p.kernel[:, 0]
        out[f"cell{c}_lifts"] = r.lifts
        idx, block, load = r.global_contribution(np.array([sk.size + c]))
        out[f"cell{c}_block"] = block
        out[f"cell{c}_load"] = load
    return name, out


def main():
    for name, case in (run_case("polygon_voronoi12_rt0_discs", 12, 3, (2, 3, 4), 1, 25, keep_cells=(0, 7)),
                       run_case("polygon_voronoi20_rt0s2_discs", 20, 11, (2, 4), 2, 40, keep_cells=(5,))):
        np.savez_compressed(HERE / f"{name}.npz", **case)
        print(name, "cells", case["count"], "N", len(case["rhs"]), "local sizes",
              int(np.diff(case["field_ptr"]).min()), int(np.diff(case["field_ptr"]).max()))


if __name__ == "__main__":
    main()
