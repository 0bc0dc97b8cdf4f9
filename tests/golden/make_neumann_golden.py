"""Write golden fixtures with Neumann faces on whole sides of the domain, by running
PyMHM itself: ``boundary_data`` prescribes those faces' trace coefficients (the L2
projection of the outward normal flux) and ``HybridSystem.solve(fixed=...)``
eliminates them, as ``solve_darcy_quadrilateral`` does (``_legacy/models/darcy/
cartesian.py:122-143``, ``core/system.py:421-447``).  For the left-and-bottom flux
case and the pure-Neumann case it also runs ``refine_hybrid`` with ``fixed`` (and, for
the latter, the mean-pressure moment) from a perturbed solution (every local field
plus 0.002 * (1, ..., n), as the reference's refinement test does).

    PYMHM_SRC=/path/to/pymhm/src python tests/golden/make_neumann_golden.py

Reuses the imports of ``make_golden`` (and its Basix shim).
"""

from __future__ import annotations

import numpy as np

from dataclasses import replace

from make_golden import (HERE, CartesianCellField, CartesianMacroMesh, FaceSpace, HybridSystem,
                         QuadrilateralDarcySolution, SkeletonSpace, _assemble_quad, _QuadTask, boundary_data,
                         lognormal_permeability, sine_source)
from pymhm.core.refinement import refine_hybrid


def side_faces(mesh, y=None, x=None):
    axis, value = (1, y) if x is None else (0, x)
    return [int(f) for f in mesh.boundary_faces if np.all(mesh.points[mesh.faces[f]][:, axis] == value)]


def pressure_drop(x):
    return 1.0 - x[:, 0]


def bottom_flux(x):
    return 0.5 + x[:, 0]


def vertical_drop(x):
    return 1.0 - x[:, 1]


def left_flux(x):
    return 0.3 - 0.2 * x[:, 1]


def run(name, mesh, face_space, refinement, permeability, source, dirichlet, neumann, refine=False,
        mean_pressure=None):
    sk = SkeletonSpace(mesh, (face_space,) * len(mesh.faces))
    order = 4
    boundary, fixed = boundary_data(sk, dirichlet, neumann, order=order)
    tasks = [_QuadTask(mesh, c, refinement, sk, 1, permeability, source, order) for c in range(len(mesh.cells))]
    system = HybridSystem.from_local_factory(_assemble_quad, tasks, boundary_load=boundary)
    constraints, moments = None, ()
    if mean_pressure is not None:  # pure Neumann: the driver's mean-pressure row (cartesian.py:135-142)
        _, means = zip(*system.local_metadata)
        constraints = [system.mean_constraint(means, mean_pressure * float(np.sum(mesh.areas)))]
        moments = ((means, mean_pressure * float(np.sum(mesh.areas))),)
    hybrid = system.solve(fixed=fixed, constraints=constraints)
    extra = {}
    if refine:
        perturbed = replace(hybrid, fields=tuple(u + 0.002 * np.arange(1, len(u) + 1) for u in hybrid.fields))
        result = refine_hybrid(system, perturbed, boundary_load=boundary, fixed=fixed, moments=moments,
                               max_steps=2, rtol=1e-10)
        extra = dict(
            refine_start_fields=np.array(perturbed.fields), refine_residual_norms=np.array(result.residual_norms),
            refine_rhs_norm=result.rhs_norm, refine_reduced=result.solution.residual,
            refine_trace=result.solution.trace, refine_coarse=np.concatenate(result.solution.coarse),
            refine_fields=np.array(result.solution.fields))
        print(name, "refinement history", result.residual_norms, "rhs", result.rhs_norm)
    fines = [meta[0] for meta in system.local_metadata]
    sol = QuadrilateralDarcySolution(sk, tuple(fines), hybrid.fields, (), hybrid, permeability, source, 1, order)
    flux = np.array([sol.evaluate(c, f.points[f.cells].mean(axis=1))[1] for c, f in enumerate(fines)])
    A = system.matrix.tocsc()
    keys = np.array(sorted(fixed), dtype=np.int64)
    return dict(
        boundary=boundary, fixed_dofs=keys, fixed_values=np.array([fixed[k] for k in keys]),
        neumann_faces=np.array(sorted(neumann), dtype=np.int64),
        indptr=A.indptr, indices=A.indices, data=A.data, rhs=system.rhs, load_scale=system.load_scale,
        trace=hybrid.trace, coarse=np.concatenate(hybrid.coarse), residual=hybrid.residual,
        fields=np.array(hybrid.fields), flux=flux, **extra,
    ), name


def main():
    mesh = CartesianMacroMesh(4)
    kap = lognormal_permeability(32, 32, sigma=2.0, ell=0.1, seed=31)
    field = CartesianCellField(kap, spacing=(1 / 32, 1 / 32))
    walls = {f: 0.0 for f in side_faces(mesh, 0.0) + side_faces(mesh, 1.0)}
    out, name = run("darcy_4x4_r8_p2_noflow_tb", mesh, FaceSpace.uniform(2), (8, 8), field, 1.0, pressure_drop,
                    walls)
    out["kappa"] = kap
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])
    flux_bottom = {f: bottom_flux for f in side_faces(mesh, 0.0)}
    out, name = run("poisson_4x4_r4_p1_flux_bottom", mesh, FaceSpace.uniform(1), (4, 4), 1.0, sine_source, 0.0,
                    flux_bottom)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])
    walls = {f: 0.0 for f in side_faces(mesh, x=0.0) + side_faces(mesh, x=1.0)}
    out, name = run("darcy_4x4_r8_p2_noflow_lr", mesh, FaceSpace.uniform(2), (8, 8), field, 1.0, vertical_drop,
                    walls)
    out["kappa"] = kap
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])
    mixed = {f: left_flux for f in side_faces(mesh, x=0.0)}
    mixed.update({f: bottom_flux for f in side_faces(mesh, 0.0)})
    out, name = run("poisson_4x4_r4_p1_flux_left_bottom", mesh, FaceSpace.uniform(1), (4, 4), 1.0, sine_source,
                    0.0, mixed, refine=True)
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])
    # Neumann data on part of two sides: an inflow through the middle of the left side,
    # no flow through the first half of the bottom and the whole top, Dirichlet 0 elsewhere
    partial = {f: -1.0 for f in side_faces(mesh, x=0.0)[1:3]}
    partial.update({f: 0.0 for f in side_faces(mesh, 0.0)[:2] + side_faces(mesh, 1.0)})
    out, name = run("darcy_4x4_r8_p2_partial_sides", mesh, FaceSpace.uniform(2), (8, 8), field, 0.0, 0.0, partial)
    out["kappa"] = kap
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])
    everywhere = {int(f): 0.25 for f in mesh.boundary_faces}  # outward flux 4 x 0.25 = the source's 1
    out, name = run("darcy_4x4_r8_p1_pure_neumann", mesh, FaceSpace.uniform(1), (8, 8), field, 1.0, 0.0,
                    everywhere, mean_pressure=0.3, refine=True)
    out["kappa"] = kap
    np.savez_compressed(HERE / f"{name}.npz", **out)
    print(name, "fixed", len(out["fixed_dofs"]), "residual", out["residual"])


if __name__ == "__main__":
    main()
