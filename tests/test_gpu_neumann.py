"""GPU parity with Neumann faces: the prescribed trace DOFs are eliminated
(mhm_skeleton_fixed_rhs + the masked projected CG, whose coarse operator takes whole
Neumann sides as Neumann ends of its 1-D factors and corrects faces on parts of sides
by a Woodbury factor) as PyMHM's solve_hybrid_system does with ``fixed``."""

import numpy as np
import pytest

from tests._cases import PixelField, load, rel
from tests.test_oracle_neumann import MEAN_PRESSURE, NEUMANN_CASES, neumann_map

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}


def make_plan(name, precision):
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    g = load(name)
    deg, ref, perm, src, dr, val = NEUMANN_CASES[name]
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(deg),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, ref, dirichlet=dr, neumann=neumann_map(g, val, mesh),
                           mean_pressure=MEAN_PRESSURE.get(name, 0.0), precision=precision)
    kap = PixelField(g["kappa"], (1 / 32, 1 / 32)) if "kappa" in g else 1.0
    plan.set_coefficients(kap, src)
    return g, plan


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(NEUMANN_CASES))
def test_neumann_solution_matches_reference(name, precision):
    g, plan = make_plan(name, precision)
    plan.launch()
    sol = plan.result()
    tol = TOL[precision]
    assert rel(sol.trace, g["trace"]) <= tol
    assert rel(sol.coarse, g["coarse"]) <= tol
    assert rel(sol.fields, g["fields"]) <= tol
    assert rel(sol.flux, g["flux"]) <= tol
    # the prescribed coefficients come back exactly
    assert np.array_equal(sol.trace[g["fixed_dofs"]], g["fixed_values"]) or \
        np.max(np.abs(sol.trace[g["fixed_dofs"]] - g["fixed_values"])) <= 1e-15
    assert sol.residual <= 1e-12


def test_neumann_online_and_captured_paths():
    g, plan = make_plan("darcy_4x4_r8_p2_noflow_tb", "fp64")
    plan.prepare_offline()
    sol = plan.solve_source(1.0)
    assert rel(sol.fields, g["fields"]) <= 1e-10
    plan.capture("condense")
    plan.replay("condense").synchronize()
    assert rel(plan.result().fields, g["fields"]) <= 1e-10


def test_driver_accepts_neumann_sides():
    from pymhm_b200.darcy import solve_darcy_quadrilateral
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    name = "poisson_4x4_r4_p1_flux_bottom"
    g = load(name)
    deg, ref, perm, src, dr, val = NEUMANN_CASES[name]
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(deg),) * len(mesh.faces))
    sol = solve_darcy_quadrilateral(mesh, skeleton=sk, local_refinement=ref, source=src, dirichlet=dr,
                                    neumann=neumann_map(g, val, mesh))
    assert rel(sol.fields, g["fields"]) <= 1e-10
    with pytest.raises(ValueError, match="boundary faces"):
        solve_darcy_quadrilateral(mesh, skeleton=sk, local_refinement=ref, neumann={int(mesh.faces.shape[0]) + 5: 0.0})


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["poisson_4x4_r4_p1_flux_left_bottom", "darcy_4x4_r8_p1_pure_neumann"])
def test_neumann_refinement_matches_reference(name, precision):
    """refine_hybrid with prescribed trace coefficients (core/refinement.py:676-709, 792):
    the right-hand-side norm takes the loads less the fixed traces' coupling, the weak
    residual the free DOFs, and the corrections hold the fixed DOFs at zero.  The
    pure-Neumann case also carries its mean-pressure moment (:690-700, 725-733)."""
    import torch

    g, plan = make_plan(name, precision)
    plan.launch()
    plan.check()
    plan.fields.copy_(torch.from_numpy(g["refine_start_fields"].reshape(plan.cells, plan.n)).to(plan.device))
    out = plan.refine(max_steps=2, rtol=1e-10)
    hist = np.array(out.residual_norms)
    ref_hist = g["refine_residual_norms"]
    assert len(ref_hist) <= len(hist) <= len(ref_hist) + (precision == "mixed")
    assert abs(hist[0] - ref_hist[0]) <= 1e-11 * ref_hist[0]
    assert abs(out.rhs_norm - float(g["refine_rhs_norm"])) <= 1e-13 * float(g["refine_rhs_norm"])
    assert hist[-1] <= 1e-10 * out.rhs_norm
    sol = out.solution
    assert rel(sol.trace, g["refine_trace"]) <= 1e-10
    assert rel(sol.coarse, g["refine_coarse"]) <= 1e-10
    assert rel(sol.fields, g["refine_fields"]) <= 1e-10
    # the prescribed coefficients are untouched by the corrections
    assert np.max(np.abs(sol.trace[g["fixed_dofs"]] - g["fixed_values"])) <= 1e-15


def test_pure_neumann_mean_pressure():
    """Every side Neumann: the pressure mean over the domain is the requested one (the
    reference's gauge row)."""
    g, plan = make_plan("darcy_4x4_r8_p1_pure_neumann", "fp64")
    plan.launch()
    sol = plan.result()
    fine_area = (0.25 / 8) ** 2
    nodes = 9
    ix, iy = np.meshgrid(np.arange(nodes), np.arange(nodes), indexing="xy")
    weights = (np.where((ix == 0) | (ix == 8), 1.0, 2.0) * np.where((iy == 0) | (iy == 8), 1.0, 2.0)).ravel()
    mean = float(np.sum(sol.fields * weights[None, :]) * fine_area / 4)
    assert abs(mean - 0.3) <= 1e-12


def test_neumann_faces_on_parts_of_sides_only():
    """No whole side Neumann: the prescribed faces still leave the solve (the plan keys
    the fixed-DOF set-up on any Neumann face, not on whole sides)."""
    from oracle import q1_mhm as o
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import sine_source

    mesh = CartesianMacroMesh(4)
    bottom = [int(f) for f in mesh.boundary_faces if np.all(mesh.points[mesh.faces[f]][:, 1] == 0.0)]
    right = [int(f) for f in mesh.boundary_faces if np.all(mesh.points[mesh.faces[f]][:, 0] == 1.0)]
    neumann = {bottom[1]: 0.4, bottom[2]: 0.4, right[3]: -0.2}
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(1),) * len(mesh.faces))
    plan = CartesianQ1Plan(mesh, sk, (4, 4), neumann=neumann)
    assert plan.neumann_bits == 0 and plan.d_fixed is not None
    plan.set_coefficients(1.0, sine_source)
    plan.launch()
    sol = plan.result()
    om = o.cartesian_mesh(4)
    osk = o.Skeleton(om, (o.FaceSpace.uniform(1),) * len(om.faces))
    ref = o.solve_darcy_q1(om, osk, (4, 4), 1.0, sine_source, neumann=neumann)
    assert rel(sol.trace, ref.trace) <= 1e-10
    assert rel(sol.fields, ref.fields) <= 1e-10
    assert rel(sol.flux, ref.flux) <= 1e-10


def test_skeleton_factorization_serves_the_reduced_system():
    """SkeletonFactorization(fixed=...) behind solve_hybrid_system(fixed=...): it matches
    the system with the fixed rows and columns removed and solves it
    (core/system.py:421-457), here on the reference's own partial-sides system."""
    from scipy import sparse

    from pymhm_b200 import SkeletonFactorization
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    g = load("darcy_4x4_r8_p2_partial_sides")
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    n = len(g["rhs"])
    matrix = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(n, n))
    fixed = g["fixed_dofs"]
    x = np.zeros(n)
    x[fixed] = g["fixed_values"]
    free = np.setdiff1d(np.arange(n), fixed)
    reduced = matrix[free][:, free]
    rhs = g["rhs"][free] - (matrix @ x)[free]
    with SkeletonFactorization(matrix, mesh, sk, fixed=fixed) as fact:
        assert fact.matches(reduced) and not fact.matches(matrix)
        x[free] = fact.solve(rhs)
    t = sk.size
    assert rel(x[:t], g["trace"]) <= 1e-10
    assert rel(x[t:], g["coarse"]) <= 1e-10
    with pytest.raises(NotImplementedError, match="all trace DOFs"):
        SkeletonFactorization(matrix, mesh, sk, fixed=fixed[:-1])
