"""Pixel fields whose lines cut the fine cells (kappa modes 3/4): exact integration of
every fine cell over its pixel intersections (``fem/scalar/quadrilateral.py:136-188,
215-234``).  The reference-written fixture ``darcy_4x4_r8_p1_cut20`` runs through the
common parity tests; these cover the tensor mode, shifted pixel origins, agreement with
the per-cell path on aligned fields, and the refinement and online paths."""

import numpy as np
import pytest

from oracle import q1_mhm as o
from tests._cases import PixelField, load, rel
from tests.test_gpu_darcy import make_plan

pytestmark = pytest.mark.gpu


def plan_for(macro, deg, refinement, precision="fp64"):
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    mesh = CartesianMacroMesh(*macro)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(deg),) * len(mesh.faces))
    return CartesianQ1Plan(mesh, sk, refinement, precision=precision)


def oracle_solution(macro, deg, refinement, field, source):
    mesh = o.cartesian_mesh(*macro)
    sk = o.Skeleton(mesh, (o.FaceSpace.uniform(deg),) * len(mesh.faces))
    return o.solve_darcy_q1(mesh, sk, refinement, o.PixelField(field.values, field.spacing, field.origin), source)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tensor_pixels_with_shifted_origin_match_oracle(precision):
    rng = np.random.default_rng(7)
    nx, ny = 11, 9
    kxx = np.exp(rng.normal(scale=1.0, size=(nx, ny)))
    kyy = np.exp(rng.normal(scale=1.0, size=(nx, ny)))
    kxy = 0.4 * np.sqrt(kxx * kyy) * rng.uniform(-1, 1, size=(nx, ny))
    tens = np.stack((np.stack((kxx, kxy), -1), np.stack((kxy, kyy), -1)), -2)
    field = PixelField(tens, (0.1, 0.125), (-0.03, -0.07))
    plan = plan_for((3,), 1, (6, 6), precision)
    plan.set_coefficients(field, 1.0)
    assert plan.q1.kappa_mode == 4
    plan.launch()
    sol = plan.result()
    ref = oracle_solution((3,), 1, (6, 6), field, 1.0)
    tol = 1e-10 if precision == "fp64" else 1e-8
    assert rel(sol.trace, ref.trace) <= tol
    assert rel(sol.coarse, ref.coarse) <= tol
    assert rel(sol.fields, ref.fields) <= tol
    assert rel(sol.flux, ref.flux) <= tol


def test_pixels_finer_than_fine_cells_match_oracle():
    """Many pixels per fine cell: every intersection is summed."""
    rng = np.random.default_rng(11)
    kap = np.exp(rng.normal(scale=1.2, size=(37, 29)))
    field = PixelField(kap, (1 / 37, 1 / 29))
    plan = plan_for((2,), 1, (4, 4))
    plan.set_coefficients(field, 1.0)
    assert plan.q1.kappa_mode == 3
    plan.launch()
    sol = plan.result()
    ref = oracle_solution((2,), 1, (4, 4), field, 1.0)
    assert rel(sol.fields, ref.fields) <= 1e-10
    assert rel(sol.trace, ref.trace) <= 1e-10
    assert rel(sol.flux, ref.flux) <= 1e-10


def test_aligned_field_through_cut_mode_equals_cell_mode():
    """The closed-form intersection integrals reduce to the per-cell element on aligned
    fields: forcing the cut mode changes results only at rounding level."""
    import torch

    g = load("darcy_4x4_r16_p2_lognormal")
    _, plan = make_plan("darcy_4x4_r16_p2_lognormal", "fp64")
    plan.launch()
    base = plan.result()
    kap = torch.from_numpy(np.ascontiguousarray(g["kappa"])).to(plan.device)
    plan.set_device_coefficients(3, kap, (0.0, 0.0, 0.0), 0, None, 1.0,
                                 pixels=((0.0, 0.0), (1 / 64, 1 / 64), (64, 64)))
    plan.launch()
    cut = plan.result()
    assert rel(cut.fields, base.fields) <= 1e-12
    assert rel(cut.trace, base.trace) <= 1e-12
    assert rel(cut.flux, base.flux) <= 1e-12
    assert rel(cut.fields, g["fields"]) <= 1e-10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cut_refinement_and_online_query(precision):
    g, plan = make_plan("darcy_4x4_r8_p1_cut20", precision)
    assert plan.q1.kappa_mode == 3
    plan.prepare_offline()
    sol = plan.solve_source(1.0)
    assert rel(sol.fields, g["fields"]) <= (1e-10 if precision == "fp64" else 1e-8)
    out = plan.refine(max_steps=2, min_steps=1)
    assert out.residual_norms[-1] <= 1e-10 * out.rhs_norm
    assert rel(out.solution.fields, g["fields"]) <= 1e-10
    with pytest.raises(NotImplementedError, match="cut load quadrature"):
        plan.set_source(lambda p: 1.0 + p[:, 0])
