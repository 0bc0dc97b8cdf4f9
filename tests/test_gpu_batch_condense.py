"""Cross-request batching of the Cartesian local stage: one ``mhm_q1_condense_batch``
launch over the cells of several independent problems of one shape gives each
problem exactly the responses, Schur blocks, status words and final solution of its
own launch, in both precisions and with kept factors for later sources."""

import numpy as np
import pytest
import torch

from tests._cases import rel

pytestmark = pytest.mark.gpu


def make_plans(count, precision, macro=8, refinement=8):
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import lognormal_permeability

    plans, fields = [], []
    for k in range(count):
        mesh = CartesianMacroMesh(macro)
        sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
        plans.append(CartesianQ1Plan(mesh, sk, refinement, precision=precision))
        fields.append(lognormal_permeability(macro * refinement, sigma=2.0, ell=0.1, seed=900 + k))
    return plans, fields


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_local_stage_equals_separate_launches(precision):
    from pymhm_b200.darcy import condense_batch

    alone, fields = make_plans(3, precision)
    for plan, kappa in zip(alone, fields):
        plan.set_coefficients(kappa, 1.0)
        plan.launch()
    ref = [plan.result() for plan in alone]
    batch, _ = make_plans(3, precision)
    for plan, kappa in zip(batch, fields):
        plan.set_coefficients(kappa, 1.0)
    condense_batch(batch)
    for plan in batch:
        plan.launch(local="batched")
    torch.cuda.synchronize()
    for a, b, r in zip(alone, batch, ref):
        for name in ("solution", "blocks", "loads", "cell_status", "cell_iters", "corrected"):
            assert torch.equal(getattr(a, name), getattr(b, name)), name
        sol = b.result()
        assert np.array_equal(sol.trace, r.trace) and np.array_equal(sol.fields, r.fields)


def test_batched_offline_stage_keeps_factors():
    """``offline=True`` keeps every plan's factors: a later source on each plan gives the
    same solution as the plan's own offline step followed by that source."""
    from pymhm_b200.darcy import condense_batch

    alone, fields = make_plans(2, "mixed")
    for plan, kappa in zip(alone, fields):
        plan.set_coefficients(kappa, 1.0)
        plan.prepare_offline()
    ref = [plan.solve_source(-2.5) for plan in alone]
    batch, _ = make_plans(2, "mixed")
    for plan, kappa in zip(batch, fields):
        plan.set_coefficients(kappa, 1.0)
    condense_batch(batch, offline=True)
    for plan in batch:
        plan.launch(local="batched")
    got = [plan.solve_source(-2.5) for plan in batch]
    for a, b in zip(ref, got):
        assert rel(b.trace, a.trace) == 0.0 and rel(b.fields, a.fields) == 0.0


def test_batched_local_stage_rejects_mixed_shapes():
    from pymhm_b200.darcy import condense_batch

    a, fa = make_plans(1, "fp64", macro=8)
    b, fb = make_plans(1, "fp64", macro=4)
    a[0].set_coefficients(fa[0], 1.0)
    b[0].set_coefficients(fb[0], 1.0)
    with pytest.raises(ValueError, match="one shape"):
        condense_batch(a + b)
