"""Offline / online reuse (``core/offline.py``): new sources with the kept factors."""

import numpy as np
import pytest

from tests._cases import face_space, CASES, load, rel

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-10, "mixed": 1e-8}


def _setup(name):
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    g = load(name)
    margs, face, ref, perm, src, dr = CASES[name]
    mesh = CartesianMacroMesh(*margs)
    sk = SkeletonSpace(mesh, (face_space(FaceSpace, face),) * len(mesh.faces))
    return g, mesh, sk, ref, perm(g), src, dr


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["darcy_4x4_r16_p2_lognormal", "poisson_8x8_r4_p1"])
def test_online_source_matches_reference(name, precision):
    """Prepared with another source, queried with the fixture's: the reference solution."""
    from pymhm_b200.offline import OfflineQ1System

    g, mesh, sk, ref, perm, src, dr = _setup(name)
    with OfflineQ1System(mesh, sk, ref, permeability=perm, source=0.37, dirichlet=dr, precision=precision) as off:
        sol = off.solve(src)
        tol = TOL[precision]
        assert rel(sol.trace, g["trace"]) <= tol
        assert rel(sol.coarse, g["coarse"]) <= tol
        assert rel(sol.fields, g["fields"]) <= tol
        assert rel(sol.flux, g["flux"]) <= tol
        assert sol.residual <= 1e-12


def test_online_equals_a_fresh_solve():
    """Several sources in order (``solve_many``) equal fresh full solves."""
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.offline import OfflineQ1System

    g, mesh, sk, ref, perm, src, dr = _setup("darcy_4x4_r16_p2_lognormal")
    sources = [1.0, lambda x: np.sin(3 * x[:, 0]) * x[:, 1], 2.5]
    with OfflineQ1System(mesh, sk, ref, permeability=perm, source=0.0, dirichlet=dr) as off:
        online = off.solve_many(sources)
    for s, on in zip(sources, online):
        plan = CartesianQ1Plan(mesh, sk, ref, dirichlet=dr)
        full = plan.solve(perm, s)
        assert rel(on.trace, full.trace) <= 1e-11
        assert rel(on.fields, full.fields) <= 1e-11
        assert rel(on.flux, full.flux) <= 1e-11


def test_online_needs_the_offline_step():
    from pymhm_b200.darcy import CartesianQ1Plan

    g, mesh, sk, ref, perm, src, dr = _setup("poisson_8x8_r4_p1")
    plan = CartesianQ1Plan(mesh, sk, ref, dirichlet=dr)
    plan.set_coefficients(perm, src)
    with pytest.raises(RuntimeError):
        plan.launch(local="online")
    assert plan.lib.mhm_q1_factor_bytes(plan.q1, 0) == 64 * 5 * 5 * 5 * 8
    assert plan.lib.mhm_q1_factor_bytes(plan.q1, 1) == 64 * 5 * 5 * 5 * 4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_captured_online_query_matches_eager(precision):
    """One online query captured as a CUDA graph gives the eager query's bits, for a
    constant and for a per-fine-cell source, replay after replay."""
    import torch

    from tests.test_gpu_darcy import make_plan

    g, plan = make_plan("darcy_4x4_r16_p2_lognormal", precision)
    plan.prepare_offline()
    rng = np.random.default_rng(4)
    cells = rng.uniform(0.5, 2.0, (plan.nxf, plan.nyf))
    eager = {}
    for key, src in (("const", 1.75), ("cells", cells)):
        sol = plan.solve_source(src)
        eager[key] = (sol.fields.copy(), sol.trace.copy())
    plan.capture_online()
    for _ in range(2):
        for key, src in (("const", 1.75), ("cells", cells)):
            st = plan.replay_online(src)
            st.synchronize()
            plan.check()
            assert np.array_equal(plan.fields.cpu().numpy(), eager[key][0])
            assert np.array_equal(plan.x.cpu().numpy()[: plan.T], eager[key][1])
    torch.cuda.synchronize()


@pytest.mark.parametrize("name", ["poisson_8x8_r4_p1", "darcy_4x4_r8_p1_cut20"])
def test_captured_fresh_solve_matches_eager(name):
    """capture('condense'): one complete fresh solve as a CUDA graph, pointwise source and
    cut-cell material included, gives the eager solve's bits; a coefficient change after
    the capture is refused instead of replaying stale buffers."""
    import torch

    from tests._cases import CASES
    from tests.test_gpu_darcy import make_plan

    g, plan = make_plan(name, "mixed")
    plan.launch()
    eager = plan.result()
    plan.capture("condense")
    for _ in range(2):
        plan.fields.zero_()
        plan.replay("condense").synchronize()
        sol = plan.result()
        assert np.array_equal(sol.fields, eager.fields)
        assert np.array_equal(sol.trace, eager.trace)
        assert np.array_equal(sol.flux, eager.flux)
    with pytest.raises(ValueError):
        plan.replay("condense", 1.0)
    perm, src = CASES[name][3], CASES[name][4]
    plan.set_coefficients(perm(g), src)
    with pytest.raises(RuntimeError, match="changed since capture"):
        plan.replay("condense")
    torch.cuda.synchronize()
