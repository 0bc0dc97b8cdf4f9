"""The serving loop (pymhm_b200.serving): every request's result is the same alone and
in the mix, agrees with an independent solve, and admission respects the HBM budget."""

import numpy as np
import pytest

from tests._cases import rel

pytestmark = pytest.mark.gpu


def make_requests(count=6, seed=11):
    from pymhm_b200.serving import DarcyRequest
    from pymhm_b200.workloads import lognormal_permeability

    rng = np.random.default_rng(seed)
    shapes = [(4, 4), (8, 4), (4, 8), (8, 8), (4, 16), (8, 16)]
    reqs = []
    for i in range(count):
        macro, ref = shapes[i % len(shapes)]
        n = macro * ref
        kappa = lognormal_permeability(n, n, sigma=float(rng.uniform(1, 2)), ell=0.1, seed=int(rng.integers(1 << 30)))
        sources = tuple(float(v) for v in rng.uniform(0.5, 2.0, int(rng.integers(1, 4))))
        reqs.append(DarcyRequest(macro, ref, kappa, sources, arrival=0.004 * i))
    return reqs


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_results_are_the_same_alone_and_in_the_mix(precision):
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.serving import ServingEngine
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    reqs = make_requests()
    mix = ServingEngine(precision=precision, max_in_flight=4, keep_fields=True)
    together = mix.run(reqs, realtime=False)
    assert mix.stats["peak_in_flight"] > 1
    alone = ServingEngine(precision=precision, max_in_flight=1, keep_fields=True).run(reqs, realtime=False)
    for req, a, b in zip(reqs, together, alone):
        assert len(a.x) == len(req.sources)
        for k in range(len(req.sources)):
            assert np.array_equal(a.x[k], b.x[k])
            assert np.array_equal(a.fields[k], b.fields[k])
            assert np.array_equal(a.flux[k], b.flux[k])
    # and each agrees with a fresh plan solving the same request source by source
    tol = 1e-10 if precision == "fp64" else 1e-8
    for req, res in zip(reqs, together):
        mesh = CartesianMacroMesh(req.macro)
        sk = SkeletonSpace(mesh, (FaceSpace.uniform(req.face_degree),) * len(mesh.faces))
        plan = CartesianQ1Plan(mesh, sk, req.refinement, precision=precision)
        for k, src in enumerate(req.sources):
            sol = plan.solve(req.permeability, src)
            assert rel(res.fields[k], sol.fields) <= tol
            assert rel(res.x[k][: plan.T], sol.trace) <= tol


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batched_local_stages_give_the_same_results(precision):
    """Requests of one shape admitted together share one local-stage launch
    (``condense_batch``); every source of every request equals the unbatched loop's
    result bit for bit."""
    from pymhm_b200.serving import DarcyRequest, ServingEngine
    from pymhm_b200.workloads import lognormal_permeability

    rng = np.random.default_rng(23)
    reqs = []
    for i in range(8):
        macro, ref = [(8, 8), (4, 16)][i % 2]
        n = macro * ref
        kappa = lognormal_permeability(n, n, sigma=2.0, ell=0.1, seed=int(rng.integers(1 << 30)))
        sources = tuple(float(v) for v in rng.uniform(0.5, 2.0, int(rng.integers(1, 4))))
        reqs.append(DarcyRequest(macro, ref, kappa, sources))
    batched = ServingEngine(precision=precision, max_in_flight=8, keep_fields=True, batch_local=True)
    got = batched.run(reqs, realtime=False)
    assert batched.stats["batched_requests"] == 8 and batched.stats["batched_local_launches"] == 2
    plain = ServingEngine(precision=precision, max_in_flight=8, keep_fields=True)
    ref = plain.run(reqs, realtime=False)
    assert "batched_requests" not in plain.stats
    for req, a, b in zip(reqs, got, ref):
        for k in range(len(req.sources)):
            assert np.array_equal(a.x[k], b.x[k])
            assert np.array_equal(a.fields[k], b.fields[k])
            assert np.array_equal(a.flux[k], b.flux[k])


def test_admission_respects_the_hbm_budget():
    from pymhm_b200.serving import ServingEngine

    reqs = [r for r in make_requests(8) if (r.macro, r.refinement) == (8, 8)] or make_requests(4)[:2]
    probe = ServingEngine(max_in_flight=4)
    probe.run(reqs[:1], realtime=False)
    one = probe.stats["peak_bytes"]
    engine = ServingEngine(max_in_flight=4, hbm_budget=1.5 * one, keep_fields=True)
    out = engine.run(reqs * 3, realtime=False)
    assert engine.stats["peak_in_flight"] == 1
    assert engine.stats["peak_bytes"] <= 1.5 * one
    for a, b in zip(out, out[len(reqs):]):
        assert np.array_equal(a.fields[0], b.fields[0])
    with pytest.raises(ValueError, match="HBM budget"):
        ServingEngine(hbm_budget=one / 2).run(reqs[:1], realtime=False)


def test_realtime_arrivals_and_latency():
    from pymhm_b200.serving import ServingEngine, summarize

    reqs = make_requests(6)
    out = ServingEngine(max_in_flight=3).run(reqs)
    for req, res in zip(reqs, out):
        assert res.admitted >= req.arrival - 1e-6
        assert res.finished >= res.admitted
        assert res.latency > 0
    s = summarize(out)
    assert s["requests"] == 6 and s["rhs"] == sum(len(r.sources) for r in reqs)
    assert s["latency_ms"]["p99"] >= s["latency_ms"]["p50"] > 0


def test_reserved_slots_and_eviction_under_the_budget():
    """Reserved slots serve later requests without new plans; when the budget is full,
    idle slots of other shapes make room for a new shape; a shape larger than the
    whole budget is rejected."""
    from pymhm_b200.serving import ServingEngine

    reqs = make_requests(6)
    small_reqs = [r for r in reqs if (r.macro, r.refinement) == (4, 4)]
    big_reqs = [r for r in reqs if (r.macro, r.refinement) == (8, 4)]
    engine = ServingEngine(max_in_flight=2, keep_fields=True)
    assert engine.reserve((4, 4, 2), 2) == 2
    assert engine.reserve((8, 4, 2), 1) == 1
    created = engine.stats["slots_created"]
    engine.run(small_reqs * 2, realtime=False)
    assert engine.stats["slots_created"] == created
    small, big = engine._shape_bytes[(4, 4, 2)], engine._shape_bytes[(8, 4, 2)]
    tight = ServingEngine(max_in_flight=1, hbm_budget=big + 1.2 * small, keep_fields=True)
    assert tight.reserve((4, 4, 2), 2) == 2
    out = tight.run(small_reqs + big_reqs, realtime=False)
    assert all(o is not None for o in out)
    assert tight._bytes() <= tight.hbm_budget
    assert any(s.shape == (8, 4, 2) for s in tight.slots)
    with pytest.raises(ValueError, match="HBM budget"):
        ServingEngine(hbm_budget=0.5 * big).run(big_reqs, realtime=False)


def test_captured_offline_step_matches_eager():
    """The offline step (factors kept) replayed from its CUDA graph gives the eager
    launch's bits."""
    import torch

    from tests.test_gpu_darcy import make_plan

    g, plan = make_plan("darcy_4x4_r16_p2_lognormal", "mixed")
    kappa = torch.from_numpy(np.ascontiguousarray(g["kappa"])).to(plan.device)
    plan.set_device_coefficients(1, kappa, (0.0, 0.0, 0.0), 0, None, 1.0)
    plan.launch(local="offline")
    plan.check()
    eager = plan.fields.cpu().numpy().copy()
    plan.capture("offline")
    plan.fields.zero_()
    st = plan.replay("offline", 1.0)
    st.synchronize()
    plan.check()
    assert np.array_equal(plan.fields.cpu().numpy(), eager)
