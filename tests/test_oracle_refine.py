"""The oracle's original-equation refinement against fixtures that PyMHM's own
``refine_hybrid`` wrote (tests/golden/make_refine_golden.py)."""

import numpy as np
import pytest

from oracle import q1_mhm as o
from tests._cases import load, rel
from tests.test_oracle_golden import oracle_case

REFINE_CASES = ["poisson_8x8_r4_p1", "darcy_4x4_r16_p2_lognormal"]


@pytest.mark.parametrize("name", REFINE_CASES)
def test_oracle_refinement_matches_reference(name):
    g, mesh, sk, ref, perm, src, dr = oracle_case(name)
    r = load(f"refine_{name}")
    out = o.refine_q1(mesh, sk, ref, r["start_trace"], r["start_coarse"], r["start_fields"], perm, src, dr,
                      max_steps=2, rtol=1e-10)
    hist = np.array(out["residual_norms"])
    assert len(hist) == len(r["residual_norms"])
    # the initial residual is that of the perturbed fields: same arithmetic up to rounding
    assert abs(hist[0] - r["residual_norms"][0]) <= 1e-12 * r["residual_norms"][0]
    assert abs(out["rhs_norm"] - float(r["rhs_norm"])) <= 1e-14 * float(r["rhs_norm"])
    assert hist[-1] <= 1e-10 * out["rhs_norm"]
    for key in ("trace", "coarse", "fields"):
        assert rel(out[key], r[key]) <= 1e-11, key
    # and the refined state is the unperturbed discrete solution
    assert rel(out["fields"], g["fields"]) <= 1e-11


def test_oracle_refinement_reports_failure_like_the_reference():
    g, mesh, sk, ref, perm, src, dr = oracle_case("poisson_8x8_r4_p1")
    r = load("refine_poisson_8x8_r4_p1")
    with pytest.raises(o.LinearSolveError, match=r"original hybrid residual .* after 0 corrections"):
        o.refine_q1(mesh, sk, ref, r["start_trace"], r["start_coarse"], r["start_fields"], perm, src, dr,
                    max_steps=0)
