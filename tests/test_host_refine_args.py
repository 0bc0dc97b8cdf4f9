"""Argument contract of the refinement entry points (no GPU needed)."""

import math

import pytest

from pymhm_b200 import _lib
from pymhm_b200.darcy import _step_limits, _tolerances, solve_darcy_quadrilateral
from pymhm_b200.topology import CartesianMacroMesh


@pytest.mark.parametrize("steps", [-1, True, 1.5])
def test_invalid_step_counts(steps):
    with pytest.raises(ValueError, match="refinement_steps must be a nonnegative integer"):
        _step_limits(steps, 0)
    with pytest.raises(ValueError, match="hybrid_refinement_steps|refinement_steps"):
        solve_darcy_quadrilateral(CartesianMacroMesh(2), hybrid_refinement_steps=steps)


def test_step_interval_and_tolerances():
    with pytest.raises(ValueError, match="min_steps must not exceed max_steps"):
        _step_limits(1, 2)
    with pytest.raises(ValueError, match="hybrid_refinement_min_steps must not exceed"):
        solve_darcy_quadrilateral(CartesianMacroMesh(2), hybrid_refinement_steps=1, hybrid_refinement_min_steps=2)
    for rtol, atol in ((math.nan, 0.0), (-1.0, 0.0), (1e-10, math.inf)):
        with pytest.raises(ValueError, match="finite and nonnegative"):
            _tolerances(rtol, atol)
    with pytest.raises(ValueError, match="at least one tolerance"):
        _tolerances(0.0, 0.0)
    _step_limits(0, 0)
    _tolerances(1e-10, 0.0)


def test_nodal_load_source_mode_and_refinement_entry_points():
    lib = _lib.load()
    q = _lib.Q1Problem()
    q.macro_nx = q.macro_ny = 1
    q.rx = q.ry = 16
    q.hx = q.hy = 1.0 / 16
    q.tf_h = q.tf_v = 3
    q.coupling_table = q.side_sign = q.side_orient = 8
    q.source_mode = 3
    assert lib.mhm_q1_condense_smem_bytes(q, 0) == 0  # nodal loads need their array
    q.source = 8
    assert lib.mhm_q1_condense_smem_bytes(q, 0) > 0
    q.source_mode = 4
    assert lib.mhm_q1_condense_smem_bytes(q, 0) == 0
    q.source_mode = 3
    assert lib.mhm_q1_original_defect(q, None, 1, None, None, None, None, None, None, None, None, None, None,
                                      None) == _lib.MHM_ERR_ARGUMENT
    assert lib.mhm_refine_norms(0, None, 0, None, None, None, 0, None, None, None, None, None, None,
                                None) == _lib.MHM_ERR_ARGUMENT
    assert lib.mhm_skeleton_fixed_rhs(0, 0, None, None, None, None, None, None, None,
                                      None) == _lib.MHM_ERR_ARGUMENT
    assert lib.mhm_vector_accumulate(-1, None, None, None) == _lib.MHM_ERR_ARGUMENT
    assert lib.mhm_vector_accumulate(0, None, None, None) == _lib.MHM_OK
    assert lib.mhm_q1_correction_response(q, 0, 0, 1e-12, None, None, None, None, None, None,
                                          None) == _lib.MHM_ERR_ARGUMENT
