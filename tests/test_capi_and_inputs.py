"""C ABI surface (no GPU needed) and host-side input validation."""

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from pymhm_b200 import _lib
from pymhm_b200.darcy import (_cut_source_check, grid_resolves_material, permeability_input, pixel_geometry,
                               source_input)
from pymhm_b200.topology import CartesianMacroMesh
from pymhm_b200.workloads import digest, lognormal_permeability
from tests._cases import PixelField, load

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "mhm_b200.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*)\s+(mhm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 10
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_lib.declared_symbols())
    assert lib.mhm_version().startswith(b"mhm_b200")


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "mhm_b200.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(mhm_q1_problem),"
        " offsetof(mhm_q1_problem, kappa_const), offsetof(mhm_q1_problem, quad_order),"
        " sizeof(mhm_skeleton_system), offsetof(mhm_skeleton_system, nx),"
        " offsetof(mhm_skeleton_system, coarse_ay), offsetof(mhm_q1_problem, pixel_origin),"
        " offsetof(mhm_q1_problem, pixel_ny), sizeof(mhm_general_system), offsetof(mhm_general_system, cells),"
        " offsetof(mhm_general_system, coarse_inverse), offsetof(mhm_general_system, block_off),"
        " offsetof(mhm_general_system, max_trace_row), sizeof(mhm_ragged_matrix),"
        " offsetof(mhm_ragged_matrix, slot)); return 0;}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [ctypes.sizeof(_lib.Q1Problem), _lib.Q1Problem.kappa_const.offset, _lib.Q1Problem.quad_order.offset,
            ctypes.sizeof(_lib.SkeletonSystem), _lib.SkeletonSystem.nx.offset, _lib.SkeletonSystem.coarse_ay.offset,
            _lib.Q1Problem.pixel_origin.offset, _lib.Q1Problem.pixel_ny.offset, ctypes.sizeof(_lib.GeneralSystem),
            _lib.GeneralSystem.cells.offset, _lib.GeneralSystem.coarse_inverse.offset,
            _lib.GeneralSystem.block_off.offset, _lib.GeneralSystem.max_trace_row.offset,
            ctypes.sizeof(_lib.RaggedMatrix), _lib.RaggedMatrix.slot.offset]
    assert got == want


def test_argument_errors_need_no_gpu():
    """Entry points validate sizes before touching the device."""
    lib = _lib.load()
    assert lib.mhm_batched_factor(0, 3, None, None, None, None, None, None, None) == _lib.MHM_ERR_ARGUMENT
    assert lib.mhm_skeleton_scatter(-1, None, None, None, None, 1, 0, None, None, None, None, None, None,
                                    None) == _lib.MHM_ERR_ARGUMENT
    q = _lib.Q1Problem()
    assert lib.mhm_q1_condense_smem_bytes(q, 0) == 0
    q.macro_nx = q.macro_ny = 1
    q.rx = q.ry = 16
    q.hx = q.hy = 1.0 / 16
    q.tf_h = q.tf_v = 3
    assert lib.mhm_q1_rhs_width(q) == 14
    assert lib.mhm_q1_condense_smem_bytes(q, 0) == 0  # null tables rejected
    q.coupling_table = q.side_sign = q.side_orient = 8
    assert 0 < lib.mhm_q1_condense_smem_bytes(q, 0) <= 227 * 1024
    assert lib.mhm_q1_condense_smem_bytes(q, 1) < lib.mhm_q1_condense_smem_bytes(q, 0)
    q.rx = q.ry = 40
    assert lib.mhm_q1_condense_smem_bytes(q, 0) == 0  # too large for the on-chip layout


def test_pixel_field_mapping_and_alignment():
    g = load("darcy_4x4_r16_p2_lognormal")
    mesh = CartesianMacroMesh(4)
    mode, arr, _ = permeability_input(PixelField(g["kappa"], (1 / 64, 1 / 64)), mesh, 16, 16, 4)
    assert mode == 1 and np.array_equal(arr, g["kappa"])
    coarse = np.arange(1, 17, dtype=float).reshape(4, 4)
    mode, arr, _ = permeability_input(PixelField(coarse, (0.25, 0.25)), mesh, 16, 16, 4)
    assert mode == 1 and np.array_equal(arr, np.repeat(np.repeat(coarse, 16, 0), 16, 1))
    # pixel lines that cut the fine cells: pixels passed as they are (cut-cell modes)
    mode, arr, _ = permeability_input(PixelField(coarse, (0.3, 0.25)), mesh, 16, 16, 4)
    assert mode == 3 and np.array_equal(arr, coarse)
    assert pixel_geometry(PixelField(coarse, (0.3, 0.25)), mesh, 16, 16) == ((0.0, 0.0), (0.3, 0.25), (4, 4))
    assert not grid_resolves_material(PixelField(coarse, (0.3, 0.25)), mesh, 16, 16)
    assert grid_resolves_material(PixelField(coarse, (0.25, 0.25), (0.0, -1 / 64)), mesh, 16, 16)
    # a shifted origin alone also cuts
    mode, _, _ = permeability_input(PixelField(np.ones((5, 5)), (0.25, 0.25), (-0.01, -0.01)), mesh, 16, 16, 4)
    assert mode == 3
    ptens = np.broadcast_to(np.array([[2.0, 0.5], [0.5, 3.0]]), (4, 4, 2, 2))
    mode, arr, _ = permeability_input(PixelField(ptens, (0.3, 0.3)), mesh, 16, 16, 4)
    assert mode == 4 and arr.shape == (4, 4, 3) and np.all(arr[..., 1] == 0.5)
    with pytest.raises(ValueError, match="outside the Cartesian material field"):
        permeability_input(PixelField(coarse, (0.2, 0.25)), mesh, 16, 16, 4)
    with pytest.raises(ValueError, match="outside the Cartesian material field"):
        permeability_input(PixelField(coarse, (0.3, 0.3), (0.01, 0.0)), mesh, 16, 16, 4)
    with pytest.raises(NotImplementedError, match="cut load quadrature"):
        _cut_source_check(2)
    _cut_source_check(0)
    _cut_source_check(1)
    with pytest.raises(ValueError, match="positive definite"):
        permeability_input(-1.0, mesh, 16, 16, 4)
    with pytest.raises(ValueError, match="positive definite"):
        permeability_input(np.zeros((64, 64)), mesh, 16, 16, 4)
    tens = np.zeros((64, 64, 2, 2))
    tens[..., 0, 0], tens[..., 1, 1], tens[..., 0, 1], tens[..., 1, 0] = 2.0, 3.0, 0.5, 0.5
    mode, arr, _ = permeability_input(tens, mesh, 16, 16, 4)
    assert mode == 2 and arr.shape == (64, 64, 3) and np.all(arr[..., 1] == 0.5)
    assert permeability_input(np.diag([2.0, 3.0]), mesh, 16, 16, 4)[2] == (2.0, 0.0, 3.0)


def test_callable_inputs():
    mesh = CartesianMacroMesh(2)
    mode, arr, _ = permeability_input(lambda p: 1.0 + (p[:, 0] > 0.5), mesh, 4, 4, 4)
    assert mode == 1 and arr.shape == (8, 8) and arr[0, 0] == 1.0 and arr[7, 0] == 2.0
    # varying inside the fine cells: every Gauss point plus the centre (modes 5/6)
    mode, arr, _ = permeability_input(lambda p: 1.0 + p[:, 0], mesh, 4, 4, 4)
    assert mode == 5 and arr.shape == (8, 8, 17)
    assert np.isclose(arr[0, 0, 16], 1.0 + 1 / 16) and np.isclose(arr[7, 0, 16], 1.0 + 15 / 16)
    tens = lambda p: np.stack((np.stack((1.0 + p[:, 0], 0.1 * p[:, 1]), -1),
                               np.stack((0.1 * p[:, 1], 2.0 + p[:, 1]), -1)), -2)
    mode, arr, _ = permeability_input(tens, mesh, 4, 4, 4)
    assert mode == 6 and arr.shape == (8, 8, 17, 3)
    with pytest.raises(ValueError, match="positive definite"):
        permeability_input(lambda p: p[:, 0] - 0.5, mesh, 4, 4, 4)
    mode, arr, _ = source_input(lambda p: p[:, 0] + 10 * p[:, 1], mesh, 4, 4, 4)
    assert mode == 2 and arr.shape == (8, 8, 16)
    from numpy.polynomial.legendre import leggauss

    xq = (leggauss(4)[0][1] + 1) / 2 / 8  # fine cell (0, 0), qx = 1, qy = 0
    yq = (leggauss(4)[0][0] + 1) / 2 / 8
    assert np.isclose(arr[0, 0, 1], xq + 10 * yq)
    assert source_input(3.0, mesh, 4, 4, 4) == (0, None, 3.0)


def test_workload_field_is_the_fixture_field():
    g = load("darcy_64x64_r16_p2_lognormal")
    assert digest(lognormal_permeability(1024, 1024, sigma=2.0, ell=0.05, seed=20261203)) == str(g["kappa_sha256"])
    small = load("darcy_4x4_r16_p2_lognormal")
    assert np.array_equal(lognormal_permeability(64, 64, sigma=2.0, ell=0.05, seed=7), small["kappa"])
