"""ctypes binding of ``libmhm_b200.so`` (the C ABI declared in ``include/mhm_b200.h``).

The shared library is the only compute path: there is no CPU fallback.  If
it is missing or no CUDA device is visible, ``lib()`` raises.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libmhm_b200.so"

MHM_OK, MHM_ERR_ARGUMENT, MHM_ERR_LAUNCH, MHM_ERR_UNSUPPORTED = 0, 1, 2, 3
CELL_OK, CELL_KERNEL, CELL_SINGULAR_PIVOT, CELL_RANK_DEFICIENT = 0, 1, 2, 3
CELL_RESIDUAL, CELL_NONFINITE, CELL_ZERO_ROW, CELL_ZERO_COLUMN = 4, 5, 6, 7
CELL_SIZE = 8
CELL_TIMEOUT = 9
SOLVE_OK, SOLVE_NOT_CONVERGED, SOLVE_BREAKDOWN, SOLVE_BARRIER_TIMEOUT, SOLVE_NONFINITE = 0, 1, 2, 3, 4
PRECISION_FP64, PRECISION_MIXED = 0, 1

CALL_ERRORS = {
    MHM_ERR_ARGUMENT: "invalid arguments",
    MHM_ERR_LAUNCH: "CUDA launch failed",
    MHM_ERR_UNSUPPORTED: "problem size is outside the supported on-chip layout",
}

# Per-cell status -> the reference's error wording (linalg/linear.py, execution/cuda.py,
# core/contracts.py) so callers can match the same messages.
CELL_MESSAGES = {
    CELL_KERNEL: "declared kernel is not a left and right nullspace",
    CELL_SINGULAR_PIVOT: "batched LU failed: a local matrix has a singular pivot",
    CELL_RANK_DEFICIENT: "batched local matrix is numerically rank deficient",
    CELL_RESIDUAL: "batched residual criterion failed",
    CELL_NONFINITE: "batched solver returned nonfinite coefficients",
    CELL_ZERO_ROW: "batched matrix contains a zero row",
    CELL_ZERO_COLUMN: "batched matrix contains a zero column",
    CELL_SIZE: "a ragged batch's matrix exceeds the launch's largest order",
    CELL_TIMEOUT: "a local factorization's on-chip copy did not complete within its wait limit",
}

SOLVE_MESSAGES = {
    SOLVE_NOT_CONVERGED: "skeleton CG failed to converge",
    SOLVE_BREAKDOWN: "skeleton CG breakdown: non-positive curvature",
    SOLVE_BARRIER_TIMEOUT: "skeleton CG grid barrier timed out",
    SOLVE_NONFINITE: "skeleton CG produced nonfinite values",
}


class Q1Problem(C.Structure):
    _fields_ = [
        ("macro_nx", C.c_int32), ("macro_ny", C.c_int32), ("rx", C.c_int32), ("ry", C.c_int32),
        ("hx", C.c_double), ("hy", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
        ("tf_h", C.c_int32), ("tf_v", C.c_int32),
        ("coupling_table", C.c_void_p), ("side_sign", C.c_void_p), ("side_orient", C.c_void_p),
        ("kappa_mode", C.c_int32), ("kappa", C.c_void_p), ("kappa_const", C.c_double * 3),
        ("source_mode", C.c_int32), ("source", C.c_void_p), ("source_const", C.c_double),
        ("quad_order", C.c_int32),
        ("pixel_origin", C.c_double * 2), ("pixel_spacing", C.c_double * 2),
        ("pixel_nx", C.c_int32), ("pixel_ny", C.c_int32), ("cut_elements", C.c_void_p),
    ]


class SkeletonSystem(C.Structure):
    _fields_ = [
        ("size", C.c_int64), ("trace_size", C.c_int64),
        ("indptr", C.c_void_p), ("indices", C.c_void_p), ("values", C.c_void_p),
        ("trace_end", C.c_void_p),
        ("faces", C.c_int32), ("face_size", C.c_int32), ("cells", C.c_int32), ("cell_width", C.c_int32),
        ("cell_dofs", C.c_void_p), ("cell_g0", C.c_void_p), ("dof_cells", C.c_void_p),
        ("dof_slot", C.c_void_p), ("nx", C.c_int32), ("ny", C.c_int32),
        ("coarse_ax", C.c_double), ("coarse_ay", C.c_double),
        ("cell_blocks", C.c_void_p), ("block_ld", C.c_int32),
        ("fixed", C.c_void_p), ("coarse_neumann", C.c_int32),
        ("coarse_qx", C.c_void_p), ("coarse_lamx", C.c_void_p), ("coarse_pinv0", C.c_void_p),
        ("coarse_partial", C.c_int32), ("coarse_partial_cells", C.c_void_p), ("coarse_partial_R", C.c_void_p),
    ]


class RaggedMatrix(C.Structure):
    _fields_ = [("mat_off", C.c_int64), ("vec_off", C.c_int64), ("rhs_off", C.c_int64), ("n", C.c_int32),
                ("nrhs", C.c_int32), ("slot", C.c_int32), ("reserved", C.c_int32)]


class GeneralSystem(C.Structure):
    _fields_ = [
        ("size", C.c_int64), ("trace_size", C.c_int64),
        ("indptr", C.c_void_p), ("indices", C.c_void_p), ("values", C.c_void_p),
        ("faces", C.c_int32), ("max_face_size", C.c_int32), ("face_ptr", C.c_void_p),
        ("cells", C.c_int32), ("cell_ptr", C.c_void_p), ("cell_dofs", C.c_void_p), ("cell_g0", C.c_void_p),
        ("dof_cells", C.c_void_p), ("dof_entry", C.c_void_p), ("coarse_inverse", C.c_void_p),
        ("cell_entries", C.c_int64), ("cell_blocks", C.c_void_p), ("block_off", C.c_void_p),
        ("blocks_size", C.c_int64), ("max_cell_dofs", C.c_int32), ("max_trace_row", C.c_int32),
    ]


P = C.c_void_p
_SIGNATURES = {
    "mhm_q1_rhs_width": (C.c_int32, [C.POINTER(Q1Problem)]),
    "mhm_q1_condense_smem_bytes": (C.c_int64, [C.POINTER(Q1Problem), C.c_int32]),
    "mhm_q1_condense": (C.c_int, [C.POINTER(Q1Problem), C.c_int32, C.c_int32, C.c_double, P, P, P, P, P, P, P]),
    "mhm_q1_condense_batch": (C.c_int, [C.c_int32, C.POINTER(Q1Problem), C.c_int32, C.c_int32, C.c_double, P, P, P,
                                        P, P, P, P, P]),
    "mhm_q1_factor_bytes": (C.c_int64, [C.POINTER(Q1Problem), C.c_int32]),
    "mhm_q1_condense_offline": (C.c_int, [C.POINTER(Q1Problem), C.c_int32, C.c_int32, C.c_double, P, P, P, P, P,
                                          P, P, P]),
    "mhm_q1_source_response": (C.c_int, [C.POINTER(Q1Problem), C.c_int32, C.c_int32, C.c_double, P, P, P, P, P,
                                         P, P]),
    "mhm_q1_correction_response": (C.c_int, [C.POINTER(Q1Problem), C.c_int32, C.c_int32, C.c_double, P, P, P,
                                             P, P, P, P]),
    "mhm_q1_original_defect": (C.c_int, [C.POINTER(Q1Problem), P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P]),
    "mhm_refine_norms": (C.c_int, [C.c_int32, P, C.c_int64, P, P, P, C.c_int64, P, P, P, P, P, P, P]),
    "mhm_vector_accumulate": (C.c_int, [C.c_int64, P, P, P]),
    "mhm_vector_accumulate_dd": (C.c_int, [C.c_int64, P, P, P, P]),
    "mhm_q1_original_defect_dd": (C.c_int, [C.POINTER(Q1Problem), P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P,
                                            P, P]),
    "mhm_q1_mean_gauge": (C.c_int, [C.POINTER(Q1Problem), P, P, C.c_double, C.c_int64, P, P, P]),
    "mhm_skeleton_fixed_rhs": (C.c_int, [C.c_int64, C.c_int64, P, P, P, P, P, P, P, P]),
    "mhm_q1_flux": (C.c_int, [C.POINTER(Q1Problem), P, P, P]),
    "mhm_skeleton_scatter": (C.c_int, [C.c_int64, P, P, P, P, C.c_int64, C.c_int64, P, P, P, P, P, P, P]),
    "mhm_skeleton_export_csc": (C.c_int, [C.c_int64, P, P, P, P, P, P, P, P]),
    "mhm_skeleton_workspace_bytes": (C.c_int64, [C.POINTER(SkeletonSystem), C.c_int32]),
    "mhm_skeleton_solve": (C.c_int, [C.POINTER(SkeletonSystem), P, P, P, C.c_double, C.c_double, C.c_int32,
                                     C.c_int32, C.c_int32, P, C.c_int64, P, P, P]),
    "mhm_skeleton_solve_static": (C.c_int, [C.POINTER(SkeletonSystem), P, P, P, C.c_double, C.c_double,
                                            C.c_int32, C.c_int32, C.c_int32, P, P, P]),
    "mhm_general_workspace_bytes": (C.c_int64, [C.POINTER(GeneralSystem)]),
    "mhm_general_solve": (C.c_int, [C.POINTER(GeneralSystem), P, P, P, C.c_int64, C.c_double, C.c_double,
                                    C.c_int32, C.c_int32, P, P, P]),
    "mhm_tet_kappa": (C.c_int, [C.c_int64, P, C.c_int32, C.c_int32, P, C.c_int32, P, P, C.c_int32, C.c_int32,
                                C.c_int32, P, P, P]),
    "mhm_dense_systems": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, P, P,
                                    P, P, P, P, P, P, P, P]),
    "mhm_dense_contributions": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P,
                                          P, P, P, P, P, P, P, P, P, P]),
    "mhm_dense_reconstruct": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, P, P, P, P, P, P, C.c_int64, P, P, P,
                                        P]),
    "mhm_p2_element_bytes": (C.c_int64, [C.c_int64]),
    "mhm_p2_assemble": (C.c_int, [C.c_int64, P, P, C.c_int32, P, P, C.c_int32, P, P, P, P, C.c_double, C.c_double,
                                  C.c_double, P, C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P]),
    "mhm_q1_reconstruct": (C.c_int, [C.POINTER(Q1Problem), P, P, C.c_int64, P, P, P, P]),
    "mhm_batched_factor": (C.c_int, [C.c_int64, C.c_int32, P, P, P, P, P, P, P]),
    "mhm_batched_factor_ragged": (C.c_int, [C.c_int64, P, C.c_int32, P, P, P, P, P, P, P]),
    "mhm_batched_solve_ragged": (C.c_int, [C.c_int64, P, C.c_int32, C.c_int32, P, P, P, P, P, P, P, C.c_double,
                                           C.c_double, C.c_int32, P, P]),
    "mhm_batched_factor_large": (C.c_int, [C.c_int64, P, C.c_int32, P, P, P, P, P, P, P]),
    "mhm_rt0_elements": (C.c_int, [C.c_int64, P, P, P, C.c_int32, P, P, C.c_int32, P, P, P, P, C.c_double,
                                   C.c_double, C.c_double, P, P]),
    "mhm_mixed_systems": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P, P, P, P,
                                    P, P, P, P, P]),
    "mhm_mixed_contributions": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P,
                                          P, P, P, P, P, P, P, P, P, P]),
    "mhm_mixed_reconstruct": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, P, P, P, P, P, P, C.c_int64, P, P, P, P,
                                        P]),
    "mhm_dense_systems_ragged": (C.c_int, [C.c_int64, P, P, P, C.c_int32, P, P, P, P, P, P, P, P, P, P, P, P]),
    "mhm_batched_solve_large": (C.c_int, [C.c_int64, P, C.c_int32, C.c_int32, P, P, P, P, P, P, P, P, C.c_double,
                                          C.c_double, C.c_int32, P, P]),
    "mhm_p2_elements": (C.c_int, [C.c_int64, P, P, C.c_int32, P, P, C.c_int32, P, P, P, P, C.c_double, C.c_double,
                                  C.c_double, P, P]),
    "mhm_p2_assemble_rows": (C.c_int, [C.c_int64, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "mhm_batched_solve": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, P, P, P, P, P, P, P, P, C.c_double,
                                    C.c_double, C.c_int32, P, P]),
    "mhm_p1_batch_assemble": (C.c_int, [C.c_int64, C.c_int32, C.c_int32, P, C.c_int32, P, P, C.c_int64,
                                        C.c_int64, P, C.c_int64, C.c_int64, P, P, P, P, P, P, P, P]),
    "mhm_p1_batch_scratch_bytes": (C.c_int64, [C.c_int64, C.c_int32, C.c_int32]),
    "mhm_version": (C.c_char_p, []),
}

_LOCK = threading.Lock()
_LIB: C.CDLL | None = None


def load() -> C.CDLL:
    """Load the library and bind every declared symbol (no GPU needed)."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            if not LIBRARY.exists():
                raise RuntimeError(f"{LIBRARY.name} is not built; run `python -m pymhm_b200.build`")
            lib = C.CDLL(str(LIBRARY))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = lib
    return _LIB


def lib() -> C.CDLL:
    """The library, after checking that a CUDA device is usable."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("pymhm_b200 requires a CUDA device (no CPU fallback)")
    return load()


def check(rc: int, what: str) -> None:
    if rc != MHM_OK:
        raise RuntimeError(f"{what}: {CALL_ERRORS.get(rc, rc)}")


def ptr(t) -> int:
    """Device pointer of a torch tensor (None -> NULL).  The kernels index dense
    row-major arrays, so a tensor whose strides are not row-major is refused."""
    if t is None:
        return 0
    if not t.is_contiguous():
        raise ValueError("device arrays passed to the library must be contiguous (row-major)")
    return int(t.data_ptr())


def stream_handle(stream) -> int:
    import torch

    s = torch.cuda.current_stream() if stream is None else stream
    return int(s.cuda_stream)


def declared_symbols() -> list[str]:
    return list(_SIGNATURES)
