"""Cartesian Q1 Primal-MHM Darcy solve on one B200: the host side of the hot path.

``solve_darcy_quadrilateral`` mirrors PyMHM's driver of the same name
(``src/pymhm/_legacy/models/darcy/cartesian.py:86-168``) for degree-one local
spaces and weak Dirichlet data; ``CartesianQ1Plan`` is the reusable,
device-resident form used for repeated solves and serving.

Per solve, four kernels run back to back on one stream:

1. ``mhm_q1_condense``   one CTA per macrocell: Q1 assembly from the fine-cell
   coefficients, pinned band LDL^T of the Neumann operator, FP64-refined
   augmented responses ``[R f | R B | R A1]``, Schur block and reduced load;
2. ``mhm_skeleton_scatter``  deterministic ordered reduction into the
   precomputed skeleton CSR (no atomics);
3. ``mhm_skeleton_solve``  persistent projected PCG with an outer FP64
   defect correction on the assembled skeleton matrix;
4. ``mhm_q1_reconstruct``  fields ``u_K = R f - (R B) lambda_K + E c_K`` and
   fine-cell-centre fluxes ``-K grad u``.
"""

from __future__ import annotations

import math
import numbers
import time
from dataclasses import dataclass, field

import numpy as np
from numpy.polynomial.legendre import leggauss

from . import _lib
from .errors import LinearSolveError
from .skeleton import attach_fixed
from .topology import (
    CartesianMacroMesh,
    FaceSpace,
    SkeletonSpace,
    boundary_data,
    coarse_coefficients,
    coupling_tables,
    dof_cell_maps,
    fixed_coarse_data,
    geometric_constraint,
    mesh_arrays,
    neumann_fixed,
    neumann_layout,
    side_orientation,
    skeleton_pattern,
    transpose_slots,
)

PRECISIONS = {"fp64": _lib.PRECISION_FP64, "mixed": _lib.PRECISION_MIXED}


def _refinement(value) -> tuple[int, int]:
    if isinstance(value, tuple):
        if len(value) != 2:
            raise ValueError("local_refinement requires two integers")
        rx, ry = (int(v) for v in value)
    else:
        rx = ry = int(value)
    if rx < 1 or ry < 1:
        raise ValueError("local_refinement must be positive")
    return rx, ry


def _is_number(value) -> bool:
    if isinstance(value, (bool, np.bool_)):
        return False
    if isinstance(value, numbers.Real):
        return True
    return isinstance(value, np.ndarray) and value.ndim == 0 and value.dtype.kind in "iuf"


def fine_grid(mesh: CartesianMacroMesh, rx: int, ry: int):
    """Fine spacing, counts and the lower-left corner of the global fine grid."""
    hx, hy = mesh.spacing
    return hx / rx, hy / ry, mesh.nx * rx, mesh.ny * ry, mesh.bounds[0], mesh.bounds[2]


def _quad_points(mesh, rx, ry, order):
    fhx, fhy, nxf, nyf, x0, y0 = fine_grid(mesh, rx, ry)
    g, _ = leggauss(order)
    g = (g + 1) / 2
    gx = x0 + (np.arange(nxf)[:, None] + g[None, :]) * fhx  # (nxf, q)
    gy = y0 + (np.arange(nyf)[:, None] + g[None, :]) * fhy
    # [gx][gy][qy][qx]
    px = np.broadcast_to(gx[:, None, None, :], (nxf, nyf, order, order))
    py = np.broadcast_to(gy[None, :, :, None], (nxf, nyf, order, order))
    return np.stack((px, py), axis=-1).reshape(-1, 2)


def _fine_centres(mesh, rx, ry):
    fhx, fhy, nxf, nyf, x0, y0 = fine_grid(mesh, rx, ry)
    cx = x0 + (np.arange(nxf) + 0.5) * fhx
    cy = y0 + (np.arange(nyf) + 0.5) * fhy
    return np.stack(np.meshgrid(cx, cy, indexing="ij"), axis=-1).reshape(-1, 2)


def _tensor_components(values: np.ndarray) -> tuple[int, np.ndarray]:
    """(mode, array) for scalar (mode 1) or 2x2 SPD tensor (mode 2) fine-cell values."""
    values = np.asarray(values, dtype=float)
    if values.ndim == 2:
        if not np.all(np.isfinite(values)) or np.any(values <= 0):
            raise ValueError("diffusion tensor must be finite, symmetric and positive definite")
        return 1, np.ascontiguousarray(values)
    if values.ndim == 4 and values.shape[2:] == (2, 2):
        if not np.allclose(values, values.swapaxes(2, 3), rtol=1e-12, atol=1e-14):
            raise ValueError("diffusion tensor must be finite, symmetric and positive definite")
        comp = np.stack((values[..., 0, 0], values[..., 0, 1], values[..., 1, 1]), axis=-1)
        det = comp[..., 0] * comp[..., 2] - comp[..., 1] ** 2
        if not np.all(np.isfinite(comp)) or np.any(comp[..., 0] <= 0) or np.any(det <= 0):
            raise ValueError("diffusion tensor must be finite, symmetric and positive definite")
        return 2, np.ascontiguousarray(comp)
    raise ValueError("fine-cell permeability must have shape (nx, ny) or (nx, ny, 2, 2)")


def _pixel_origin(field) -> np.ndarray:
    origin = getattr(field, "origin", None)
    return np.zeros(2) if origin is None else np.asarray(origin, dtype=float)


def grid_resolves_material(field, mesh: CartesianMacroMesh, rx: int, ry: int) -> bool:
    """Every pixel line of ``field`` lies on a fine-grid line (``grid_resolves_material``,
    ``quadrilateral.py:116-132``): the pixel spacing is a whole number of fine cells and
    the pixel origin sits a whole number of fine cells from the domain corner, each to
    64 eps of the compared value."""
    fhx, fhy, _, _, x0, y0 = fine_grid(mesh, rx, ry)
    spacing = np.asarray(field.spacing, dtype=float)
    if spacing.shape != (2,):
        raise ValueError("quadrilateral material integration requires a two-dimensional field")
    fine = np.array([fhx, fhy])
    values = np.r_[spacing / fine, (np.array([x0, y0]) - _pixel_origin(field)) / fine]
    tolerance = 64 * np.finfo(float).eps * max(1.0, float(np.max(np.abs(values))))
    return bool(np.all(np.abs(values - np.rint(values)) <= tolerance))


def pixel_geometry(field, mesh: CartesianMacroMesh, rx: int, ry: int):
    """(origin, spacing, counts) of a pixel field whose lines cut the fine cells, after
    the reference's coverage check (``quadrilateral.py:149-158``)."""
    fhx, fhy, nxf, nyf, x0, y0 = fine_grid(mesh, rx, ry)
    origin, spacing = _pixel_origin(field), np.asarray(field.spacing, dtype=float)
    if not (np.all(np.isfinite(origin)) and np.all(np.isfinite(spacing)) and np.all(spacing > 0)):
        raise ValueError("material field spacing must be positive and its origin finite")
    shape = np.asarray(np.shape(field.values)[:2])
    lower = (np.array([x0, y0]) - origin) / spacing
    upper = (np.array([x0 + nxf * fhx, y0 + nyf * fhy]) - origin) / spacing
    tolerance = 64 * np.finfo(float).eps * shape
    if np.any(lower < -tolerance) or np.any(upper > shape + tolerance):
        raise ValueError("a fine rectangle lies outside the Cartesian material field")
    return (float(origin[0]), float(origin[1])), (float(spacing[0]), float(spacing[1])), (int(shape[0]), int(shape[1]))


def permeability_input(permeability, mesh: CartesianMacroMesh, rx: int, ry: int, order: int):
    """Map a permeability description to (mode, array | None, constant triple).

    Accepted: a positive scalar or constant 2x2 tensor; a pixel field with
    ``values``, ``spacing`` and ``origin`` (``materials/cartesian.py``); an array of
    fine-cell values; or a callable that is constant on every fine cell at the Gauss
    points.  A pixel field whose lines coincide with fine-grid lines is sampled per
    fine cell (modes 1/2); one whose lines cut the fine cells is passed as pixels
    (modes 3/4, geometry from ``pixel_geometry``) and integrated on each fine cell's
    exact pixel intersections, as ``quadrilateral.py:136-188, 215-234`` does.
    """
    _, _, nxf, nyf, _, _ = fine_grid(mesh, rx, ry)
    if _is_number(permeability):
        k = float(permeability)
        if not (np.isfinite(k) and k > 0):
            raise ValueError("diffusion tensor must be finite, symmetric and positive definite")
        return 0, None, (k, 0.0, k)
    arr = None if callable(permeability) or hasattr(permeability, "spacing") else np.asarray(permeability)
    if arr is not None and arr.shape == (2, 2):
        mode, comp = _tensor_components(arr.reshape(1, 1, 2, 2))
        return 0, None, tuple(float(v) for v in comp.reshape(3))
    if arr is not None:
        if arr.shape[:2] != (nxf, nyf):
            raise ValueError(f"fine-cell permeability must have leading shape ({nxf}, {nyf})")
        mode, comp = _tensor_components(arr)
        return mode, comp, (0.0, 0.0, 0.0)
    if hasattr(permeability, "spacing") and hasattr(permeability, "values"):
        spacing = np.asarray(permeability.spacing, dtype=float)
        origin = _pixel_origin(permeability)
        vals = np.asarray(permeability.values, dtype=float)
        if not grid_resolves_material(permeability, mesh, rx, ry):
            pixel_geometry(permeability, mesh, rx, ry)  # coverage
            mode, comp = _tensor_components(vals)
            return mode + 2, comp, (0.0, 0.0, 0.0)
        centres = _fine_centres(mesh, rx, ry)
        idx = np.floor((centres - origin) / spacing).astype(np.int64)
        shape = np.array(vals.shape[:2])
        if np.any(idx < 0) or np.any(idx >= shape):
            raise ValueError("a fine rectangle lies outside the Cartesian material field")
        sampled = vals[idx[:, 0], idx[:, 1]]
        sampled = sampled.reshape(nxf, nyf, *vals.shape[2:])
        mode, comp = _tensor_components(sampled)
        return mode, comp, (0.0, 0.0, 0.0)
    if callable(permeability):
        # at the Gauss points of every fine cell: one value per cell if it is constant
        # there (modes 1/2), else every point plus the centre for the flux (modes 5/6)
        pts = _quad_points(mesh, rx, ry, order)
        raw = np.asarray(permeability(pts), dtype=float)
        q = order * order
        if raw.shape == (len(pts),):
            per = raw.reshape(nxf, nyf, q)
            if np.all(per == per[..., :1]):
                mode, comp = _tensor_components(per[..., 0])
                return mode, comp, (0.0, 0.0, 0.0)
            centre = np.asarray(permeability(_fine_centres(mesh, rx, ry)), dtype=float).reshape(nxf, nyf, 1)
            full = np.concatenate((per, centre), axis=2)
            mode, comp = _tensor_components(full.reshape(nxf, nyf * (q + 1)))
            return 5, comp.reshape(nxf, nyf, q + 1), (0.0, 0.0, 0.0)
        if raw.shape == (len(pts), 2, 2):
            per = raw.reshape(nxf, nyf, q, 2, 2)
            if np.all(per == per[:, :, :1]):
                mode, comp = _tensor_components(per[:, :, 0])
                return mode, comp, (0.0, 0.0, 0.0)
            centre = np.asarray(permeability(_fine_centres(mesh, rx, ry)), dtype=float).reshape(nxf, nyf, 1, 2, 2)
            full = np.concatenate((per, centre), axis=2)
            mode, comp = _tensor_components(full.reshape(nxf, nyf * (q + 1), 2, 2))
            return 6, comp.reshape(nxf, nyf, q + 1, 3), (0.0, 0.0, 0.0)
        raise ValueError("permeability callable must return scalars or 2x2 tensors per point")
    raise TypeError("unsupported permeability description")


def _cut_source_check(smode: int) -> None:
    """With pixel lines cutting the fine cells the reference integrates the load on the
    cut rule too; a pointwise source is sampled here on the fine cells' own Gauss
    points, which is a different quadrature unless the source is constant per cell."""
    if smode == 2:
        raise NotImplementedError("a pointwise source with a cut material field needs the cut load quadrature; "
                                  "pass a constant or per-fine-cell source")


def source_input(source, mesh: CartesianMacroMesh, rx: int, ry: int, order: int):
    """(mode, array | None, constant) for a scalar, fine-cell array or pointwise callable."""
    _, _, nxf, nyf, _, _ = fine_grid(mesh, rx, ry)
    if _is_number(source):
        return 0, None, float(source)
    if callable(source):
        pts = _quad_points(mesh, rx, ry, order)
        vals = np.broadcast_to(np.asarray(source(pts), dtype=float), (len(pts),))
        if not np.all(np.isfinite(vals)):
            raise ValueError("scalar coefficient must be finite")
        return 2, np.ascontiguousarray(vals.reshape(nxf, nyf, order * order)), 0.0
    arr = np.asarray(source, dtype=float)
    if arr.shape != (nxf, nyf):
        raise ValueError(f"fine-cell source must have shape ({nxf}, {nyf})")
    return 1, np.ascontiguousarray(arr), 0.0


@dataclass
class Q1Solution:
    """Host copy of one solve (``HybridSolution`` + ``QuadrilateralDarcySolution`` fields)."""

    trace: np.ndarray
    coarse: np.ndarray
    fields: np.ndarray
    flux: np.ndarray
    residual: float
    raw_residual: float
    corrected: np.ndarray
    local_iterations: np.ndarray
    global_iterations: int
    outer_corrections: int
    seconds: float = 0.0
    extra: dict = field(default_factory=dict)


@dataclass(frozen=True)
class HybridRefinement:
    """Corrected solution and original-equation residual history (``HybridRefinement``,
    ``core/refinement.py:30-47``).

    ``residual_norms`` holds the residual of the uncondensed local equations and the
    weak trace equations before the first and after every accepted correction;
    ``rhs_norm`` is the norm of their right-hand side (local loads and boundary
    data).  ``solution.residual`` is the reduced residual of the corrected fields.
    """

    solution: Q1Solution
    residual_norms: tuple
    rhs_norm: float


def _refinement_steps(steps) -> None:
    """``_refinement_steps`` (``linalg/linear.py:84-87``)."""
    if isinstance(steps, (bool, np.bool_)) or not isinstance(steps, (int, np.integer)) or steps < 0:
        raise ValueError("refinement_steps must be a nonnegative integer")


def _step_limits(max_steps, min_steps) -> None:
    """``_step_limits`` (``core/refinement.py:343-348``)."""
    _refinement_steps(max_steps)
    _refinement_steps(min_steps)
    if min_steps > max_steps:
        raise ValueError("min_steps must not exceed max_steps")


def _tolerances(rtol, atol) -> None:
    """``_tolerances`` (``linalg/linear.py:76-81``)."""
    if not np.isfinite(rtol) or not np.isfinite(atol) or min(rtol, atol) < 0:
        raise ValueError("rtol and atol must be finite and nonnegative")
    if rtol == 0 and atol == 0:
        raise ValueError("at least one tolerance must be positive")


class CartesianQ1Plan:
    """Device-resident plan: topology, tables, pattern and buffers for one problem shape.

    The plan owns every device buffer the four kernels use, so repeated solves
    (new coefficients or sources on the same mesh) allocate nothing.
    """

    def __init__(self, mesh, skeleton=None, local_refinement=4, *, dirichlet=0.0, neumann=None, mean_pressure=0.0,
                 quadrature_order=4, degree=1, precision="fp64", device=None, max_refine=None, local_tol=1e-12,
                 global_rtol=1e-13, inner_rtol=1e-10, max_inner=5000, max_outer=6, grid=0):
        import torch

        if int(degree) != 1:
            raise NotImplementedError("the GPU path implements degree-one (Q1) local spaces")
        if precision not in PRECISIONS:
            raise ValueError("precision must be 'fp64' or 'mixed'")
        self.torch = torch
        self.mesh = mesh_arrays(mesh)
        self.skeleton = SkeletonSpace(self.mesh) if skeleton is None else SkeletonSpace.of(skeleton, self.mesh)
        self.rx, self.ry = _refinement(local_refinement)
        self.order = max(int(quadrature_order), 2)
        self.precision = precision
        self.device = torch.device("cuda" if device is None else device)
        self.max_refine = int(max_refine or (10 if precision == "fp64" else 30))
        self.local_tol = float(local_tol)
        self.global_rtol, self.inner_rtol = float(global_rtol), float(inner_rtol)
        self.max_inner, self.max_outer, self.grid = int(max_inner), int(max_outer), int(grid)
        self.lib = _lib.lib()
        m, sk = self.mesh, self.skeleton
        space_h, space_v = sk.uniform_by_orientation()
        fs = space_h.size
        if space_v.size != fs:
            raise NotImplementedError("the GPU skeleton solver requires equal face sizes")
        self.cells = len(m.cells)
        self.n = (self.rx + 1) * (self.ry + 1)
        self.t = 2 * (space_h.size + space_v.size)
        self.w = self.t + 2
        self.T = sk.size
        self.N = self.T + self.cells
        self.nfine = self.rx * self.ry
        # ---- host tables --------------------------------------------------------------
        hx, hy = m.spacing
        self.table_h = coupling_tables(space_h, space_v, self.rx, self.ry, hx, hy)
        self.cell_dofs_h = sk.cell_dof_array
        self.pattern = skeleton_pattern(self.cell_dofs_h, self.T)
        dof_cells, dof_slot = dof_cell_maps(self.cell_dofs_h, self.T)
        g0 = geometric_constraint(m, space_h, space_v)
        # Neumann faces: their trace DOFs are prescribed
        # (boundary_data's `fixed`) and eliminated from the global solve
        self.neumann_bits, neumann_partial = neumann_layout(m, neumann)
        self.boundary_h = boundary_data(sk, dirichlet, self.order, neumann)
        fixed_dofs, fixed_values = neumann_fixed(sk, neumann, self.order)
        # ---- device constants ---------------------------------------------------------
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)

        def up(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(dev)

        self.d_table = up(self.table_h, torch.float64)
        self.d_sign = up(m.signs.astype(np.int8), torch.int8)
        self.d_orient = up(side_orientation(m), torch.int8)
        self.d_cell_dofs = up(self.cell_dofs_h, torch.int64)
        p = self.pattern
        self.d_indptr = up(p.indptr, torch.int64)
        self.d_indices = up(p.indices, torch.int32)
        self.d_slot_ptr = up(p.slot_ptr, torch.int64)
        self.d_contrib = up(p.contrib, torch.int64)
        self.d_load_ptr = up(p.load_ptr, torch.int64)
        self.d_load_contrib = up(p.load_contrib, torch.int64)
        self.d_trace_end = up(p.trace_end, torch.int64)
        self.d_boundary = up(self.boundary_h, torch.float64)
        self.d_g0 = up(g0, torch.float64)
        self.d_dof_cells = up(dof_cells, torch.int32)
        self.d_dof_slot = up(dof_slot, torch.int32)
        self.coarse_ab = coarse_coefficients(m, space_h, space_v)
        # ---- device buffers -----------------------------------------------------------
        M, n, w, t1 = self.cells, self.n, self.w, self.t + 1
        self.solution = torch.empty((M, w, n + 1), **f64)
        self.blocks = torch.empty((M, t1, t1), **f64)
        self.loads = torch.empty((M, t1), **f64)
        self.corrected = torch.empty(M, dtype=torch.uint8, device=dev)
        self.cell_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.cell_iters = torch.empty(M, dtype=torch.int32, device=dev)
        self.values = torch.empty(len(p.indices), **f64)
        self.rhs = torch.empty(self.N, **f64)
        self.load_scale = torch.empty(self.N, **f64)
        self.x = torch.empty(self.N, **f64)
        self.info = torch.zeros(4, dtype=torch.int32, device=dev)
        self.stats = torch.zeros(4, **f64)
        self.fields = torch.empty((M, n), **f64)
        self.flux = torch.empty((M, self.nfine, 2), **f64)
        self.kappa = None
        self.source = None
        # structures
        fhx, fhy, self.nxf, self.nyf, x0, y0 = fine_grid(m, self.rx, self.ry)
        self.q1 = _lib.Q1Problem()
        q = self.q1
        q.macro_nx, q.macro_ny, q.rx, q.ry = m.nx, m.ny, self.rx, self.ry
        q.hx, q.hy, q.x0, q.y0 = fhx, fhy, x0, y0
        q.tf_h, q.tf_v = space_h.size, space_v.size
        q.coupling_table = _lib.ptr(self.d_table)
        q.side_sign = _lib.ptr(self.d_sign)
        q.side_orient = _lib.ptr(self.d_orient)
        q.quad_order = self.order
        if self.lib.mhm_q1_condense_smem_bytes(q, PRECISIONS[precision]) <= 0:
            raise NotImplementedError("local refinement too large for the on-chip factor layout")
        self.sys = _lib.SkeletonSystem()
        s = self.sys
        s.size, s.trace_size = self.N, self.T
        s.indptr, s.indices, s.values = _lib.ptr(self.d_indptr), _lib.ptr(self.d_indices), _lib.ptr(self.values)
        s.trace_end = _lib.ptr(self.d_trace_end)
        s.faces, s.face_size, s.cells, s.cell_width = len(m.faces), fs, M, self.t
        s.cell_dofs, s.cell_g0 = _lib.ptr(self.d_cell_dofs), _lib.ptr(self.d_g0)
        s.dof_cells, s.dof_slot = _lib.ptr(self.d_dof_cells), _lib.ptr(self.d_dof_slot)
        s.nx, s.ny = m.nx, m.ny
        s.coarse_ax, s.coarse_ay = self.coarse_ab
        s.cell_blocks, s.block_ld = _lib.ptr(self.blocks), self.t + 1
        self.d_fixed = self.d_xfixed = None
        if neumann:  # any Neumann face, on whole sides or on parts of them
            self._fixed_keep = attach_fixed(s, fixed_coarse_data(m, sk, neumann, *self.coarse_ab), up)
            self.d_fixed = self._fixed_keep["mask"]
            xfixed = np.zeros(self.N)
            xfixed[fixed_dofs] = fixed_values
            self.d_xfixed = up(xfixed, torch.float64)
            self.rhs_red = torch.empty(self.N, dtype=torch.float64, device=dev)
        # pure Neumann: the mean-pressure condition sum_cells C . u = mean_pressure |domain|
        # fixes the constant coarse mode (cartesian.py:136-142)
        self.pure_neumann = self.neumann_bits == 15 and not neumann_partial
        if self.pure_neumann:
            x0, x1, y0, y1 = m.bounds
            self.mean_value = float(mean_pressure) * (x1 - x0) * (y1 - y0)
            if not np.isfinite(self.mean_value):
                raise ValueError("mean_pressure must be finite")
            self.gauge = torch.empty(2 * self.cells + 1, dtype=torch.float64, device=dev)
        nbytes = self.lib.mhm_skeleton_workspace_bytes(s, self.grid)
        if nbytes <= 0:
            raise RuntimeError("could not size the skeleton solver workspace")
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)

    # ------------------------------------------------------------------------------------
    def set_coefficients(self, permeability=1.0, source=0.0, *, non_blocking=False):
        """Upload (or keep constant) coefficient data for the next ``launch``."""
        torch = self.torch
        kmode, karr, kconst = permeability_input(permeability, self.mesh, self.rx, self.ry, self.order)
        smode, sarr, sconst = source_input(source, self.mesh, self.rx, self.ry, self.order)
        pixels = pixel_geometry(permeability, self.mesh, self.rx, self.ry) if kmode in (3, 4) else None
        self.kappa = None if karr is None else torch.as_tensor(np.array(karr)).to(self.device, non_blocking=non_blocking)
        self.source = None if sarr is None else torch.as_tensor(np.array(sarr)).to(self.device, non_blocking=non_blocking)
        self.set_device_coefficients(kmode, self.kappa, kconst, smode, self.source, sconst, pixels=pixels)

    def set_device_coefficients(self, kmode, kappa, kconst, smode, source, sconst, *, pixels=None):
        """Point the plan at device-resident coefficient tensors (no copies).

        ``pixels`` = (origin, spacing, counts) is required for the cut-cell modes 3/4,
        where ``kappa`` holds pixel values [px][py][comp]; modes 5/6 hold the values at
        the fine cells' Gauss points and centres [gx][gy][Q*Q + 1][comp]."""
        q = self.q1
        if kmode in (3, 4):
            if pixels is None:
                raise ValueError("kappa modes 3 and 4 need the pixel geometry")
            _cut_source_check(smode)
            (q.pixel_origin[0], q.pixel_origin[1]), (q.pixel_spacing[0], q.pixel_spacing[1]), \
                (q.pixel_nx, q.pixel_ny) = pixels
        if kmode >= 3:  # element matrices from a pre-pass
            if getattr(self, "cut_elements", None) is None:
                self.cut_elements = self.torch.empty(10 * self.nxf * self.nyf, dtype=self.torch.float64,
                                                     device=self.device)
            q.cut_elements = _lib.ptr(self.cut_elements)
        q.kappa_mode, q.kappa = kmode, _lib.ptr(kappa)
        q.kappa_const[0], q.kappa_const[1], q.kappa_const[2] = kconst
        q.source_mode, q.source, q.source_const = smode, _lib.ptr(source), float(sconst)
        self._keep = (kappa, source)
        self._factors_current = False  # factors kept by prepare_offline belong to the old permeability

    def launch(self, stream=None, *, reconstruct=True, events=None, global_stream=None, local="condense"):
        """Enqueue the four kernels on ``stream`` (no host synchronisation).

        ``events``, if given, is a list of at least five ``torch.cuda.Event``s
        recorded before, between and after the kernels (per-kernel timing).
        ``global_stream``, if given, runs the skeleton solve and the reconstruction
        after the local stage on that stream instead (ordered by an event), so that
        a serving loop can put the latency-bound global solve on a higher-priority
        stream and overlap it with the next request's local stage.
        ``local`` selects the local stage: ``"condense"``; ``"offline"`` (condense and
        keep each cell's factor, see ``prepare_offline``); ``"online"`` (source
        response only with the kept factors; Schur blocks and the skeleton matrix
        are reused, only the right-hand side is reduced); ``"batched"`` (the local
        stage was enqueued on ``stream`` by ``condense_batch`` together with other
        plans': the launch starts at the reduction).
        """
        L, s = self.lib, _lib.stream_handle(stream)
        P = _lib.ptr
        torch = self.torch
        cur = torch.cuda.current_stream() if stream is None else stream
        gcur = cur if global_stream is None else global_stream
        gs = s if global_stream is None else _lib.stream_handle(global_stream)
        if getattr(self, "_done", None) is not None and self._done_stream is not cur:
            cur.wait_event(self._done)  # the previous solve's global stage still reads the buffers

        def mark(k, st):
            if events is not None:
                events[k].record(st)

        mark(0, cur)
        prec = PRECISIONS[self.precision]
        if local == "condense":
            _lib.check(L.mhm_q1_condense(self.q1, prec, self.max_refine, self.local_tol, P(self.solution),
                                         P(self.blocks), P(self.loads), P(self.corrected), P(self.cell_status),
                                         P(self.cell_iters), s), "mhm_q1_condense")
        elif local == "offline":
            if getattr(self, "factors", None) is None:
                nbytes = int(L.mhm_q1_factor_bytes(self.q1, prec))
                if nbytes <= 0:
                    raise RuntimeError("could not size the factor store")
                self.factors = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            _lib.check(L.mhm_q1_condense_offline(self.q1, prec, self.max_refine, self.local_tol, P(self.solution),
                                                 P(self.blocks), P(self.loads), P(self.corrected),
                                                 P(self.cell_status), P(self.cell_iters), P(self.factors), s),
                       "mhm_q1_condense_offline")
            self._factors_current = True
        elif local == "online":
            if getattr(self, "factors", None) is None:
                raise RuntimeError("prepare_offline() must run before online source responses")
            if not getattr(self, "_factors_current", False):
                raise RuntimeError("the permeability changed since prepare_offline(): the kept factors are stale")
            _lib.check(L.mhm_q1_source_response(self.q1, prec, self.max_refine, self.local_tol, P(self.factors),
                                                P(self.solution), P(self.loads), P(self.corrected),
                                                P(self.cell_status), P(self.cell_iters), s),
                       "mhm_q1_source_response")
        elif local != "batched":
            raise ValueError("local must be 'condense', 'offline', 'online' or 'batched'")
        mark(1, cur)
        pat = self.pattern
        # online: the skeleton matrix is unchanged, only the right-hand side is reduced
        _lib.check(L.mhm_skeleton_scatter(0 if local == "online" else len(pat.indices), P(self.d_slot_ptr),
                                          P(self.d_contrib),
                                          P(self.blocks), P(self.values), self.N, self.T,
                                          P(self.d_load_ptr), P(self.d_load_contrib), P(self.loads),
                                          P(self.d_boundary), P(self.rhs), P(self.load_scale), s),
                   "mhm_skeleton_scatter")
        if self.d_fixed is not None:  # the global solve sees the reduced right-hand side
            _lib.check(L.mhm_skeleton_fixed_rhs(self.N, self.T, P(self.d_indptr), P(self.d_indices), P(self.values),
                                                P(self.d_fixed), P(self.d_xfixed), P(self.rhs), P(self.rhs_red), s),
                       "mhm_skeleton_fixed_rhs")
        mark(2, cur)
        if global_stream is not None:
            if not hasattr(self, "_handoff"):
                self._handoff = torch.cuda.Event()
            self._handoff.record(cur)
            global_stream.wait_event(self._handoff)
        _lib.check(L.mhm_skeleton_solve(self.sys, P(self.rhs if self.d_fixed is None else self.rhs_red),
                                        P(self.load_scale), P(self.x), self.global_rtol,
                                        self.inner_rtol, self.max_inner, self.max_outer, self.grid,
                                        P(self.workspace), self.workspace.numel(), P(self.info), P(self.stats), gs),
                   "mhm_skeleton_solve")
        if self.d_xfixed is not None:  # the prescribed Neumann coefficients
            _lib.check(L.mhm_vector_accumulate(self.N, P(self.x), P(self.d_xfixed), gs), "mhm_vector_accumulate")
        mark(3, gcur)
        if self.pure_neumann:  # fields of the gauge-free solve, then the mean-pressure shift
            _lib.check(L.mhm_q1_reconstruct(self.q1, P(self.solution), P(self.d_cell_dofs), self.T, P(self.x),
                                            P(self.fields), None, gs), "mhm_q1_reconstruct")
            _lib.check(L.mhm_q1_mean_gauge(self.q1, P(self.solution), P(self.fields), self.mean_value, self.T,
                                           P(self.x), P(self.gauge), gs), "mhm_q1_mean_gauge")
        if reconstruct:
            _lib.check(L.mhm_q1_reconstruct(self.q1, P(self.solution), P(self.d_cell_dofs), self.T, P(self.x),
                                            P(self.fields), P(self.flux), gs), "mhm_q1_reconstruct")
        mark(4, gcur)
        if global_stream is not None:
            if getattr(self, "_done", None) is None:
                self._done = torch.cuda.Event()
            self._done.record(gcur)
            self._done_stream = gcur
        else:
            self._done = None

    def check(self):
        """Synchronise and raise the reference's error for any failed cell or solve."""
        torch = self.torch
        status = self.cell_status.cpu().numpy()
        bad = np.flatnonzero(status)
        if len(bad):
            code = int(status[bad[0]])
            msg = _lib.CELL_MESSAGES.get(code, f"status {code}")
            if code == _lib.CELL_KERNEL:
                raise ValueError(msg)
            raise LinearSolveError(f"{msg} (macrocell {int(bad[0])}, {len(bad)} cells)")
        info = self.info.cpu().numpy()
        if info[0] != _lib.SOLVE_OK:
            raise LinearSolveError(_lib.SOLVE_MESSAGES.get(int(info[0]), f"status {info[0]}"))
        stats = self.stats.cpu().numpy()
        if not stats[1] <= 1e-8:
            raise ValueError("incompatible data: gauge changed physical equations")
        del torch
        return info, stats

    def prepare_offline(self, stream=None):
        """Offline step of ``OfflineHybridSystem`` (``core/offline.py:148-229``): one full
        solve with the current coefficients that also keeps every cell's factor in HBM
        (``mhm_q1_factor_bytes``: 161 MB in FP64, 80 MB with binary32 factors at
        64x64 x 16x16).  Later ``solve_source`` calls change the source only."""
        nbytes = int(self.lib.mhm_q1_factor_bytes(self.q1, PRECISIONS[self.precision]))
        if nbytes <= 0:
            raise RuntimeError("could not size the factor store")
        if getattr(self, "factors", None) is None or self.factors.numel() != nbytes:
            self.factors = self.torch.empty(nbytes, dtype=self.torch.uint8, device=self.device)
        self.launch(stream, local="offline")
        self.check()

    def set_source(self, source=0.0, *, non_blocking=False):
        """Replace the source only (the permeability and the kept factors stay)."""
        smode, sarr, sconst = source_input(source, self.mesh, self.rx, self.ry, self.order)
        if self.q1.kappa_mode >= 3:
            _cut_source_check(smode)
        self.source = None if sarr is None else self.torch.as_tensor(np.array(sarr)).to(
            self.device, non_blocking=non_blocking)
        q = self.q1
        q.source_mode, q.source, q.source_const = smode, _lib.ptr(self.source), float(sconst)
        self._keep = (self._keep[0], self.source)

    def solve_source(self, source=0.0, stream=None) -> Q1Solution:
        """Online step (``OfflineHybridSystem.solve``, ``core/offline.py:231-307``): the
        new source's local responses with the kept factors, the reduced right-hand
        side, the global solve with the unchanged skeleton matrix, reconstruction."""
        t0 = time.perf_counter()
        self.set_source(source)
        self.launch(stream, local="online")
        sol = self.result()
        sol.seconds = time.perf_counter() - t0
        return sol

    def refine(self, *, max_steps=2, min_steps=0, rtol=1e-10, atol=0.0, stream=None,
               refinement_precision="double") -> HybridRefinement:
        """Defect correction of the original equations (``refine_hybrid``,
        ``core/refinement.py:612-800``) applied to the plan's last solve.

        Each step evaluates the uncondensed local residuals d = f - B lambda - A u and
        the weak trace residual boundary - sum B^T u in double-double arithmetic
        (``mhm_q1_original_defect``).  It accepts when their norm is at most
        ``max(atol, rtol * rhs_norm)`` (after at least ``min_steps`` corrections).
        Otherwise it solves every cell once more with its defect as the source: with
        the factors kept by ``prepare_offline`` when they belong to the current
        permeability, else with a fresh factorization.  The reduced loads of those
        responses and the weak residual form the right-hand side of a global solve
        with the unchanged skeleton matrix.  The correction's trace and coarse values
        and its reconstructed fields are added to the current ones, so the fields
        need not be the reconstruction of the kept responses (the reference accepts
        any ``HybridSolution``); the fluxes are evaluated again from the corrected
        fields.  The source column of the local responses
        then holds the last defect's response.  A residual still above the threshold
        after ``max_steps`` corrections raises ``LinearSolveError``.  With Neumann faces
        the prescribed trace coefficients stay as they are: the right-hand-side norm
        takes the loads less their coupling and the free DOFs' boundary data, the
        weak residual counts the free DOFs, and each correction solves with those
        DOFs held at zero (``refinement.py:676-709, 792``).  A pure-Neumann solve carries
        its mean-pressure moment as the reference's ``moments``: the residual includes
        the moment defect value - sum_cells C . u, the right-hand-side norm the value,
        and each correction is gauged to the moment defect (``refinement.py:690-700,
        725-733, 787-797``).

        ``refinement_precision="extended"`` keeps the solution as double-double values
        (the reference stores it in a wider NumPy type, ``refinement.py:636-643``): the
        defects are evaluated from both parts and each correction is added in
        double-double arithmetic, so the residual can fall below the binary64 floor of
        the stored solution.  The returned fields and unknowns are the high parts; the
        low parts are in ``extra["trace_lo"]``, ``extra["coarse_lo"]`` and
        ``extra["fields_lo"]``.
        """
        if refinement_precision not in ("double", "extended"):
            raise ValueError("refinement_precision must be double or extended")
        extended = refinement_precision == "extended"
        _step_limits(max_steps, min_steps)
        _tolerances(rtol, atol)
        torch, L, P = self.torch, self.lib, _lib.ptr
        s = _lib.stream_handle(stream)
        cur = torch.cuda.current_stream() if stream is None else stream
        self.check()
        M, n, t = self.cells, self.n, self.t
        if getattr(self, "_refine", None) is None:
            f64 = dict(dtype=torch.float64, device=self.device)
            self._refine = dict(defect=torch.empty((M, n), **f64), slots=torch.empty((M, t), **f64),
                                weak=torch.empty(self.T, **f64), partial=torch.empty((M, 3), **f64),
                                norms=torch.empty(5 + 5 * 256, **f64), dx=torch.empty(self.N, **f64),
                                zero=torch.zeros(self.N, **f64), gauge_x=torch.zeros(self.N, **f64),
                                gauge_partial=torch.zeros(2 * M + 1, **f64), shift=torch.zeros(self.N, **f64),
                                rhs=torch.empty(self.N, **f64), scale=torch.empty(self.N, **f64),
                                dfields=torch.empty((M, n), **f64))
        B = self._refine
        if extended:
            B["x_lo"] = torch.zeros_like(self.x)
            B["fields_lo"] = torch.zeros_like(self.fields)
        qd = _lib.Q1Problem.from_buffer_copy(self.q1)
        qd.source_mode, qd.source, qd.source_const = 3, P(B["defect"]), 0.0
        factors = self.factors if getattr(self, "_factors_current", False) else None
        pat = self.pattern
        history, step = [], 0
        while True:
            if extended:
                _lib.check(L.mhm_q1_original_defect_dd(self.q1, P(self.d_cell_dofs), self.T, P(self.d_dof_cells),
                                                       P(self.d_dof_slot), P(self.d_fixed), P(self.x),
                                                       P(B["x_lo"]), P(self.fields), P(B["fields_lo"]),
                                                       P(self.d_boundary), P(B["defect"]), P(B["slots"]),
                                                       P(B["weak"]), P(B["partial"]), s),
                           "mhm_q1_original_defect_dd")
            else:
                _lib.check(L.mhm_q1_original_defect(self.q1, P(self.d_cell_dofs), self.T, P(self.d_dof_cells),
                                                    P(self.d_dof_slot), P(self.d_fixed), P(self.x), P(self.fields),
                                                    P(self.d_boundary), P(B["defect"]), P(B["slots"]),
                                                    P(B["weak"]), P(B["partial"]), s),
                           "mhm_q1_original_defect")
            _lib.check(L.mhm_refine_norms(M, P(B["partial"]), self.T, P(self.d_fixed), P(B["weak"]),
                                          P(self.d_boundary), self.N,
                                          P(self.d_indptr), P(self.d_indices), P(self.values), P(self.x),
                                          P(self.rhs), P(B["norms"]), s), "mhm_refine_norms")
            moment_defect = 0.0
            if self.pure_neumann:  # sum_cells C . u from the gauge kernel's per-cell partials
                _lib.check(L.mhm_q1_mean_gauge(self.q1, P(self.solution), P(self.fields), 0.0, self.T,
                                               P(B["gauge_x"]), P(B["gauge_partial"]), s), "mhm_q1_mean_gauge")
            cur.synchronize()
            norms = B["norms"][:5].cpu().numpy()
            if self.pure_neumann:
                moment_defect = self.mean_value - float(np.sum(B["gauge_partial"][0:2 * M:2].cpu().numpy()))
                norms[0] += moment_defect * moment_defect
                norms[1] += self.mean_value * self.mean_value
            residual, rhs_norm = math.sqrt(norms[0]), math.sqrt(norms[1])
            history.append(residual)
            threshold = max(atol, rtol * rhs_norm)
            if step >= min_steps and math.isfinite(residual) and residual <= threshold:
                sol = self.result()
                scale = max(math.sqrt(norms[3]), math.sqrt(norms[4]), np.finfo(float).tiny)
                sol.residual = math.sqrt(norms[2]) / scale
                sol.extra["refinement_steps"] = step
                if extended:
                    xl = B["x_lo"].cpu().numpy()
                    sol.extra["trace_lo"], sol.extra["coarse_lo"] = xl[: self.T].copy(), xl[self.T:].copy()
                    sol.extra["fields_lo"] = B["fields_lo"].cpu().numpy()
                return HybridRefinement(sol, tuple(history), rhs_norm)
            if step == max_steps or not math.isfinite(residual):
                raise LinearSolveError(f"original hybrid residual {residual:.6e} exceeds {threshold:.6e} "
                                       f"after {step} corrections")
            _lib.check(L.mhm_q1_correction_response(qd, PRECISIONS[self.precision], self.max_refine,
                                                    self.local_tol, P(factors), P(self.solution), P(self.loads),
                                                    P(self.corrected), P(self.cell_status), P(self.cell_iters), s),
                       "mhm_q1_correction_response")
            _lib.check(L.mhm_skeleton_scatter(0, P(self.d_slot_ptr), P(self.d_contrib), P(self.blocks),
                                              P(self.values), self.N, self.T, P(self.d_load_ptr),
                                              P(self.d_load_contrib), P(self.loads), P(B["weak"]), P(B["rhs"]),
                                              P(B["scale"]), s), "mhm_skeleton_scatter")
            if self.d_fixed is not None:  # the correction holds the prescribed DOFs at zero
                _lib.check(L.mhm_skeleton_fixed_rhs(self.N, self.T, P(self.d_indptr), P(self.d_indices),
                                                    P(self.values), P(self.d_fixed), P(B["zero"]), P(B["rhs"]),
                                                    P(B["rhs"]), s), "mhm_skeleton_fixed_rhs")
            if self.pure_neumann:
                # The correction's loads come from binary64 defects, so their component
                # along the kernel of the system (a uniform shift of the coarse unknowns)
                # is rounding of the defects, not of the data.  The reference's bordered
                # solve absorbs it in its multiplier; here it leaves the right-hand side.
                cur.synchronize()
                mean = float(np.mean(B["rhs"][self.T:].cpu().numpy()))
                B["shift"][self.T:].fill_(-mean)
                _lib.check(L.mhm_vector_accumulate(self.N, P(B["rhs"]), P(B["shift"]), s), "mhm_vector_accumulate")
            _lib.check(L.mhm_skeleton_solve(self.sys, P(B["rhs"]), P(B["scale"]), P(B["dx"]), self.global_rtol,
                                            self.inner_rtol, self.max_inner, self.max_outer, self.grid,
                                            P(self.workspace), self.workspace.numel(), P(self.info), P(self.stats),
                                            s), "mhm_skeleton_solve")
            if self.pure_neumann:  # the correction carries the moment defect (its gauge row)
                _lib.check(L.mhm_q1_reconstruct(self.q1, P(self.solution), P(self.d_cell_dofs), self.T, P(B["dx"]),
                                                P(B["dfields"]), None, s), "mhm_q1_reconstruct")
                _lib.check(L.mhm_q1_mean_gauge(self.q1, P(self.solution), P(B["dfields"]), moment_defect, self.T,
                                               P(B["dx"]), P(B["gauge_partial"]), s), "mhm_q1_mean_gauge")
            _lib.check(L.mhm_q1_reconstruct(self.q1, P(self.solution), P(self.d_cell_dofs), self.T, P(B["dx"]),
                                            P(B["dfields"]), None, s), "mhm_q1_reconstruct")
            for dst, lo, src in ((self.x, "x_lo", B["dx"]), (self.fields, "fields_lo", B["dfields"])):
                if extended:
                    _lib.check(L.mhm_vector_accumulate_dd(dst.numel(), P(dst), P(B[lo]), P(src), s),
                               "mhm_vector_accumulate_dd")
                else:
                    _lib.check(L.mhm_vector_accumulate(dst.numel(), P(dst), P(src), s), "mhm_vector_accumulate")
            _lib.check(L.mhm_q1_flux(self.q1, P(self.fields), P(self.flux), s), "mhm_q1_flux")
            cur.synchronize()
            self.check()
            step += 1

    def capture(self, local="online", stream=None):
        """Capture one solve as a CUDA graph that ``replay`` runs again.

        ``local="offline"`` captures the condensation that keeps every cell's factor,
        the skeleton reduction, the global solve and the reconstruction
        (``OfflineHybridSystem``'s offline step); ``"online"`` captures a new source's
        responses with the kept factors, the right-hand-side reduction, the global
        solve and the reconstruction.  Kernel arguments are fixed at capture: the
        permeability buffer must stay where ``set_device_coefficients`` put it, and the
        source is read from a persistent per-fine-cell device buffer that each replay
        overwrites first (a constant source gives the same element loads as
        ``source_mode`` 0).  ``"condense"`` captures a complete fresh solve with the
        coefficients exactly as set (pointwise sources included); its replays take no
        source and refuse to run once ``set_coefficients`` has moved the coefficient
        buffers.  ``"batched"`` captures the reduction, global solve and reconstruction
        that follow a ``condense_batch`` local stage (its replays take no source).  The
        graph's launches run once eagerly before the capture."""
        torch = self.torch
        if local not in ("offline", "online", "condense", "batched"):
            raise ValueError("local must be 'offline', 'online', 'condense' or 'batched'")
        if local == "condense":
            return self._capture_graph(local, stream, keep=self._keep)
        if local == "batched":  # the rest of a solve whose local stage ran in condense_batch
            return self._capture_graph(local, stream)
        if local == "online" and not getattr(self, "_factors_current", False):
            raise RuntimeError("prepare_offline() must run before capturing online queries")
        if local == "offline" and getattr(self, "factors", None) is None:
            nbytes = int(self.lib.mhm_q1_factor_bytes(self.q1, PRECISIONS[self.precision]))
            self.factors = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        if getattr(self, "_graph_source", None) is None:
            self._graph_source = torch.zeros((self.nxf, self.nyf), dtype=torch.float64, device=self.device)
        q = self.q1
        q.source_mode, q.source, q.source_const = 1, _lib.ptr(self._graph_source), 0.0
        self._keep = (self._keep[0], self._graph_source)
        return self._capture_graph(local, stream)

    def _capture_graph(self, local, stream, keep=None):
        torch = self.torch
        if getattr(self, "_graphs", None) is None:
            self._graphs, self._graph_stream = {}, None
        st = self._graph_stream or (torch.cuda.Stream(device=self.device) if stream is None else stream)
        self._graph_stream = st
        st.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(st):
            self.launch(st, local=local)  # warm-up outside the capture
        st.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=st):
            self.launch(st, local=local)
        self._graphs[local] = graph
        if keep is not None:
            # the captured kernels read these buffers: hold them, and remember where they were
            self._graph_keep = (keep, self.q1.kappa, self.q1.source)
        return graph

    def capture_online(self, stream=None):
        """``capture("online")``; requires ``prepare_offline``."""
        return self.capture("online", stream)

    def replay(self, local="online", source=None, *, stream=None, after=None):
        """Run the captured ``local`` solve for ``source`` (a constant or one value per
        fine cell, shape (nx*rx, ny*ry); default 0 for ``"offline"``/``"online"``, none
        for ``"condense"``), asynchronously on ``stream`` (default: the capture stream)
        after ``after`` (default: the current stream).  Returns the stream it ran on."""
        torch = self.torch
        graph = (getattr(self, "_graphs", None) or {}).get(local)
        if graph is None:
            raise RuntimeError(f"capture({local!r}) must run first")
        if local == "batched":
            if source is not None:
                raise ValueError("the batched remainder takes no source: the local stage consumed it")
            st = self._graph_stream if stream is None else stream
            if after is not st:
                st.wait_stream(torch.cuda.current_stream() if after is None else after)
            with torch.cuda.stream(st):
                graph.replay()
            return st
        if local == "condense":
            if source is not None:
                raise ValueError("the captured fresh solve reads the coefficients set before capture; "
                                 "set_coefficients and capture('condense') again to change them")
            _, kappa_ptr, source_ptr = self._graph_keep
            if self.q1.kappa != kappa_ptr or self.q1.source != source_ptr:
                raise RuntimeError("the coefficients changed since capture('condense'); capture again")
            st = self._graph_stream if stream is None else stream
            if after is not st:
                st.wait_stream(torch.cuda.current_stream() if after is None else after)
            with torch.cuda.stream(st):
                graph.replay()
            return st
        source = 0.0 if source is None else source
        st = self._graph_stream if stream is None else stream
        if after is not st:
            st.wait_stream(torch.cuda.current_stream() if after is None else after)
        with torch.cuda.stream(st):
            if isinstance(source, numbers.Number):
                self._graph_source.fill_(float(source))
            else:
                arr = np.asarray(source, dtype=float)
                if arr.shape != (self.nxf, self.nyf):
                    raise ValueError(f"fine-cell source must have shape ({self.nxf}, {self.nyf})")
                self._graph_source.copy_(torch.as_tensor(arr), non_blocking=False)
            graph.replay()
        if local == "offline":
            self._factors_current = True
        return st

    def replay_online(self, source=0.0, *, stream=None):
        """``replay("online", source, after=stream)``."""
        return self.replay("online", source, after=stream)

    def result(self, seconds=0.0) -> Q1Solution:
        info, stats = self.check()
        x = self.x.cpu().numpy()
        return Q1Solution(
            trace=x[: self.T].copy(), coarse=x[self.T:].copy(), fields=self.fields.cpu().numpy(),
            flux=self.flux.cpu().numpy(), residual=float(stats[1]), raw_residual=float(stats[0]),
            corrected=self.corrected.cpu().numpy().astype(bool), local_iterations=self.cell_iters.cpu().numpy(),
            global_iterations=int(info[1]), outer_corrections=int(info[2]), seconds=seconds)

    def solve(self, permeability=1.0, source=0.0, stream=None) -> Q1Solution:
        t0 = time.perf_counter()
        self.set_coefficients(permeability, source)
        self.launch(stream)
        sol = self.result()
        sol.seconds = time.perf_counter() - t0
        return sol

    def export_csc(self, stream=None):
        """The assembled skeleton matrix as the reference hands it on, on the device:
        CSC with the entries whose sum is exactly zero dropped (``coo_matrix(...).tocsc()``
        then ``eliminate_zeros()``, ``core/contributions.py:184-185``).  Returns
        ``(indptr int64 (N+1), indices int32, data float64)`` device tensors trimmed to
        the kept entries; the solver keeps using the structural pattern."""
        torch = self.torch
        if getattr(self, "_csc", None) is None:
            p = self.pattern
            nnz = len(p.indices)
            self._csc = dict(
                transpose=torch.as_tensor(transpose_slots(p.indptr, p.indices)).to(self.device),
                indptr=torch.empty(self.N + 1, dtype=torch.int64, device=self.device),
                indices=torch.empty(nnz, dtype=torch.int32, device=self.device),
                data=torch.empty(nnz, dtype=torch.float64, device=self.device))
        c = self._csc
        P = _lib.ptr
        _lib.check(self.lib.mhm_skeleton_export_csc(self.N, P(self.d_indptr), P(self.d_indices), P(c["transpose"]),
                                                    P(self.values), P(c["indptr"]), P(c["indices"]), P(c["data"]),
                                                    _lib.stream_handle(stream)), "mhm_skeleton_export_csc")
        kept = int(c["indptr"][-1])
        return c["indptr"], c["indices"][:kept], c["data"][:kept]

    def matrix(self):
        """Host copy of the assembled skeleton matrix in the reference's form
        (``export_csc``): a SciPy CSC matrix whose ``indptr`` / ``indices`` follow the
        reference's rule for which entries are stored."""
        from scipy import sparse

        indptr, indices, data = self.export_csc()
        return sparse.csc_matrix((data.cpu().numpy(), indices.cpu().numpy(), indptr.cpu().numpy()),
                                 shape=(self.N, self.N))


def condense_batch(plans, *, offline=False, stream=None):
    """One launch of the local stage of several plans of one shape (macro grid, local
    refinement, trace spaces, precision), each with its own permeability and source
    already set: the cells of plan k are the CTAs (x, k) of ``mhm_q1_condense_batch``,
    which writes every plan's own responses, Schur blocks and status words exactly as
    its own ``mhm_q1_condense`` launch would.  With ``offline``, each plan keeps its
    cells' factors for later sources (``prepare_offline``).  Follow with
    ``plan.launch(stream, local="batched")`` per plan.  This is the cross-request
    batching of a serving loop's local stages; at most 16 plans per launch and
    permeabilities without a pre-pass (constant, per fine cell, or pixels aligned with
    the fine grid)."""
    import ctypes as C

    plans = list(plans)
    if not 1 <= len(plans) <= 16:
        raise ValueError("condense_batch takes 1 to 16 plans")
    first = plans[0]
    for p in plans:
        if p.precision != first.precision or (p.mesh.nx, p.mesh.ny, p.rx, p.ry) != (first.mesh.nx, first.mesh.ny,
                                                                                   first.rx, first.ry):
            raise ValueError("condense_batch needs plans of one shape and precision")
    torch = first.torch
    lib = first.lib
    prec = PRECISIONS[first.precision]
    if offline:
        for p in plans:
            if getattr(p, "factors", None) is None:
                nbytes = int(lib.mhm_q1_factor_bytes(p.q1, prec))
                if nbytes <= 0:
                    raise RuntimeError("could not size the factor store")
                p.factors = torch.empty(nbytes, dtype=torch.uint8, device=p.device)
    k = len(plans)
    P = _lib.ptr

    def arr(name):
        return (C.c_void_p * k)(*[P(getattr(p, name)) for p in plans])

    problems = (_lib.Q1Problem * k)(*[p.q1 for p in plans])
    factors = arr("factors") if offline else None
    _lib.check(lib.mhm_q1_condense_batch(k, problems, prec, first.max_refine, first.local_tol, arr("solution"),
                                         arr("blocks"), arr("loads"), arr("corrected"), arr("cell_status"),
                                         arr("cell_iters"), factors, _lib.stream_handle(stream)),
               "mhm_q1_condense_batch")
    for p in plans:
        p._factors_current = bool(offline)


def solve_darcy_quadrilateral(mesh, *, permeability=1.0, source=0.0, dirichlet=0.0, neumann=None,
                              skeleton=None, local_refinement=4, degree=1, quadrature_order=4,
                              mean_pressure=0.0, solver="gpu", local_solver="gpu", backend="serial",
                              workers=None, precision="fp64", hybrid_refinement_steps=0,
                              hybrid_refinement_min_steps=0) -> Q1Solution:
    """GPU counterpart of ``solve_darcy_quadrilateral`` (``cartesian.py:86-168``).

    Weak Dirichlet data on the faces not listed in ``neumann``; Neumann data (outward
    normal fluxes) on any set of boundary faces prescribes those faces' trace
    coefficients, which the global solve eliminates; with every face Neumann the
    pressure mean over the domain is ``mean_pressure`` (the reference's gauge).  The
    ``solver``, ``local_solver``, ``backend`` and ``workers`` arguments are
    accepted for signature compatibility: the whole solve runs on the GPU.
    ``hybrid_refinement_steps`` / ``hybrid_refinement_min_steps`` follow the Darcy
    driver's keywords (``_legacy/models/darcy/primal.py:191-244, 306-316``): a positive
    count corrects the original equations after condensation (``refine_hybrid``,
    relative residual 1e-10) and raises ``LinearSolveError`` if that fails.
    """
    _refinement_steps(hybrid_refinement_steps)
    _refinement_steps(hybrid_refinement_min_steps)
    if hybrid_refinement_min_steps > hybrid_refinement_steps:
        raise ValueError("hybrid_refinement_min_steps must not exceed hybrid_refinement_steps")
    del solver, local_solver, backend, workers
    order = max(int(quadrature_order), int(degree) + 1)
    plan = CartesianQ1Plan(mesh, skeleton, local_refinement, dirichlet=dirichlet, neumann=neumann,
                           mean_pressure=mean_pressure, quadrature_order=order, degree=degree, precision=precision)
    sol = plan.solve(permeability, source)
    if hybrid_refinement_steps:
        sol = plan.refine(max_steps=hybrid_refinement_steps, min_steps=hybrid_refinement_min_steps).solution
    return sol


def refine_hybrid(plan, *, max_steps=2, min_steps=0, rtol=1e-10, atol=0.0, stream=None,
                  refinement_precision="double") -> HybridRefinement:
    """``refine_hybrid`` (``core/refinement.py:612-800``) for a solved ``CartesianQ1Plan``:
    the plan holds the system, the solution and the boundary load that the reference
    passes separately.  See ``CartesianQ1Plan.refine``."""
    return plan.refine(max_steps=max_steps, min_steps=min_steps, rtol=rtol, atol=atol, stream=stream,
                       refinement_precision=refinement_precision)
