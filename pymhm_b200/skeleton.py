"""GPU global skeleton solver behind the reference's ``LinearFactorization`` contract.

``SkeletonFactorization`` follows ``LinearFactorization`` (``src/pymhm/linalg/
linear.py:240-331``) the way ``SaddleBlockSolver.as_factorization`` does
(``linalg/block.py:211-217``): ``matches``, ``solve``, ``close``, ``rtol``.  It is
passed as ``HybridSystem.solve(factorization=...)`` (``core/system.py:448-457``)
for a Cartesian macro mesh with a uniform scalar skeleton and no gauge rows.  With
``fixed`` (the prescribed trace DOFs of Neumann faces, as passed to
``solve(fixed=...)``) it serves the reduced system that ``solve_hybrid_system`` hands
over (``:421-447``).  The solve is ``mhm_skeleton_solve`` (projected PCG with FP64 outer
correction); every result is checked against the columnwise residual criterion
of ``_checked`` (``linear.py:132-152``).
"""

from __future__ import annotations

import numpy as np
from scipy import sparse

from . import _lib
from .errors import LinearSolveError
from .topology import (
    SkeletonSpace,
    coarse_coefficients,
    dof_cell_maps,
    fixed_coarse_data,
    geometric_constraint,
    mesh_arrays,
    skeleton_pattern,
)


def attach_fixed(system, data: dict, up) -> dict:
    """Point ``system`` (an ``mhm_skeleton_system``) at device copies of
    ``topology.fixed_coarse_data``; ``up(array, dtype)`` uploads.  Returns the device
    tensors, which must outlive the solves."""
    import torch

    keep = {"mask": up(data["mask"], torch.uint8)}
    system.fixed, system.coarse_neumann = _lib.ptr(keep["mask"]), int(data["bits"])
    if data["qx"] is not None:
        keep["qx"], keep["lamx"] = up(data["qx"], torch.float64), up(data["lamx"], torch.float64)
        system.coarse_qx, system.coarse_lamx = _lib.ptr(keep["qx"]), _lib.ptr(keep["lamx"])
    if data["pinv0"] is not None:
        keep["pinv0"] = up(data["pinv0"], torch.float64)
        system.coarse_pinv0 = _lib.ptr(keep["pinv0"])
    if data["wb_cells"] is not None:
        keep["wb_cells"], keep["wb_R"] = up(data["wb_cells"], torch.int32), up(data["wb_R"], torch.float64)
        system.coarse_partial = len(data["wb_cells"])
        system.coarse_partial_cells, system.coarse_partial_R = _lib.ptr(keep["wb_cells"]), _lib.ptr(keep["wb_R"])
    return keep


def _canonical(matrix) -> sparse.csr_matrix:
    op = sparse.csr_matrix(matrix, dtype=float, copy=True)
    op.sum_duplicates()
    op.sort_indices()
    return op


class SkeletonFactorization:
    """Prepared GPU solver for one assembled skeleton matrix."""

    solver = "mhm_b200"

    def __init__(self, matrix, mesh, skeleton=None, *, fixed=None, rtol: float = 1e-10, inner_rtol: float = 1e-10,
                 max_inner: int = 5000, max_outer: int = 8):
        """``matrix``: the assembled system (``system.matrix``).  ``fixed``: trace DOF
        indices (or the ``{dof: value}`` map of ``boundary_data``) prescribed on whole
        boundary faces; the factorization then matches and solves the system with
        those rows and columns removed."""
        import torch

        self.torch = torch
        self.lib = _lib.lib()
        self.mesh = mesh_arrays(mesh)
        self.skeleton = SkeletonSpace(self.mesh) if skeleton is None else SkeletonSpace.of(skeleton, self.mesh)
        space_h, space_v = self.skeleton.uniform_by_orientation()
        if space_h.size != space_v.size:
            raise NotImplementedError("the GPU skeleton solver requires equal face sizes")
        self._matrix = _canonical(matrix)
        self.rtol = float(rtol)
        cell_dofs = self.skeleton.cell_dof_array
        T = self.skeleton.size
        M = len(self.mesh.cells)
        N = T + M
        if self._matrix.shape != (N, N):
            raise ValueError("matrix does not match the skeleton layout")
        pat = skeleton_pattern(cell_dofs, T)
        rows = np.repeat(np.arange(N), np.diff(pat.indptr))
        cols = pat.indices.astype(np.int64)
        values = np.asarray(self._matrix[rows, cols]).ravel()
        if not np.isclose(np.abs(values).sum(), np.abs(self._matrix.data).sum(), rtol=1e-14, atol=0):
            raise ValueError("matrix has entries outside the skeleton pattern")
        dev = torch.device("cuda")

        def up(a, dtype):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)

        dof_cells, dof_slot = dof_cell_maps(cell_dofs, T)
        self._keep = dict(
            indptr=up(pat.indptr, torch.int64), indices=up(pat.indices, torch.int32),
            values=up(values, torch.float64), trace_end=up(pat.trace_end, torch.int64),
            cell_dofs=up(cell_dofs, torch.int64), g0=up(geometric_constraint(self.mesh, space_h, space_v), torch.float64),
            dof_cells=up(dof_cells, torch.int32), dof_slot=up(dof_slot, torch.int32))
        k = self._keep
        s = self.sys = _lib.SkeletonSystem()
        s.size, s.trace_size = N, T
        s.indptr, s.indices, s.values = _lib.ptr(k["indptr"]), _lib.ptr(k["indices"]), _lib.ptr(k["values"])
        s.trace_end = _lib.ptr(k["trace_end"])
        s.faces, s.face_size, s.cells, s.cell_width = len(self.mesh.faces), space_h.size, M, cell_dofs.shape[1]
        s.cell_dofs, s.cell_g0 = _lib.ptr(k["cell_dofs"]), _lib.ptr(k["g0"])
        s.dof_cells, s.dof_slot = _lib.ptr(k["dof_cells"]), _lib.ptr(k["dof_slot"])
        s.nx, s.ny = self.mesh.nx, self.mesh.ny
        s.coarse_ax, s.coarse_ay = coarse_coefficients(self.mesh, space_h, space_v)
        self._free = None
        if fixed is not None and len(fixed):
            idx = np.array(sorted(int(i) for i in fixed), dtype=np.int64)
            if idx[0] < 0 or idx[-1] >= T:
                raise ValueError("fixed DOFs must be valid trace indices")
            faces = [int(f) for f in self.mesh.boundary_faces if np.all(np.isin(self.skeleton.dofs(int(f)), idx))]
            covered = np.concatenate([self.skeleton.dofs(f) for f in faces]) if faces else np.zeros(0, np.int64)
            if not np.array_equal(np.sort(covered), idx):
                raise NotImplementedError("fixed DOFs must be all trace DOFs of boundary faces")
            if len(faces) == len(self.mesh.boundary_faces):
                raise NotImplementedError("a system with every boundary face fixed needs its gauge rows, "
                                          "which this factorization does not take")
            self._fixed_keep = attach_fixed(s, fixed_coarse_data(self.mesh, self.skeleton, faces, s.coarse_ax,
                                                                 s.coarse_ay),
                                            lambda a, dtype: up(a, dtype))
            self._free = np.setdiff1d(np.arange(N), idx)
            self._reduced = _canonical(self._matrix[self._free][:, self._free])
        nbytes = self.lib.mhm_skeleton_workspace_bytes(s, 0)
        self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        self.info = torch.zeros(4, dtype=torch.int32, device=dev)
        self.stats = torch.zeros(4, dtype=torch.float64, device=dev)
        self.inner_rtol, self.max_inner, self.max_outer = inner_rtol, max_inner, max_outer
        self._open = True
        self.N = N

    def matches(self, matrix) -> bool:
        own = self._matrix if self._free is None else self._reduced
        other = _canonical(matrix)
        return bool(own.shape == other.shape and (own != other).nnz == 0)

    def _solve_one(self, b: np.ndarray) -> np.ndarray:
        torch = self.torch
        rhs = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64), device="cuda")
        x = torch.empty_like(rhs)
        P = _lib.ptr
        _lib.check(self.lib.mhm_skeleton_solve(self.sys, P(rhs), 0, P(x), 1e-13,
                                               self.inner_rtol, self.max_inner, self.max_outer, 0,
                                               P(self.workspace), self.workspace.numel(), P(self.info),
                                               P(self.stats), _lib.stream_handle(None)), "mhm_skeleton_solve")
        info = self.info.cpu().numpy()
        if info[0] not in (_lib.SOLVE_OK, _lib.SOLVE_NOT_CONVERGED):
            raise LinearSolveError(_lib.SOLVE_MESSAGES.get(int(info[0]), f"status {info[0]}"))
        return x.cpu().numpy()

    def solve(self, rhs, *, refinement_precision: str = "double", refinement_steps: int = 2) -> np.ndarray:
        if not self._open:
            raise RuntimeError("factorization is closed")
        if refinement_precision != "double":
            raise ValueError("the GPU skeleton solver refines in double precision")
        del refinement_steps
        forcing = np.asarray(rhs, dtype=float)
        n = self.N if self._free is None else len(self._free)
        if forcing.ndim not in (1, 2) or forcing.shape[0] != n or not np.all(np.isfinite(forcing)):
            raise ValueError("rhs must have shape (n,) or (n, nrhs) matching matrix")
        cols = forcing[:, None] if forcing.ndim == 1 else forcing
        if self._free is None:
            out = np.column_stack([self._solve_one(cols[:, j]) for j in range(cols.shape[1])])
            op = self._matrix
        else:  # the masked solve on the full layout, fixed rows zero
            full = np.zeros((self.N, cols.shape[1]))
            full[self._free] = cols
            out = np.column_stack([self._solve_one(full[:, j])[self._free] for j in range(cols.shape[1])])
            op = self._reduced
        # columnwise acceptance as in linalg/linear.py:132-152
        diff = op @ out - cols
        scale = np.max(np.abs(cols), axis=0)
        scale = np.where(scale > 0, scale, 1.0)
        res = np.linalg.norm(diff / scale, axis=0)
        thr = self.rtol * np.linalg.norm(cols / scale, axis=0)
        if np.any(res > thr):
            raise LinearSolveError(f"residual criterion failed: scaled ||Ax-b||={res}, allowed={thr}")
        return out[:, 0] if forcing.ndim == 1 else out

    def close(self) -> None:
        self._open = False
        self._keep = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
