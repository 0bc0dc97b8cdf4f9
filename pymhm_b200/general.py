"""Global skeleton solve for macro meshes of any shape (``mhm_general_solve``).

The Cartesian solver (``skeleton.py``) inverts its coarse operator with a sine
transform over the macro grid.  Tetrahedral and polygonal macro meshes have no such
structure, so this module describes their reduced system to the general kernel: the
cells' trace DOFs (ragged: a polygon has as many faces as edges), the exact geometric
constraint G0 = B^T 1 of every (cell, DOF), the DOF -> cell maps, the skeleton faces
that group the DOFs for the block-Jacobi preconditioner, and the dense inverse of the
coarse operator G0^T G0, which depends on the mesh only and is formed once here.
Callers that hold the cells' condensed blocks on the device (the local stage writes
them) pass them to ``launch``; the solver then preconditions with the cells'
D S_c^-1 D (cell-Dirichlet), which needs far fewer iterations than the face blocks.

``GeneralSkeleton.solve`` replaces the global solve of ``solve_hybrid_system``
(``core/system.py:355-528``) for systems without fixed DOFs or gauge rows;
``GeneralFactorization`` wraps it in the ``LinearFactorization`` contract
(``linalg/linear.py:240-331``: ``matches``, ``solve``, ``close``, ``rtol``).
"""

from __future__ import annotations

import numpy as np
from scipy import sparse

from . import _lib
from .errors import LinearSolveError
from .topology import block_offsets

MAX_FACE_DOFS = 8
MAX_CELL_DOFS_DIRICHLET = 32


def ragged(cell_dofs, cell_g0):
    """Flat (cell_ptr, dofs, g0) from per-cell sequences or equal-width 2-D arrays."""
    dofs = [np.asarray(d, dtype=np.int64).ravel() for d in cell_dofs]
    g0 = [np.asarray(g, dtype=np.float64).ravel() for g in cell_g0]
    if len(dofs) != len(g0) or any(len(a) != len(b) for a, b in zip(dofs, g0)):
        raise ValueError("cell_dofs and cell_g0 must have the same layout")
    ptr = np.zeros(len(dofs) + 1, dtype=np.int64)
    ptr[1:] = np.cumsum([len(d) for d in dofs])
    return ptr, np.concatenate(dofs), np.concatenate(g0)


def dof_maps(cell_ptr, flat_dofs, trace_size):
    """(T, 2) cells holding each trace DOF (first cell first, -1 padded) and the
    flat index of the DOF in each of them."""
    cells = np.repeat(np.arange(len(cell_ptr) - 1), np.diff(cell_ptr))
    entry = np.arange(len(flat_dofs), dtype=np.int64)
    order = np.lexsort((cells, flat_dofs))
    d, c, e = flat_dofs[order], cells[order], entry[order]
    if np.any(np.bincount(d, minlength=trace_size) > 2):
        raise ValueError("a trace DOF is shared by more than two cells")
    if len(d) and (d.min() < 0 or d.max() >= trace_size):
        raise ValueError("cell DOFs must be valid trace indices")
    first = np.ones(len(d), dtype=bool)
    first[1:] = d[1:] != d[:-1]
    k = np.where(first, 0, 1)
    dof_cells = np.full((trace_size, 2), -1, dtype=np.int32)
    dof_entry = np.zeros((trace_size, 2), dtype=np.int64)
    dof_cells[d, k] = c
    dof_entry[d, k] = e
    if np.any(dof_cells[:, 0] < 0):
        raise ValueError("every trace DOF must belong to at least one cell")
    return dof_cells, dof_entry


def coarse_inverse(cell_ptr, flat_dofs, flat_g0, trace_size):
    """Dense (G0^T G0)^-1 (cells x cells) of the geometric constraint."""
    M = len(cell_ptr) - 1
    cells = np.repeat(np.arange(M), np.diff(cell_ptr))
    G = sparse.csr_matrix((flat_g0, (flat_dofs, cells)), shape=(trace_size, M))
    A = (G.T @ G).toarray()
    try:
        chol = np.linalg.cholesky(A)
    except np.linalg.LinAlgError:
        raise NotImplementedError("the coarse operator G0^T G0 is singular (every boundary face fixed or "
                                  "a cell without constraint): this solver needs Dirichlet faces") from None
    inv = np.linalg.solve(chol.T, np.linalg.solve(chol, np.eye(M)))
    return 0.5 * (inv + inv.T)


class GeneralSkeleton:
    """Device-resident description of one reduced system layout.

    ``cell_dofs`` / ``cell_g0``: per cell, its trace DOFs and their G0 = B^T 1 entries;
    ``face_ptr`` (faces + 1): face f owns the trace DOFs ``face_ptr[f]..face_ptr[f+1]-1``
    (at most 8); ``indptr`` / ``indices``: the structural CSR of the whole reduced
    system (trace DOFs first, then one coarse unknown per cell), as the ordered scatter
    fills it.  ``block_off`` (cells + 1, from ``topology.block_offsets``) locates the
    cells' (t + 1)^2 condensed blocks in the flat array ``launch`` may be given.
    """

    def __init__(self, cell_dofs, cell_g0, face_ptr, trace_size, indptr, indices, *, device=None):
        import torch

        self.torch = torch
        self.lib = _lib.lib()
        self.device = torch.device("cuda" if device is None else device)
        self.T = int(trace_size)
        self.cell_ptr, self.flat_dofs, self.flat_g0 = ragged(cell_dofs, cell_g0)
        self.M = len(self.cell_ptr) - 1
        self.N = self.T + self.M
        face_ptr = np.asarray(face_ptr, dtype=np.int64)
        sizes = np.diff(face_ptr)
        if face_ptr[0] != 0 or face_ptr[-1] != self.T or np.any(sizes < 1) or sizes.max() > MAX_FACE_DOFS:
            raise ValueError(f"faces must partition the trace DOFs into groups of 1..{MAX_FACE_DOFS}")
        indptr = np.asarray(indptr, dtype=np.int64)
        if len(indptr) != self.N + 1:
            raise ValueError("the CSR pattern must cover trace and coarse unknowns")
        dof_cells, dof_entry = dof_maps(self.cell_ptr, self.flat_dofs, self.T)
        qinv = coarse_inverse(self.cell_ptr, self.flat_dofs, self.flat_g0, self.T)

        def up(a, dtype):
            return torch.as_tensor(np.array(a, order="C", copy=True), dtype=dtype).to(self.device)

        self._keep = dict(
            indptr=up(indptr, torch.int64), indices=up(indices, torch.int32), face_ptr=up(face_ptr, torch.int64),
            cell_ptr=up(self.cell_ptr, torch.int64), cell_dofs=up(self.flat_dofs, torch.int64),
            cell_g0=up(self.flat_g0, torch.float64), dof_cells=up(dof_cells, torch.int32),
            dof_entry=up(dof_entry, torch.int64), qinv=up(qinv, torch.float64))
        k = self._keep
        s = self.sys = _lib.GeneralSystem()
        s.size, s.trace_size = self.N, self.T
        s.indptr, s.indices, s.values = _lib.ptr(k["indptr"]), _lib.ptr(k["indices"]), 0
        s.faces, s.max_face_size, s.face_ptr = len(face_ptr) - 1, int(sizes.max()), _lib.ptr(k["face_ptr"])
        s.cells, s.cell_ptr = self.M, _lib.ptr(k["cell_ptr"])
        s.cell_dofs, s.cell_g0 = _lib.ptr(k["cell_dofs"]), _lib.ptr(k["cell_g0"])
        s.dof_cells, s.dof_entry = _lib.ptr(k["dof_cells"]), _lib.ptr(k["dof_entry"])
        s.coarse_inverse = _lib.ptr(k["qinv"])
        s.cell_entries = int(self.cell_ptr[-1])
        rows = np.repeat(np.arange(self.N), np.diff(indptr))
        trace_cols = np.asarray(indices) < self.T
        s.max_trace_row = int(np.bincount(rows[trace_cols], minlength=self.N).max())
        widths = np.diff(self.cell_ptr)
        bofs, _ = block_offsets([np.empty(int(t)) for t in widths])
        self.block_off = bofs
        self.cell_dirichlet = bool(widths.max() <= MAX_CELL_DOFS_DIRICHLET)
        if self.cell_dirichlet:
            k["block_off"] = up(bofs[:-1], torch.int64)
            s.block_off, s.blocks_size, s.max_cell_dofs = _lib.ptr(k["block_off"]), int(bofs[-1]), int(widths.max())
        nbytes = int(self.lib.mhm_general_workspace_bytes(s))
        if nbytes <= 0:
            raise RuntimeError("could not size the general skeleton workspace")
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        self.info = torch.zeros(4, dtype=torch.int32, device=self.device)
        self.stats = torch.zeros(3, dtype=torch.float64, device=self.device)

    def launch(self, values, rhs, x, *, blocks=None, rtol=1e-13, inner_rtol=1e-10, max_inner=20000, max_outer=16,
               stream=None):
        """Enqueue x = K^-1 rhs for the CSR ``values`` (device tensors, no host sync).

        ``blocks``: the cells' condensed blocks (flat, at ``block_off``) whose ordered
        scatter gave ``values``; with them (and cells of at most 32 DOFs) the solve
        uses the cell-Dirichlet preconditioner, else face block-Jacobi."""
        self.sys.values = _lib.ptr(values)
        if blocks is not None and self.cell_dirichlet:
            if blocks.numel() < int(self.block_off[-1]) or blocks.dtype != self.torch.float64:
                raise ValueError("blocks must hold every cell's (t + 1)^2 float64 block")
            self.sys.cell_blocks = _lib.ptr(blocks)
        else:
            self.sys.cell_blocks = 0
        P = _lib.ptr
        _lib.check(self.lib.mhm_general_solve(self.sys, P(rhs), P(x), P(self.workspace), self.workspace.numel(),
                                              float(rtol), float(inner_rtol), int(max_inner), int(max_outer),
                                              P(self.info), P(self.stats), _lib.stream_handle(stream)),
                   "mhm_general_solve")

    def check(self):
        """Status of the last solve (synchronises); raises the reference's error class."""
        info = self.info.cpu().numpy()
        stats = self.stats.cpu().numpy()
        if info[0] != _lib.SOLVE_OK:
            raise LinearSolveError(_lib.SOLVE_MESSAGES.get(int(info[0]), f"status {info[0]}"))
        return info, stats


class GeneralFactorization:
    """``LinearFactorization`` drop-in (``linalg/linear.py:240-331``) for the reduced
    system of any macro mesh: pass it as ``HybridSystem.solve(factorization=...)``.

    ``cell_dofs`` / ``cell_g0`` / ``face_ptr`` describe the skeleton (see
    ``GeneralSkeleton``); the matrix's stored entries must lie in the structural
    pattern those cells span.
    """

    solver = "mhm_b200_general"

    def __init__(self, matrix, cell_dofs, cell_g0, face_ptr, *, rtol: float = 1e-10, inner_rtol: float = 1e-10):
        import torch

        from .topology import skeleton_pattern_ragged

        op = sparse.csr_matrix(matrix, dtype=float, copy=True)
        op.sum_duplicates()
        op.sort_indices()
        self._matrix = op
        M = len(cell_dofs)
        T = op.shape[0] - M
        pat = skeleton_pattern_ragged(cell_dofs, T)
        N = T + M
        rows = np.repeat(np.arange(N), np.diff(pat.indptr))
        cols = pat.indices.astype(np.int64)
        values = np.asarray(op[rows, cols]).ravel()
        if not np.isclose(np.abs(values).sum(), np.abs(op.data).sum(), rtol=1e-14, atol=0):
            raise ValueError("matrix has entries outside the skeleton pattern")
        self.plan = GeneralSkeleton(cell_dofs, cell_g0, face_ptr, T, pat.indptr, pat.indices)
        self.values = torch.as_tensor(values, dtype=torch.float64, device=self.plan.device)
        self.rtol, self.inner_rtol, self.N = float(rtol), float(inner_rtol), N
        self._open = True

    def matches(self, matrix) -> bool:
        other = sparse.csr_matrix(matrix, dtype=float, copy=True)
        other.sum_duplicates()
        other.sort_indices()
        return bool(self._matrix.shape == other.shape and (self._matrix != other).nnz == 0)

    def solve(self, rhs, *, refinement_precision: str = "double", refinement_steps: int = 2) -> np.ndarray:
        if not self._open:
            raise RuntimeError("factorization is closed")
        if refinement_precision != "double":
            raise ValueError("the GPU skeleton solver refines in double precision")
        del refinement_steps
        torch = self.plan.torch
        forcing = np.asarray(rhs, dtype=float)
        if forcing.ndim not in (1, 2) or forcing.shape[0] != self.N or not np.all(np.isfinite(forcing)):
            raise ValueError("rhs must have shape (n,) or (n, nrhs) matching matrix")
        cols = forcing[:, None] if forcing.ndim == 1 else forcing
        out = np.empty_like(cols)
        for j in range(cols.shape[1]):
            b = torch.as_tensor(np.ascontiguousarray(cols[:, j]), device=self.plan.device)
            x = torch.empty_like(b)
            self.plan.launch(self.values, b, x)
            self.plan.check()
            out[:, j] = x.cpu().numpy()
        diff = self._matrix @ out - cols
        scale = np.max(np.abs(cols), axis=0)
        scale = np.where(scale > 0, scale, 1.0)
        res = np.linalg.norm(diff / scale, axis=0)
        thr = self.rtol * np.linalg.norm(cols / scale, axis=0)
        if np.any(res > thr):
            raise LinearSolveError(f"residual criterion failed: scaled ||Ax-b||={res}, allowed={thr}")
        return out[:, 0] if forcing.ndim == 1 else out

    def close(self) -> None:
        self._open = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
