"""Drop-ins for the reference's batched GPU local algebra and its local-solver protocol.

* ``BatchedFactorization`` mirrors ``pymhm.execution.cuda.BatchedFactorization``
  (``src/pymhm/execution/cuda.py:165-288``): equilibrated partial-pivoting LU of
  a ``(batch, n, n)`` FP64 stack, resident factors, columnwise FP64 residual
  acceptance with at most two corrections, the same error messages.
* ``condense_batched`` mirrors ``cuda.py:291-312``: groups problems by augmented
  size and right-hand-side width, solves each group in one batched call and
  decodes responses with the problem's own ``response_from_solution``.
* ``GpuLocalSolver`` implements ``LocalLinearSolver`` (``core/assembly.py:32-47``)
  for ``SolverConfig(local_solver=GpuLocalSolver())``.
* ``assemble_p1_batch`` mirrors ``cuda.py:27-105``: dense P1 stiffness, mass and
  load of a batch of triangle or tetrahedron meshes sharing one connectivity.

Compute is ``mhm_batched_factor`` / ``mhm_batched_solve`` / ``mhm_p1_batch_assemble``
from libmhm_b200.so.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .errors import LinearSolveError


def _torch():
    import torch

    return torch


class BatchedFactorization:
    """Resident equilibrated LU of real ``(batch, n, n)`` arrays on the current CUDA device."""

    def __init__(self, matrices, *, rtol: float = 1e-10, atol: float = 0.0) -> None:
        torch = _torch()
        if not (np.isfinite(rtol) and np.isfinite(atol)) or min(rtol, atol) < 0 or (rtol == 0 and atol == 0):
            raise ValueError("rtol and atol must be finite and nonnegative")
        self.lib = _lib.lib()
        self.device_id = torch.cuda.current_device()
        self.device = torch.device("cuda", self.device_id)
        self._closed = False
        self.matrix = self.factors = self.row_scale = self.col_scale = None
        try:
            raw = self._owned(matrices)
            if (raw.ndim != 3 or raw.shape[0] == 0 or raw.shape[1] == 0 or raw.shape[1] != raw.shape[2]
                    or raw.is_complex() or not bool(torch.isfinite(raw).all())):
                raise ValueError("matrices must be finite real arrays of shape (batch,n,n)")
            self.matrix = raw.to(torch.float64).contiguous().clone()
            count, n, _ = self.matrix.shape
            self.count, self.n = count, n
            self.factors = torch.empty_like(self.matrix)
            self.pivots = torch.empty((count, n), dtype=torch.int32, device=self.device)
            self.row_scale = torch.empty((count, n), dtype=torch.float64, device=self.device)
            self.col_scale = torch.empty((count, n), dtype=torch.float64, device=self.device)
            self.status = torch.empty(count, dtype=torch.int32, device=self.device)
            P = _lib.ptr
            _lib.check(self.lib.mhm_batched_factor(count, n, P(self.matrix), P(self.factors), P(self.pivots),
                                                   P(self.row_scale), P(self.col_scale), P(self.status),
                                                   _lib.stream_handle(None)), "mhm_batched_factor")
            self._raise(self.status.cpu().numpy())
            self.rtol, self.atol = float(rtol), float(atol)
        except BaseException:
            self.close()
            raise

    @staticmethod
    def _raise(status: np.ndarray) -> None:
        bad = np.flatnonzero(status)
        if len(bad):
            raise LinearSolveError(_lib.CELL_MESSAGES.get(int(status[bad[0]]), "batched LU failed"))

    def _owned(self, value):
        torch = _torch()
        if isinstance(value, torch.Tensor):
            if value.is_cuda and value.device.index != self.device_id:
                raise ValueError("resident arrays must belong to the factorization's CUDA device")
            return value.to(self.device)
        arr = np.asarray(value)
        if np.iscomplexobj(arr):
            raise ValueError("matrices must be finite real arrays")
        return torch.as_tensor(np.array(arr, dtype=np.float64), device=self.device)

    def solve(self, rhs, *, host: bool = False):
        """Solve ``(batch, n, nrhs)`` loads; resident tensor unless ``host=True``."""
        torch = _torch()
        if self._closed:
            raise RuntimeError("batched factorization is closed")
        raw = self._owned(rhs)
        if (raw.ndim != 3 or tuple(raw.shape[:2]) != (self.count, self.n) or raw.shape[2] == 0
                or raw.is_complex() or not bool(torch.isfinite(raw).all())):
            raise ValueError("rhs must be finite real arrays of shape (batch,n,nrhs)")
        forcing = raw.to(torch.float64).contiguous()
        nrhs = forcing.shape[2]
        x = torch.empty_like(forcing)
        work = torch.empty_like(forcing)
        status = self.status.clone()
        P = _lib.ptr
        _lib.check(self.lib.mhm_batched_solve(self.count, self.n, nrhs, P(self.matrix), P(self.factors),
                                              P(self.pivots), P(self.row_scale), P(self.col_scale), P(forcing),
                                              P(x), P(work), self.rtol, self.atol, 2, P(status),
                                              _lib.stream_handle(None)), "mhm_batched_solve")
        self._raise(status.cpu().numpy())
        return x.cpu().numpy() if host else x

    def close(self) -> None:
        if not self._closed:
            torch = _torch()
            try:
                if torch.cuda.is_available():
                    torch.cuda.synchronize(self.device_id)
            finally:
                self._closed = True
                self.factors = self.matrix = self.row_scale = self.col_scale = None

    def __enter__(self) -> "BatchedFactorization":
        if self._closed:
            raise RuntimeError("batched factorization is closed")
        return self

    def __exit__(self, *exc) -> None:
        self.close()


def _dense(matrix) -> np.ndarray:
    return matrix.toarray() if hasattr(matrix, "toarray") else np.asarray(matrix, dtype=float)


def condense_batched(problems):
    """Condense equal-size groups on the GPU, preserving input order (``cuda.py:291-312``).

    ``problems`` are objects with ``condensation_system()`` and
    ``response_from_solution(solution)`` (the reference's ``LocalProblem``).
    """
    groups: dict[tuple[int, int], list] = {}
    for index, problem in enumerate(problems):
        if not hasattr(problem, "condensation_system"):
            raise TypeError("every batch entry must be a LocalProblem")
        matrix, rhs = problem.condensation_system()
        groups.setdefault((matrix.shape[0], rhs.shape[1]), []).append((index, problem, matrix, rhs))
    responses = {}
    for group in groups.values():
        with BatchedFactorization(np.stack([_dense(e[2]) for e in group])) as batch:
            solved = batch.solve(np.stack([e[3] for e in group]), host=True)
        for (index, problem, _, _), result in zip(group, solved):
            responses[index] = problem.response_from_solution(result)
    return tuple(responses[i] for i in range(len(responses)))


class GpuLocalSolver:
    """``LocalLinearSolver`` callable: ``solver(matrix, rhs) -> solution`` on the GPU.

    Picklable (no device state is kept between calls), so it also works with the
    reference's spawn-process backend; each worker opens its own CUDA context.
    """

    def __init__(self, rtol: float = 1e-10):
        self.rtol = rtol

    def __call__(self, matrix, rhs):
        rhs = np.asarray(rhs, dtype=float)
        vector = rhs.ndim == 1
        cols = rhs[:, None] if vector else rhs
        with BatchedFactorization(_dense(matrix)[None], rtol=self.rtol) as f:
            out = f.solve(cols[None], host=True)[0]
        return out[:, 0] if vector else out

    def prepare_runtime(self) -> None:
        _lib.lib()

    def close(self) -> None:
        pass


_INCIDENCE: dict = {}


def _node_incidence(cells: np.ndarray, npoints: int):
    """Per node, element * (d+1) + local index of every incidence in ascending element
    order (CSR), cached per connectivity."""
    key = (cells.shape, npoints, cells.tobytes())
    hit = _INCIDENCE.get(key)
    if hit is None:
        nv = cells.shape[1]
        flat = cells.ravel().astype(np.int64)
        codes = np.arange(flat.size, dtype=np.int64)  # element * nv + local, ascending
        order = np.argsort(flat, kind="stable")
        ptr = np.zeros(npoints + 1, dtype=np.int64)
        np.add.at(ptr, flat + 1, 1)
        hit = (np.cumsum(ptr), codes[order].astype(np.int32))
        if len(_INCIDENCE) > 16:
            _INCIDENCE.clear()
        _INCIDENCE[key] = hit
    return hit


def _broadcast_strides(value, torch, lead, item_shape, dev):
    """``value`` broadcast to ``lead + item_shape``, lead = (batch, cells), as a
    contiguous FP64 base holding only the non-broadcast items, with the strides (in
    items) over batch and cells that address it (0 where broadcast)."""
    t = torch.as_tensor(value, device=dev)
    if t.is_complex():
        raise TypeError("complex coefficient")
    view = torch.broadcast_to(t, (*lead, *item_shape))
    nb = lead[0] if view.stride(0) != 0 else 1
    nc = lead[1] if view.stride(1) != 0 else 1
    base = view[:nb, :nc].to(torch.float64).contiguous()
    return base, (nc if nb > 1 else 0), (1 if nc > 1 else 0)


def assemble_p1_batch(points, cells, *, diffusion=1.0, source=0.0):
    """Dense P1 simplex operators of a batch of local meshes on the current CUDA device
    (``assemble_p1_batch``, ``execution/cuda.py:27-105``).

    ``points`` has shape ``(batch, npoints, d)``, d = 2 or 3; every mesh shares the
    integer connectivity ``cells[ncells, d+1]``.  ``diffusion`` is a positive scalar
    or SPD tensors broadcastable to ``(batch, ncells, d, d)``; ``source`` is constant
    per fine cell, broadcastable to ``(batch, ncells)``.  Returns the dense stiffness,
    consistent mass ``(batch, npoints, npoints)`` and load ``(batch, npoints)`` as
    CUDA tensors (the reference returns CuPy arrays).  Each entry sums its elements in
    ascending element order, so repeated calls give identical bits.  The same
    ``ValueError`` messages as the reference reject malformed geometry and
    coefficients.
    """
    torch = _torch()
    dev = torch.device("cuda", torch.cuda.current_device())
    pts = torch.as_tensor(points, device=dev) if not isinstance(points, torch.Tensor) else points.to(dev)
    if (pts.dim() != 3 or pts.shape[-1] not in (2, 3) or not pts.shape[0] or not pts.shape[1]
            or pts.is_complex() or not (pts.dtype.is_floating_point or pts.dtype in (torch.int32, torch.int64))):
        raise ValueError("points must be finite real arrays shaped (batch,npoints,2 or 3)")
    count, size, dim = (int(v) for v in pts.shape)
    conn = cells.cpu().numpy() if isinstance(cells, torch.Tensor) else np.asarray(cells)
    if (conn.ndim != 2 or conn.shape[1] != dim + 1 or not len(conn) or conn.dtype.kind not in "iu"
            or np.any(conn < 0) or np.any(conn >= size)):
        raise ValueError("cells must contain valid simplex node indices")
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    ncells = len(conn)
    pts = pts.to(torch.float64).contiguous()
    try:
        raw = torch.as_tensor(diffusion, device=dev)
        if raw.dim() == 0:
            raw = raw.to(torch.float64) * torch.eye(dim, dtype=torch.float64, device=dev)
        kbase, kb, kc = _broadcast_strides(raw, torch, (count, ncells), (dim, dim), dev)
    except (RuntimeError, TypeError, ValueError):
        raise ValueError("diffusion must be finite real symmetric positive definite") from None
    try:
        sbase, sb, sc = _broadcast_strides(source, torch, (count, ncells), (), dev)
    except (RuntimeError, TypeError, ValueError):
        raise ValueError("source must be real finite cell values") from None
    ptr, contrib = _node_incidence(conn, size)
    lib = _lib.lib()
    d_cells = torch.from_numpy(conn).to(dev)
    d_ptr = torch.from_numpy(ptr).to(dev)
    d_contrib = torch.from_numpy(contrib).to(dev)
    nbytes = int(lib.mhm_p1_batch_scratch_bytes(count, dim, ncells))
    scratch = torch.empty(nbytes // 8, dtype=torch.float64, device=dev)
    stiffness = torch.empty((count, size, size), dtype=torch.float64, device=dev)
    mass = torch.empty_like(stiffness)
    load = torch.empty((count, size), dtype=torch.float64, device=dev)
    status = torch.empty(4, dtype=torch.int32, device=dev)
    P = _lib.ptr
    _lib.check(lib.mhm_p1_batch_assemble(count, size, dim, P(pts), ncells, P(d_cells), P(kbase), kb, kc, P(sbase),
                                         sb, sc, P(d_ptr), P(d_contrib), P(scratch), P(stiffness), P(mass), P(load),
                                         P(status), _lib.stream_handle(None)), "mhm_p1_batch_assemble")
    flags = status.cpu().numpy()
    if flags[0]:
        raise ValueError("points must be finite real arrays shaped (batch,npoints,2 or 3)")
    if flags[1]:
        raise ValueError("degenerate simplex in resident geometry")
    if flags[2]:
        raise ValueError("diffusion must be finite real symmetric positive definite")
    if flags[3]:
        raise ValueError("source must be real finite cell values")
    return stiffness, mass, load
