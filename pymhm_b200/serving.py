"""Continuous-batching request loop for independent Cartesian Q1 Darcy solves.

Requests arrive over time, each with its own macro grid, local refinement,
permeability field and 1..8 sources.  The engine keeps *slots*: a resident
``CartesianQ1Plan`` for one request shape with its own CUDA stream, device
permeability buffer and pinned host buffers.  A request is admitted, in arrival
order, as soon as a slot of its shape is idle or a new one fits both the in-flight
limit and the HBM budget; otherwise it waits, and idle slots of other shapes are
released to make room.  Each slot captures both steps of a request as CUDA graphs
when it is created.  An admitted request is enqueued on its slot's stream without
host synchronisation: the permeability upload, then graph replays of the
condensation that keeps
every cell's factor (``OfflineHybridSystem``'s offline step,
``core/offline.py:148-229``), the global solve and the reconstruction for the first
source, then for each further source only the source responses with the kept
factors, the right-hand-side reduction, the global solve and the reconstruction
(``core/offline.py:231-313``), each followed by asynchronous copies of its results
and status to pinned memory.  With ``batch_local``, requests of one shape admitted in
the same pass share one local-stage launch (``condense_batch``) that keeps every
request's factors; each then replays the rest of its first solve and its further
sources on its own stream.  Work of different slots overlaps on the device.  The
host loop polls the slots' completion events, checks every status and records
arrival, admission and completion times.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .darcy import PRECISIONS, CartesianQ1Plan
from .errors import LinearSolveError
from .topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

MAX_SOURCES = 8


@dataclass
class DarcyRequest:
    """One serving request: unit-square macro grid ``macro`` x ``macro``, ``refinement``
    x ``refinement`` Q1 cells per macrocell, the fine-cell permeability (shape
    ``(macro*refinement, macro*refinement)``, indexed [x][y]), 1..8 constant sources,
    and its arrival time in seconds after the stream starts."""

    macro: int
    refinement: int
    permeability: np.ndarray
    sources: tuple = (1.0,)
    arrival: float = 0.0
    face_degree: int = 2

    @property
    def shape(self):
        return (int(self.macro), int(self.refinement), int(self.face_degree))


@dataclass
class DarcyResult:
    """Per source: the skeleton unknowns ``x`` (trace, then coarse) and, when the engine
    keeps them, the nodal fields and fine-cell fluxes; plus the request's times."""

    index: int
    x: list
    fields: list | None
    flux: list | None
    arrival: float
    admitted: float
    finished: float
    global_iterations: list = field(default_factory=list)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class _Slot:
    def __init__(self, engine, shape):
        import torch

        macro, refinement, degree = shape
        self.shape = shape
        mesh = CartesianMacroMesh(macro)
        sk = SkeletonSpace(mesh, (FaceSpace.uniform(degree),) * len(mesh.faces))
        self.plan = plan = CartesianQ1Plan(mesh, sk, refinement, precision=engine.precision, device=engine.device)
        nbytes = int(plan.lib.mhm_q1_factor_bytes(plan.q1, PRECISIONS[engine.precision]))
        plan.factors = torch.empty(nbytes, dtype=torch.uint8, device=plan.device)
        n_fine = macro * refinement
        self.kappa = torch.ones((n_fine, n_fine), dtype=torch.float64, device=plan.device)
        self.kappa_host = torch.empty((n_fine, n_fine), dtype=torch.float64).pin_memory()
        self.stream = torch.cuda.Stream(device=plan.device)
        # both steps of a request captured once as CUDA graphs on the slot's stream
        plan.set_device_coefficients(1, self.kappa, (0.0, 0.0, 0.0), 0, None, 1.0)
        plan.capture("offline", stream=self.stream)
        plan.capture("online", stream=self.stream)
        plan.capture("batched", stream=self.stream)
        self.done = torch.cuda.Event()
        pin = dict(dtype=torch.float64)
        self.x_host = [torch.empty(plan.N, **pin).pin_memory() for _ in range(MAX_SOURCES)]
        self.status_host = [torch.empty(plan.cells, dtype=torch.int32).pin_memory() for _ in range(MAX_SOURCES)]
        self.info_host = [torch.empty(4, dtype=torch.int32).pin_memory() for _ in range(MAX_SOURCES)]
        self.stats_host = [torch.empty(4, **pin).pin_memory() for _ in range(MAX_SOURCES)]
        self.fields_host = self.flux_host = None
        if engine.keep_fields:
            self.fields_host = [torch.empty(tuple(plan.fields.shape), **pin).pin_memory() for _ in range(MAX_SOURCES)]
            self.flux_host = [torch.empty(tuple(plan.flux.shape), **pin).pin_memory() for _ in range(MAX_SOURCES)]
        self.bytes = self._device_bytes()
        self.request = None

    def _device_bytes(self) -> int:
        import torch

        seen, total = set(), 0
        for obj in list(vars(self.plan).values()) + [self.kappa]:
            if isinstance(obj, torch.Tensor) and obj.is_cuda and obj.data_ptr() not in seen:
                seen.add(obj.data_ptr())
                total += obj.numel() * obj.element_size()
        return total

    def enqueue(self, index, request, keep_fields):
        import torch

        plan, st = self.plan, self.stream
        self.request = (index, request)
        with torch.cuda.stream(st):
            np.copyto(self.kappa_host.numpy(), request.permeability)
            self.kappa.copy_(self.kappa_host, non_blocking=True)
            for k, src in enumerate(request.sources):
                plan.replay("offline" if k == 0 else "online", float(src), stream=st, after=st)
                self._copy_out(k, keep_fields)
            self.done.record(st)

    def _copy_out(self, k, keep_fields):
        plan = self.plan
        self.x_host[k].copy_(plan.x, non_blocking=True)
        self.status_host[k].copy_(plan.cell_status, non_blocking=True)
        self.info_host[k].copy_(plan.info, non_blocking=True)
        self.stats_host[k].copy_(plan.stats, non_blocking=True)
        if keep_fields:
            self.fields_host[k].copy_(plan.fields, non_blocking=True)
            self.flux_host[k].copy_(plan.flux, non_blocking=True)

    def stage(self, index, request):
        """First half of a batched admission: the permeability upload and the first
        source on this slot's stream; returns the event the batched local stage waits
        for."""
        import torch

        self.request = (index, request)
        with torch.cuda.stream(self.stream):
            np.copyto(self.kappa_host.numpy(), request.permeability)
            self.kappa.copy_(self.kappa_host, non_blocking=True)
            self.plan._graph_source.fill_(float(request.sources[0]))
            ready = torch.cuda.Event()
            ready.record(self.stream)
        return ready

    def finish(self, local_done, keep_fields):
        """Second half: after the batched local stage (event ``local_done``), the first
        source's reduction, global solve and reconstruction, then the further sources
        on the kept factors, each followed by its copies to pinned memory."""
        import torch

        plan, st = self.plan, self.stream
        _, request = self.request
        st.wait_event(local_done)
        with torch.cuda.stream(st):
            plan.replay("batched", stream=st, after=st)
            self._copy_out(0, keep_fields)
            for k, src in enumerate(request.sources[1:], start=1):
                plan.replay("online", float(src), stream=st, after=st)
                self._copy_out(k, keep_fields)
            self.done.record(st)

    def collect(self, admitted, finished, keep_fields) -> DarcyResult:
        """The finished request's results; the slot is free again afterwards, also
        when a status check raises."""
        try:
            return self._collect(admitted, finished, keep_fields)
        finally:
            self.request = None

    def _collect(self, admitted, finished, keep_fields) -> DarcyResult:
        from . import _lib

        index, request = self.request
        xs, fields, flux, iters = [], [] if keep_fields else None, [] if keep_fields else None, []
        for k in range(len(request.sources)):
            status = self.status_host[k].numpy()
            bad = np.flatnonzero(status)
            if len(bad):
                raise LinearSolveError(f"request {index}: {_lib.CELL_MESSAGES.get(int(status[bad[0]]), 'cell failed')}"
                                       f" (macrocell {int(bad[0])})")
            info = self.info_host[k].numpy()
            if info[0] != _lib.SOLVE_OK:
                raise LinearSolveError(f"request {index}: "
                                       f"{_lib.SOLVE_MESSAGES.get(int(info[0]), f'status {info[0]}')}")
            if not self.stats_host[k].numpy()[1] <= 1e-8:
                raise ValueError(f"request {index}: incompatible data: gauge changed physical equations")
            xs.append(self.x_host[k].numpy().copy())
            iters.append(int(info[1]))
            if keep_fields:
                fields.append(self.fields_host[k].numpy().copy())
                flux.append(self.flux_host[k].numpy().copy())
        return DarcyResult(index, xs, fields, flux, request.arrival, admitted, finished, iters)


class ServingEngine:
    """Admit and run ``DarcyRequest`` streams (see the module docstring).

    ``hbm_budget`` bounds the device bytes of all slots together (plans, kept factors,
    permeability buffers); ``max_in_flight`` bounds the requests on the device at
    once; idle slots stay resident for later requests of their shape until the budget
    (or ``max_slots``, if given) needs their room.  ``keep_fields`` also returns every
    source's fields and fluxes (pinned buffers of that size per slot and source).
    ``batch_local`` condenses same-shape requests admitted together in one launch (the
    results are bit-identical either way).  It is off by default: on the mixed request
    streams measured here it lowered throughput by about 4 %, because the batched local
    stage fills every SM at once and the cooperative global solves that follow wait for
    room, where separate launches let them overlap other requests' local stages.
    """

    def __init__(self, *, precision="mixed", hbm_budget=150e9, max_in_flight=8, max_slots=None, keep_fields=False,
                 device=None, batch_local=False):
        import torch

        if precision not in ("mixed", "fp64"):
            raise ValueError("precision must be 'fp64' or 'mixed'")
        if max_in_flight < 1:
            raise ValueError("max_in_flight must be positive")
        self.precision = precision
        self.hbm_budget = float(hbm_budget)
        self.max_in_flight = int(max_in_flight)
        self.max_slots = None if max_slots is None else max(int(max_slots), self.max_in_flight)
        self.keep_fields = bool(keep_fields)
        self.device = torch.device("cuda" if device is None else device)
        self.batch_local = bool(batch_local)
        self._batch_stream = None
        self.slots: list[_Slot] = []
        self._shape_bytes: dict = {}
        self.stats: dict = {}

    def _bytes(self) -> int:
        return sum(s.bytes for s in self.slots)

    def _slot_for(self, shape):
        """An idle slot of ``shape``, or a new one if the in-flight limit and the HBM
        budget allow it after releasing idle slots of other shapes (oldest first);
        None if the request has to wait."""
        for s in self.slots:
            if s.request is None and s.shape == shape:
                return s
        if sum(1 for s in self.slots if s.request is not None) >= self.max_in_flight:
            return None
        need = self._shape_bytes.get(shape, 0)
        if need > self.hbm_budget:
            raise ValueError(f"a request of shape {shape} needs {need} device bytes, more than the HBM budget")
        while ((self.max_slots is not None and len(self.slots) >= self.max_slots)
               or self._bytes() + need > self.hbm_budget):
            idle = [s for s in self.slots if s.request is None]
            if not idle:
                return None
            self.slots.remove(idle[0])
        slot = _Slot(self, shape)
        self._shape_bytes[shape] = slot.bytes
        if slot.bytes > self.hbm_budget:
            raise ValueError(f"a request of shape {shape} needs {slot.bytes} device bytes, more than the HBM budget")
        if self._bytes() + slot.bytes > self.hbm_budget:
            return None  # first slot of this shape, now measured: idle slots make room on the next try
        self.slots.append(slot)
        self.stats["slots_created"] = self.stats.get("slots_created", 0) + 1
        self.stats["peak_bytes"] = max(self.stats.get("peak_bytes", 0), self._bytes())
        return slot

    def reserve(self, shape, count=1) -> int:
        """Create idle slots for ``shape`` (macro, refinement, face degree) until there are
        ``count`` of them or the budget is reached, so that later requests do not pay
        for plan construction and graph capture; returns the slots of that shape."""
        shape = tuple(int(v) for v in shape)
        have = [s for s in self.slots if s.shape == shape]
        while len(have) < count:
            need = self._shape_bytes.get(shape, 0)
            if (self.max_slots is not None and len(self.slots) >= self.max_slots) or \
                    self._bytes() + need > self.hbm_budget:
                break
            slot = _Slot(self, shape)
            self._shape_bytes[shape] = slot.bytes
            if self._bytes() + slot.bytes > self.hbm_budget:
                break
            self.slots.append(slot)
            have.append(slot)
            self.stats["slots_created"] = self.stats.get("slots_created", 0) + 1
            self.stats["peak_bytes"] = max(self.stats.get("peak_bytes", 0), self._bytes())
        return len(have)

    def _launch_admitted(self, admitted, requests):
        """Enqueue the requests admitted in one pass of the loop.  Requests of one shape
        admitted together share one local-stage launch (``condense_batch``, up to 16 at
        a time, each keeping its cells' factors for its further sources); the rest of
        each request runs on its own slot's stream."""
        import torch

        from .darcy import condense_batch

        for group in _groups(admitted):
            for start in range(0, len(group), 16):
                part = group[start:start + 16]
                if not self.batch_local or len(part) < 2:
                    for slot, idx in part:
                        slot.enqueue(idx, requests[idx], self.keep_fields)
                    continue
                if self._batch_stream is None:
                    self._batch_stream = torch.cuda.Stream(device=self.device)
                bs = self._batch_stream
                for slot, idx in part:
                    bs.wait_event(slot.stage(idx, requests[idx]))
                condense_batch([slot.plan for slot, _ in part], offline=True, stream=bs)
                done = torch.cuda.Event()
                done.record(bs)
                for slot, _ in part:
                    slot.finish(done, self.keep_fields)
                self.stats["batched_local_launches"] = self.stats.get("batched_local_launches", 0) + 1
                self.stats["batched_requests"] = self.stats.get("batched_requests", 0) + len(part)

    def run(self, requests, *, realtime=True) -> list[DarcyResult]:
        """Serve ``requests`` (arrival times relative to the call) and return their
        results in request order.  With ``realtime`` a request is not admitted
        before its arrival time; without it every request is available at once."""
        for r in requests:
            if not 1 <= len(r.sources) <= MAX_SOURCES:
                raise ValueError(f"a request carries 1 to {MAX_SOURCES} sources")
            n_fine = r.macro * r.refinement
            if np.shape(r.permeability) != (n_fine, n_fine):
                raise ValueError(f"permeability must have shape ({n_fine}, {n_fine})")
        order = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
        pending = deque(order)
        queue: deque = deque()
        running: list = []
        results: list = [None] * len(requests)
        admit: list = []
        peak = 0
        t0 = time.perf_counter()
        while pending or queue or running:
            now = time.perf_counter() - t0
            while pending and (not realtime or requests[pending[0]].arrival <= now):
                queue.append(pending.popleft())
            for item in list(running):
                slot, admitted = item
                if slot.done.query():
                    finished = time.perf_counter() - t0
                    res = slot.collect(admitted, finished, self.keep_fields)
                    if not realtime:
                        res.arrival = 0.0
                    results[res.index] = res
                    running.remove(item)
            while queue:
                idx = queue[0]
                slot = self._slot_for(requests[idx].shape)
                if slot is None and not running:
                    # nothing on the device: all slots are idle and can be released
                    slot = self._slot_for(requests[idx].shape)
                    if slot is None:
                        raise RuntimeError(f"request {idx} cannot be admitted within the HBM budget")
                if slot is None:
                    break
                queue.popleft()
                admitted = time.perf_counter() - t0
                slot.request = (idx, requests[idx])  # taken: the next admission needs another slot
                admit.append((slot, idx))
                running.append((slot, admitted))
                peak = max(peak, len(running))
            self._launch_admitted(admit, requests)
            admit.clear()
            if running or queue:
                time.sleep(2e-5)
            elif pending:
                time.sleep(max(0.0, min(1e-3, requests[pending[0]].arrival - (time.perf_counter() - t0))))
        self.stats["peak_in_flight"] = max(self.stats.get("peak_in_flight", 0), peak)
        return results


def _groups(admitted):
    """Admitted (slot, index) pairs grouped by request shape, in admission order."""
    out: dict = {}
    for slot, idx in admitted:
        out.setdefault(slot.shape, []).append((slot, idx))
    return list(out.values())


def summarize(results) -> dict:
    """Throughput and latency of one served stream."""
    lat = np.array([r.latency for r in results]) * 1e3
    start = min(r.arrival for r in results)
    end = max(r.finished for r in results)
    rhs = sum(len(r.x) for r in results)
    return {"requests": len(results), "rhs": rhs, "seconds": end - start,
            "requests_per_s": len(results) / (end - start), "rhs_per_s": rhs / (end - start),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())}}
