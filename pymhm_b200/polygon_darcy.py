"""Primal P2 (and mixed RT0 / P0) Darcy on polygonal macro meshes (config 3), on the GPU.

GPU counterpart of ``solve_darcy`` (PyMHM 1.3.2, ``src/pymhm/_legacy/models/darcy/
primal.py:173-344``) for degree-two local spaces on every macrocell's own refinement
(``PolygonMesh.submesh``, uneven sizes), one ``FaceSpace`` per polygon edge, homogeneous
Dirichlet data, a constant source and a constant or disc-inclusion permeability.

Local problems differ in size, so cells are binned by their augmented size rounded up
to ``bin_width``: each bin is one launch of the dense kernels with uniform strides, the
cells padded with an identity block (their solution is zero there).  One solve:

1. ``mhm_p2_assemble``: P2 element operators and the dense rows of every cell;
2. per bin: ``mhm_dense_systems`` (local contract, constraint M 1 / 1^T M 1 as the 2D
   driver normalises it), ``mhm_batched_factor`` / ``mhm_batched_solve`` (checked
   equilibrated LU), ``mhm_dense_contributions`` (tensor-core products);
3. ``mhm_skeleton_scatter`` (ordered, ragged blocks) and ``mhm_general_solve``;
4. per bin: ``mhm_dense_reconstruct``.

Cells above augmented order 640 (the large tier) take, per workspace chunk,
``mhm_p2_assemble_rows``, ``mhm_dense_systems_ragged``, ``mhm_batched_factor_large``
and ``mhm_batched_solve_large`` in step 2.

The mixed formulation (``formulation="mixed"``) replaces step 1 by ``mhm_rt0_elements``
and ``mhm_p2_assemble_rows`` and the dense calls by ``mhm_mixed_systems``,
``mhm_mixed_contributions`` and ``mhm_mixed_reconstruct`` (declared kernel zero on the
fluxes; blocks and loads negated, which leaves the solution unchanged and the trace
block positive semi-definite for the global PCG).
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .errors import LinearSolveError
from .general import GeneralSkeleton
from .polygon import EdgeSkeleton, PolygonMesh, check_rt0_skeleton, local_data, p2_nodal_space
from .topology import block_offsets, skeleton_pattern_ragged, transpose_slots
from .workloads import DiscInclusions

MAX_AUGMENTED = 640  # the batched LU's blocked shared-memory panel (small tier)
LARGE_MAX = 4096  # the large-order LU in HBM (large tier)


def triangle_rule(order: int):
    """``triangle_quadrature`` (``fem/scalar/operators.py:63-69``): Duffy-product Gauss
    points (barycentric) and weights summing to one."""
    t, w = np.polynomial.legendre.leggauss(order)
    t, w = (t + 1) / 2, w / 2
    bary = np.array([(1 - a - (1 - a) * b, a, (1 - a) * b) for a in t for b in t])
    weights = np.array([2 * wa * wb * (1 - a) for a, wa in zip(t, w) for wb in w])
    return bary, weights


def disc_grid(field: DiscInclusions, grid: int = 64):
    """Cell lists of the discs over a grid x grid partition of the unit square: every
    disc is listed in each cell its bounding box meets."""
    lists = [[] for _ in range(grid * grid)]
    for d, ((cx, cy), r) in enumerate(zip(field.centres, field.radii)):
        x0, x1 = np.clip([(cx - r) * grid, (cx + r) * grid], 0, grid - 1).astype(int)
        y0, y1 = np.clip([(cy - r) * grid, (cy + r) * grid], 0, grid - 1).astype(int)
        for gx in range(x0, x1 + 1):
            for gy in range(y0, y1 + 1):
                lists[gx * grid + gy].append(d)
    ptr = np.r_[0, np.cumsum([len(l) for l in lists])].astype(np.int32)
    flat = np.array([d for l in lists for d in l], dtype=np.int32)
    return ptr, flat if len(flat) else np.zeros(1, np.int32)


def p2_size(mesh: PolygonMesh, cell: int, r: int) -> int:
    """P2 unknowns of ``mesh.submesh(cell, r)``: 1 + m r (2 r + 1) for a fan of m
    triangles around the cell's centroid (every convex cell), else counted."""
    _, base = mesh.base_triangles(cell)
    centre = len(base)
    if np.all(base[:, 2] == centre) and len(base) == len(mesh.cells[cell]):
        return 1 + len(base) * r * (2 * r + 1)
    return len(p2_nodal_space(mesh.submesh(cell, r))[1])


def refinement_for_sizes(mesh: PolygonMesh, lo: int = 200, hi: int = MAX_AUGMENTED - 1, seed: int = 0):
    """Per-cell subdivision counts for P2 sizes drawn uniformly in [lo, hi]: for each
    cell's target size, the largest count whose local space stays within it (at least 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.empty(len(mesh.cells), dtype=np.int64)
    for c in range(len(mesh.cells)):
        target = rng.uniform(lo, hi)
        r = 1
        while p2_size(mesh, c, r + 1) <= target:
            r += 1
        out[c] = r
    return out


@dataclass
class PolygonSolution:
    trace: np.ndarray
    coarse: np.ndarray
    fields: list  # per cell, its P2 nodal values
    residual: float
    corrected: np.ndarray
    global_iterations: int
    outer_corrections: int
    seconds: float = 0.0


class PolygonP2Plan:
    """Device-resident plan of one polygonal problem shape (mesh, skeleton, per-cell
    refinement): local meshes, couplings, bins, sparsity and every buffer.

    Local P2 spaces up to 639 unknowns form the small tier (every dense matrix
    resident, ragged launches of the shared-memory-panel LU); larger ones, up to 4095,
    the large tier: their dense matrices pass through a workspace of
    ``workspace_bytes`` (default: the smaller of 112 GiB and 60 % of free device
    memory) in chunks, largest first, factored by the windowed-pivot LU in HBM.
    ``workers`` spawned processes build the cells' local meshes and couplings on the
    host (1: in this process).

    ``formulation="mixed"`` condenses the mixed RT0 / P0 local problems of the same
    cells instead (``_DarcyLocalFactory``'s mixed branch, ``primal.py:80-103``: fine-face
    fluxes, fine-cell pressures and boundary multipliers, the declared kernel zero on
    the fluxes and one on the rest, the skeleton a degree-zero ``FaceSpace`` aligned
    with every cell's fine edges); its saddle systems take the small tier only (order
    up to 639, full partial pivoting)."""

    def __init__(self, mesh: PolygonMesh, skeleton: EdgeSkeleton | None = None, refinements=2, *, order=4,
                 bin_width=32, streams=4, ragged=True, device=None, global_rtol=1e-13, inner_rtol=1e-10,
                 max_inner=20000, max_outer=16, preconditioner="cell", workspace_bytes=None, workers=1,
                 formulation="primal"):
        import torch

        self.torch = torch
        self.lib = _lib.lib()
        self.device = torch.device("cuda" if device is None else device)
        self.mesh = mesh
        self.skeleton = EdgeSkeleton(mesh) if skeleton is None else skeleton
        self.global_rtol, self.inner_rtol = float(global_rtol), float(inner_rtol)
        self.max_inner, self.max_outer = int(max_inner), int(max_outer)
        if preconditioner not in ("cell", "face"):
            raise ValueError("preconditioner must be 'cell' (the cells' D S^-1 D) or 'face' (face blocks)")
        self.preconditioner = preconditioner
        if formulation not in ("primal", "mixed"):
            raise ValueError("formulation must be 'primal' or 'mixed'")
        self.mixed = formulation == "mixed"
        M = len(mesh.cells)
        self.M = M
        rs = np.broadcast_to(np.asarray(refinements, dtype=np.int64), (M,))
        sk = self.skeleton
        if self.mixed:
            check_rt0_skeleton(sk, rs)
        self.T, self.N = sk.size, sk.size + M
        data = local_data(mesh, sk, rs, workers=int(workers), formulation=formulation)
        fines = [f for f, _, _ in data]
        spaces = [sp for _, sp, _ in data]
        self.n_cells = np.array([len(sp[-1]) for sp in spaces], dtype=np.int64)
        cell_dofs = [sk.cell_dofs(c) for c in range(M)]
        self.t_cells = np.array([len(d) for d in cell_dofs], dtype=np.int64)
        if self.n_cells.max() + 1 > LARGE_MAX:
            raise NotImplementedError(f"local P2 spaces up to {LARGE_MAX - 1} unknowns on this path")
        if self.mixed and self.n_cells.max() + 1 > MAX_AUGMENTED:
            raise NotImplementedError(f"mixed local problems up to {MAX_AUGMENTED - 1} unknowns on this path")
        # Cells whose augmented systems exceed the small tier's order are condensed in
        # chunks: their dense matrices share one workspace (two halves: the augmented
        # matrix, assembled in place over the stiffness, and the factors, which first
        # hold the mass matrix), so only their responses stay resident.
        self.workspace_bytes = None if workspace_bytes is None else int(workspace_bytes)
        if self.t_cells.max() > 28:
            raise NotImplementedError("at most 28 trace DOFs per cell")
        couplings = [cp for _, _, cp in data]
        self.nodes = int(sum(self.n_cells))
        # ---- skeleton reduction and global solve -------------------------------------
        self.cell_dofs_list = cell_dofs
        self.pattern = skeleton_pattern_ragged(cell_dofs, self.T)
        bofs, lofs = block_offsets(cell_dofs)
        flat_dofs = np.concatenate(cell_dofs)
        dofs_off = np.r_[0, np.cumsum(self.t_cells)][:-1]
        field_off = np.r_[0, np.cumsum(self.n_cells)][:-1]
        self.field_off_h = np.r_[field_off, self.nodes]
        self.general = GeneralSkeleton(cell_dofs, [sk.geometric_constraint(c) for c in range(M)], sk.offsets,
                                       self.T, self.pattern.indptr, self.pattern.indices, device=self.device)
        self._quad = triangle_rule(max(int(order), 4))
        self._fines, self._spaces, self._couplings = fines, spaces, couplings
        self._offsets = (bofs, lofs, flat_dofs, dofs_off, field_off)
        self.field = None
        self.source = 0.0
        self.streams = max(1, int(streams))
        self.ragged = bool(ragged)
        self._layout(int(bin_width))

    def _layout(self, bin_width: int):
        """Bins by padded augmented size (n + 1 rounded up to a multiple of ``bin_width``),
        the flattened elements and node incidences in bin order, and every buffer whose
        layout follows the bins."""
        torch = self.torch
        M, dev = self.M, self.device
        fines, spaces, couplings = self._fines, self._spaces, self._couplings
        bofs, lofs, flat_dofs, dofs_off, field_off = self._offsets
        qbary, qw = self._quad
        f64 = dict(dtype=torch.float64, device=dev)

        def up(a, dtype):
            return torch.as_tensor(np.array(a, order="C", copy=True), dtype=dtype).to(dev)

        self.bin_width = bin_width
        # ---- bins by padded augmented size -------------------------------------------
        nb_c = ((self.n_cells + 1 + bin_width - 1) // bin_width) * bin_width
        small_c = self.n_cells + 1 <= MAX_AUGMENTED
        nb_c = np.where(small_c, np.minimum(nb_c, MAX_AUGMENTED), np.minimum(nb_c, LARGE_MAX))
        order_cells = np.argsort(nb_c, kind="stable")
        self.order = order_cells
        self.bins = []
        dense_base = rhs_base = cpl_base = load_base = act_base = vec_base = 0
        pos = 0
        for nb in np.unique(nb_c):
            members = order_cells[nb_c[order_cells] == nb]
            k = len(members)
            tld = int(self.t_cells[members].max())
            w = tld + 2
            large = bool(nb > MAX_AUGMENTED or not small_c[members].all())
            self.bins.append(dict(nb=int(nb), tld=tld, w=w, k=k, cells=members, pos=pos, dense=dense_base,
                                  rhs=rhs_base, cpl=cpl_base, load=load_base, act=act_base, vec=vec_base,
                                  large=large))
            if not large:
                dense_base += k * nb * nb
            rhs_base += k * nb * w
            cpl_base += k * nb * tld
            load_base += k * nb
            act_base += k * 3 * nb
            vec_base += k * nb
            pos += k
        # ---- flattened elements and node incidences (cells in bin order) -------------
        pts, tris, edofs, node_cell, node_row, inc_ptr, incs = [], [], [], [], [], [0], []
        rt_info, kvec_parts, kfield_parts = [], [], []
        dense_off = np.empty(M, dtype=np.int64)
        load_off = np.empty(M, dtype=np.int64)
        ld_of = np.empty(M, dtype=np.int32)
        p_base = e_base = 0
        for b in self.bins:
            for j, c in enumerate(b["cells"]):
                fine = fines[c]
                dofs = spaces[c][0]
                valid = spaces[c][1] if self.mixed else np.ones(dofs.shape, dtype=bool)
                slot = b["pos"] + j
                dense_off[slot] = b["dense"] + j * b["nb"] * b["nb"]  # large tier: set per chunk below
                load_off[slot] = b["load"] + j * b["nb"]
                ld_of[slot] = b["nb"]
                pts.append(fine.points)
                tris.append(fine.cells + p_base)
                edofs.append(dofs.astype(np.int32))
                n = int(self.n_cells[c])
                flat = dofs[valid]
                code = ((e_base + np.arange(len(dofs)))[:, None] * 6 + np.arange(6)[None, :])[valid]
                srt = np.lexsort((code, flat))
                counts = np.bincount(flat, minlength=n)
                incs.append(code[srt])
                if self.mixed:
                    rt_info.append(spaces[c][2])
                    z = spaces[c][3]
                    kvec_parts.append(np.r_[z, np.zeros(b["nb"] - n)])
                    kfield_parts.append((c, z))
                inc_ptr.extend((inc_ptr[-1] + np.cumsum(counts)).tolist())
                node_cell.append(np.full(n, slot, dtype=np.int32))
                node_row.append(np.arange(n, dtype=np.int32))
                p_base += len(fine.points)
                e_base += len(dofs)
        self.elements = e_base
        node_ptr = np.r_[0, np.cumsum(self.n_cells[self.order])]
        # ---- large tier: chunks of consecutive slots (largest first) whose dense
        # matrices fit one half of the workspace; their dense offsets are chunk-relative
        large_bins = [b for b in self.bins if b["large"]]
        self.chunks = []
        ws_half = 0
        if large_bins:
            need = sum(b["k"] * b["nb"] * b["nb"] for b in large_bins)
            budget = self.workspace_bytes
            if budget is None:
                free, _ = torch.cuda.mem_get_info(dev)
                budget = min(112 << 30, int(0.6 * free))
            half = max(budget // 16, max(b["nb"] for b in large_bins) ** 2)  # doubles per half
            cur = None
            for b in reversed(large_bins):
                for j in reversed(range(b["k"])):
                    size = b["nb"] * b["nb"]
                    if cur is None or cur["used"] + size > half:
                        cur = dict(used=0, slots=[])
                        self.chunks.append(cur)
                    cur["slots"].append((b, j))
                    cur["used"] += size
            for ch in self.chunks:
                ws_half = max(ws_half, ch["used"])
                # ascending slots at ascending offsets, so that a bin's cells in a chunk
                # sit at the bin's stride from one another
                off, placed = 0, []
                for b, j in reversed(ch["slots"]):
                    dense_off[b["pos"] + j] = off
                    placed.append((b, j, off))
                    off += b["nb"] * b["nb"]
                ch["slots"] = placed
                s0 = ch["slots"][0][0]["pos"] + ch["slots"][0][1]
                s1 = ch["slots"][-1][0]["pos"] + ch["slots"][-1][1] + 1
                ch["s0"], ch["s1"] = s0, s1
                ch["nodes"] = (int(node_ptr[s0]), int(node_ptr[s1]))
                parts = []
                for b, j, off in ch["slots"]:
                    if parts and parts[-1]["bin"] is b:
                        parts[-1]["j1"] = j + 1
                    else:
                        parts.append(dict(bin=b, j0=j, j1=j + 1, ws=off))
                ch["parts"] = parts
                rec = np.array([(off, b["vec"] + j * b["nb"], b["rhs"] + j * b["nb"] * b["w"], b["nb"], b["w"],
                                 b["pos"] + j, 0) for b, j, off in reversed(ch["slots"])],
                               dtype=[("mat_off", "<i8"), ("vec_off", "<i8"), ("rhs_off", "<i8"), ("n", "<i4"),
                                      ("nrhs", "<i4"), ("slot", "<i4"), ("reserved", "<i4")])
                ch["desc"] = torch.as_tensor(rec.view(np.uint8).copy()).to(dev)
                # the coupling blocks and widths, in the descriptors' order
                ch["cpl_off"] = torch.as_tensor(np.array([b["cpl"] + j * b["nb"] * b["tld"]
                                                          for b, j, _ in reversed(ch["slots"])], dtype=np.int64)).to(dev)
                ch["tld_of"] = torch.as_tensor(np.array([b["tld"] for b, _, _ in reversed(ch["slots"])],
                                                        dtype=np.int32)).to(dev)
                ch["count"] = len(rec)
                ch["max_n"] = int(rec["n"].max())
                ch["max_w"] = int(rec["nrhs"].max())
        self.small_nodes = int(node_ptr[sum(b["k"] for b in self.bins if not b["large"])])
        # per bin-order slot: sizes and output offsets
        o = self.order
        self.d = dict(
            points=up(np.concatenate(pts), torch.float64), tris=up(np.concatenate(tris), torch.int64),
            edofs=up(np.concatenate(edofs), torch.int32), node_cell=up(np.concatenate(node_cell), torch.int32),
            node_row=up(np.concatenate(node_row), torch.int32), inc_ptr=up(np.asarray(inc_ptr), torch.int64),
            inc=up(np.concatenate(incs), torch.int64), dense_off=up(dense_off, torch.int64),
            ld_of=up(ld_of, torch.int32), load_off=up(load_off, torch.int64),
            qbary=up(qbary, torch.float64), qw=up(qw, torch.float64),
            n_of=up(self.n_cells[o], torch.int32), t_of=up(self.t_cells[o], torch.int32),
            block_off=up(bofs[:-1][o], torch.int64), lofs=up(lofs[:-1][o], torch.int64),
            dof_off=up(dofs_off[o], torch.int64), cell_id=up(o, torch.int32), field_off=up(field_off[o], torch.int64),
            flat_dofs=up(flat_dofs, torch.int64),
            slot_ptr=up(self.pattern.slot_ptr, torch.int64), contrib=up(self.pattern.contrib, torch.int64),
            load_ptr=up(self.pattern.load_ptr, torch.int64), load_contrib=up(self.pattern.load_contrib, torch.int64),
            indptr=up(self.pattern.indptr, torch.int64), indices=up(self.pattern.indices, torch.int32))
        if self.mixed:
            # the declared kernels: in the load's layout (bin order, padded to each
            # bin's order) and in the fields' layout (cell order)
            self.d["rt_info"] = up(np.concatenate(rt_info), torch.int32)
            self.d["kvec"] = up(np.concatenate(kvec_parts), torch.float64)
            kf = np.empty(self.nodes)
            for c, z in kfield_parts:
                kf[self.field_off_h[c]: self.field_off_h[c + 1]] = z
            self.d["kfield"] = up(kf, torch.float64)
        cpl = np.zeros(cpl_base)
        for b in self.bins:
            for j, c in enumerate(b["cells"]):
                base = b["cpl"] + j * b["nb"] * b["tld"]
                B = couplings[c]
                view = cpl[base: base + b["nb"] * b["tld"]].reshape(b["nb"], b["tld"])
                view[: B.shape[0], : B.shape[1]] = B
        self.d["coupling"] = up(cpl, torch.float64)
        self.elem = torch.empty(int(self.lib.mhm_p2_element_bytes(self.elements)) // 8, **f64)
        self.stiffness = torch.empty(dense_base, **f64)
        self.mass = torch.empty(dense_base, **f64)
        self.load = torch.empty(load_base, **f64)
        self.aug = torch.empty(dense_base, **f64)
        self.factors = torch.empty(dense_base, **f64)
        self.ws_aug = torch.empty(ws_half, **f64) if ws_half else None
        self.ws_factors = torch.empty(ws_half, **f64) if ws_half else None
        self.large_work = torch.empty(66 * vec_base, **f64) if ws_half else None
        self.rhs = torch.empty(rhs_base, **f64)
        self.solution = torch.empty(rhs_base, **f64)
        self.work = torch.empty(rhs_base, **f64)
        self.action = torch.empty(act_base, **f64)
        self.pivots = torch.empty(vec_base, dtype=torch.int32, device=dev)
        self.row_scale = torch.empty(vec_base, **f64)
        self.col_scale = torch.empty(vec_base, **f64)
        self.corrected = torch.empty(M, dtype=torch.uint8, device=dev)
        self.cell_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.bin_streams = [torch.cuda.Stream(device=dev) for _ in range(min(self.streams, len(self.bins)))]
        # one ragged descriptor per cell for the single-launch factor and solve, the
        # largest systems first (CTAs start in this order)
        desc = []
        for b in reversed([b for b in self.bins if not b["large"]]):
            nb, w = b["nb"], b["w"]
            for j in range(b["k"]):
                desc.append((b["dense"] + j * nb * nb, b["vec"] + j * nb, b["rhs"] + j * nb * w, nb, w, b["pos"] + j, 0))
        rec = np.array(desc, dtype=[("mat_off", "<i8"), ("vec_off", "<i8"), ("rhs_off", "<i8"), ("n", "<i4"),
                                    ("nrhs", "<i4"), ("slot", "<i4"), ("reserved", "<i4")])
        self.d_ragged = torch.as_tensor(rec.view(np.uint8).copy()).to(dev) if desc else None
        self.ragged_count = len(desc)
        self.ragged_max_n = int(max([b["nb"] for b in self.bins if not b["large"]], default=0))
        self.ragged_max_nrhs = int(max([b["w"] for b in self.bins if not b["large"]], default=0))
        self.factor_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.solve_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.blocks = torch.empty(int(bofs[-1]), **f64)
        self.loads = torch.empty(int(lofs[-1]), **f64)
        self.values = torch.empty(len(self.pattern.indices), **f64)
        self.grhs = torch.empty(self.N, **f64)
        self.load_scale = torch.empty(self.N, **f64)
        self.d_boundary = torch.zeros(self.T, **f64)
        self.x = torch.empty(self.N, **f64)
        self.fields = torch.empty(self.nodes, **f64)

    def autotune(self, permeability=1.0, source=0.0, *, widths=(16, 32, 64, 128), streams=(1, 4),
                 ragged=(True, False), repeats=2, cache=None):
        """Choose the bin width, the number of bin streams and whether the bins' LU
        factorizations and checked solves run as one ragged launch each, by timing the
        local stage (CUDA events, after one warm-up launch per candidate) on this
        device; keep the fastest layout and return the choice with every timing.
        ``cache``: a JSON file recording choices per device and size signature
        (``autotune.choose``)."""
        from . import autotune as at

        torch = self.torch
        self.set_coefficients(permeability, source)
        cands = [(int(w), int(k), bool(g)) for w in widths for k in streams for g in ragged
                 if int(w) >= 8 and int(k) >= 1]

        def apply(c):
            w, k, g = c
            self.ragged = bool(g)
            if (w, k) != (self.bin_width, self.streams):
                self.streams = k
                self._layout(w)

        def measure(c):
            apply(c)
            st = torch.cuda.current_stream()
            self.launch(st)
            times = []
            for _ in range(repeats):
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
                self.launch(st, events=ev)
                torch.cuda.synchronize()
                times.append(ev[0].elapsed_time(ev[1]))
            self.check()
            return float(np.median(times))

        key = at.shape_key(torch.cuda.get_device_name(self.device), self.n_cells, self.t_cells)
        best, info = at.choose(cands, measure, key=key, cache=cache)
        apply(tuple(best))
        return {"bin_width": self.bin_width, "streams": self.streams, "ragged": self.ragged, **info}

    def set_coefficients(self, permeability=1.0, source=0.0):
        """A ``DiscInclusions`` field or a positive constant permeability; a constant source."""
        torch = self.torch
        if isinstance(permeability, DiscInclusions):
            ptr, flat = disc_grid(permeability)
            self.field = dict(grid=int(np.sqrt(len(ptr) - 1)), ptr=torch.as_tensor(ptr).to(self.device),
                              flat=torch.as_tensor(flat).to(self.device),
                              centres=torch.as_tensor(np.ascontiguousarray(permeability.centres)).to(self.device),
                              r2=torch.as_tensor(np.ascontiguousarray(permeability.r2)).to(self.device),
                              inside=permeability.inside, outside=permeability.outside)
        elif np.ndim(permeability) == 0 and float(permeability) > 0:
            self.field = dict(grid=0, ptr=None, flat=None, centres=None, r2=None, inside=float(permeability),
                              outside=float(permeability))
        else:
            raise NotImplementedError("permeability: DiscInclusions or a positive constant")
        if np.ndim(source) != 0 or not np.isfinite(float(source)):
            raise NotImplementedError("the GPU polygon path takes a constant source")
        self.source = float(source)

    def _bin_views(self, b):
        """Sub-tensors of one bin (contiguous slices of the flat buffers)."""
        k, nb, w, tld = b["k"], b["nb"], b["w"], b["tld"]
        s = slice(b["pos"], b["pos"] + k)
        d = self.d
        dense = None if b["large"] else slice(b["dense"], b["dense"] + k * nb * nb)  # large tier: chunk workspace
        return dict(
            stiffness=None if dense is None else self.stiffness[dense],
            mass=None if dense is None else self.mass[dense],
            aug=None if dense is None else self.aug[dense],
            factors=None if dense is None else self.factors[dense],
            load=self.load[b["load"]: b["load"] + k * nb],
            kvec=self.d["kvec"][b["load"]: b["load"] + k * nb] if self.mixed else None,
            coupling=d["coupling"][b["cpl"]: b["cpl"] + k * nb * tld],
            rhs=self.rhs[b["rhs"]: b["rhs"] + k * nb * w], solution=self.solution[b["rhs"]: b["rhs"] + k * nb * w],
            work=self.work[b["rhs"]: b["rhs"] + k * nb * w], action=self.action[b["act"]: b["act"] + k * 3 * nb],
            pivots=self.pivots[b["vec"]: b["vec"] + k * nb], rs=self.row_scale[b["vec"]: b["vec"] + k * nb],
            cs=self.col_scale[b["vec"]: b["vec"] + k * nb], n_of=d["n_of"][s], t_of=d["t_of"][s],
            block_off=d["block_off"][s], lofs=d["lofs"][s], dof_off=d["dof_off"][s], cell_id=d["cell_id"][s],
            field_off=d["field_off"][s], corrected=self.corrected[s], cell_status=self.cell_status[s],
            factor_status=self.factor_status[s], solve_status=self.solve_status[s])

    def launch(self, stream=None, *, events=None, factor_events=None):
        """Enqueue one complete solve on ``stream`` (no host synchronisation).  ``events``:
        five CUDA events around the local stage, reduction, global solve and reconstruction;
        ``factor_events``: a list that receives a (start, end) pair of CUDA events around
        each large-tier factorization launch."""
        torch = self.torch
        P, lib, sh = _lib.ptr, self.lib, _lib.stream_handle(stream)
        st = torch.cuda.current_stream() if stream is None else stream
        d, fld = self.d, self.field

        def mark(k):
            if events is not None:
                events[k].record(st)

        mark(0)
        if self.mixed:
            _lib.check(lib.mhm_rt0_elements(self.elements, P(d["points"]), P(d["tris"]), P(d["rt_info"]), len(d["qw"]),
                                            P(d["qbary"]), P(d["qw"]), fld["grid"], P(fld["ptr"]), P(fld["flat"]),
                                            P(fld["centres"]), P(fld["r2"]), fld["inside"], fld["outside"],
                                            self.source, P(self.elem), sh), "mhm_rt0_elements")
            self._assemble_rows(0, self.nodes, self.stiffness, self.mass, sh)
        elif not self.chunks:
            _lib.check(lib.mhm_p2_assemble(self.elements, P(d["points"]), P(d["tris"]), len(d["qw"]), P(d["qbary"]),
                                           P(d["qw"]), fld["grid"], P(fld["ptr"]), P(fld["flat"]), P(fld["centres"]),
                                           P(fld["r2"]), fld["inside"], fld["outside"], self.source, P(self.elem),
                                           self.nodes, P(d["node_cell"]), P(d["node_row"]), P(d["inc_ptr"]),
                                           P(d["inc"]), P(d["edofs"]), P(d["dense_off"]), P(d["ld_of"]),
                                           P(d["load_off"]), P(self.stiffness), P(self.mass), P(self.load), sh),
                       "mhm_p2_assemble")
        else:
            _lib.check(lib.mhm_p2_elements(self.elements, P(d["points"]), P(d["tris"]), len(d["qw"]), P(d["qbary"]),
                                           P(d["qw"]), fld["grid"], P(fld["ptr"]), P(fld["flat"]), P(fld["centres"]),
                                           P(fld["r2"]), fld["inside"], fld["outside"], self.source, P(self.elem),
                                           sh), "mhm_p2_elements")
            if self.small_nodes:
                self._assemble_rows(0, self.small_nodes, self.stiffness, self.mass, sh)
        small = [b for b in self.bins if not b["large"]]
        # the bins' chains are independent until the scatter: fork them over side
        # streams (largest bins first) so that one bin's last wave overlaps the next's.
        # With ``ragged`` the factorizations and the checked solves of all bins run as
        # one launch each (ragged descriptors) between a forked system stage and a
        # forked contribution stage.
        def forked(stage, bins):
            if not bins:
                return
            fork = torch.cuda.Event()
            fork.record(st)
            used = []
            for idx, b in enumerate(reversed(bins)):
                bs = self.bin_streams[idx % len(self.bin_streams)]
                if idx < len(self.bin_streams):
                    bs.wait_event(fork)
                    used.append(bs)
                stage(b, self._bin_views(b), bs, _lib.stream_handle(bs))
            for bs in used:
                join = torch.cuda.Event()
                join.record(bs)
                st.wait_event(join)

        def systems(b, v, bs, shb):
            if self.mixed:
                _lib.check(lib.mhm_mixed_systems(b["k"], b["nb"], b["tld"], b["nb"], b["w"], P(v["n_of"]),
                                                 P(v["t_of"]), P(v["stiffness"]), P(v["mass"]), P(v["load"]),
                                                 P(v["coupling"]), P(v["kvec"]), P(v["aug"]), P(v["rhs"]),
                                                 P(v["action"]), P(v["corrected"]), P(v["cell_status"]), shb),
                           "mhm_mixed_systems")
                return
            _lib.check(lib.mhm_dense_systems(b["k"], b["nb"], b["tld"], b["nb"], b["w"], 1, P(v["n_of"]), P(v["t_of"]),
                                             P(v["stiffness"]), P(v["mass"]), P(v["load"]), P(v["coupling"]),
                                             P(v["aug"]), P(v["rhs"]), P(v["action"]), P(v["corrected"]),
                                             P(v["cell_status"]), shb), "mhm_dense_systems")

        def factor_solve(b, v, bs, shb):
            k, nb, w = b["k"], b["nb"], b["w"]
            _lib.check(lib.mhm_batched_factor(k, nb, P(v["aug"]), P(v["factors"]), P(v["pivots"]), P(v["rs"]),
                                              P(v["cs"]), P(v["factor_status"]), shb), "mhm_batched_factor")
            with torch.cuda.stream(bs):
                v["solve_status"].copy_(v["factor_status"])
            _lib.check(lib.mhm_batched_solve(k, nb, w, P(v["aug"]), P(v["factors"]), P(v["pivots"]), P(v["rs"]),
                                             P(v["cs"]), P(v["rhs"]), P(v["solution"]), P(v["work"]), 1e-10, 0.0,
                                             2, P(v["solve_status"]), shb), "mhm_batched_solve")

        def contributions(b, v, bs, shb):
            if self.mixed:
                _lib.check(lib.mhm_mixed_contributions(b["k"], b["nb"], b["tld"], b["nb"], b["w"], b["tld"],
                                                       P(v["n_of"]), P(v["t_of"]), P(v["solution"]),
                                                       P(v["coupling"]), P(v["action"]), P(v["load"]), P(v["kvec"]),
                                                       P(v["block_off"]), P(v["lofs"]), P(self.blocks),
                                                       P(self.loads), shb), "mhm_mixed_contributions")
                return
            _lib.check(lib.mhm_dense_contributions(b["k"], b["nb"], b["tld"], b["nb"], b["w"], b["tld"],
                                                   P(v["n_of"]), P(v["t_of"]), P(v["solution"]), P(v["coupling"]),
                                                   P(v["action"]), P(v["load"]), P(v["block_off"]), P(v["lofs"]),
                                                   P(self.blocks), P(self.loads), shb), "mhm_dense_contributions")

        if self.ragged:
            forked(systems, small)
            cnt = self.ragged_count
            if cnt:
                _lib.check(lib.mhm_batched_factor_ragged(cnt, P(self.d_ragged), self.ragged_max_n, P(self.aug),
                                                         P(self.factors), P(self.pivots), P(self.row_scale),
                                                         P(self.col_scale), P(self.factor_status), sh),
                           "mhm_batched_factor_ragged")
                with torch.cuda.stream(st):
                    self.solve_status[:cnt].copy_(self.factor_status[:cnt])
                _lib.check(lib.mhm_batched_solve_ragged(cnt, P(self.d_ragged), self.ragged_max_n,
                                                        self.ragged_max_nrhs, P(self.aug), P(self.factors),
                                                        P(self.pivots), P(self.row_scale), P(self.col_scale),
                                                        P(self.rhs), P(self.solution), 1e-10, 0.0, 2,
                                                        P(self.solve_status), sh), "mhm_batched_solve_ragged")
            self._large_chunks(st, sh, factor_events)
            forked(contributions, self.bins)
        else:
            def chain(b, v, bs, shb):
                systems(b, v, bs, shb)
                factor_solve(b, v, bs, shb)
                contributions(b, v, bs, shb)

            forked(chain, small)
            self._large_chunks(st, sh, factor_events)
            forked(contributions, [b for b in self.bins if b["large"]])
        mark(1)
        p = self.pattern
        _lib.check(lib.mhm_skeleton_scatter(len(p.indices), P(d["slot_ptr"]), P(d["contrib"]), P(self.blocks),
                                            P(self.values), self.N, self.T, P(d["load_ptr"]), P(d["load_contrib"]),
                                            P(self.loads), P(self.d_boundary), P(self.grhs), P(self.load_scale), sh),
                   "mhm_skeleton_scatter")
        mark(2)
        self.general.launch(self.values, self.grhs, self.x, rtol=self.global_rtol, inner_rtol=self.inner_rtol,
                            max_inner=self.max_inner, max_outer=self.max_outer, stream=stream,
                            blocks=self.blocks if self.preconditioner == "cell" else None)
        mark(3)
        for b in self.bins:
            v = self._bin_views(b)
            if self.mixed:
                _lib.check(lib.mhm_mixed_reconstruct(b["k"], b["nb"], b["w"], P(v["n_of"]), P(v["t_of"]),
                                                     P(v["solution"]), P(d["flat_dofs"]), P(v["dof_off"]),
                                                     P(v["cell_id"]), self.T, P(self.x), P(v["field_off"]),
                                                     P(d["kfield"]), P(self.fields), sh), "mhm_mixed_reconstruct")
                continue
            _lib.check(lib.mhm_dense_reconstruct(b["k"], b["nb"], b["w"], P(v["n_of"]), P(v["t_of"]),
                                                 P(v["solution"]), P(d["flat_dofs"]), P(v["dof_off"]),
                                                 P(v["cell_id"]), self.T, P(self.x), P(v["field_off"]),
                                                 P(self.fields), sh), "mhm_dense_reconstruct")
        mark(4)

    def _assemble_rows(self, n0, n1, stiffness, mass, sh):
        """Dense rows of the nodes n0 .. n1 - 1 (bin order) into ``stiffness`` / ``mass``
        at the slots' dense offsets (chunk-relative for the large tier)."""
        P, d = _lib.ptr, self.d
        _lib.check(self.lib.mhm_p2_assemble_rows(n1 - n0, P(d["node_cell"][n0:]), P(d["node_row"][n0:]),
                                                 P(d["inc_ptr"][n0:]), P(d["inc"]), P(d["edofs"]), P(self.elem),
                                                 P(d["dense_off"]), P(d["ld_of"]), P(d["load_off"]), P(stiffness),
                                                 P(mass), P(self.load), sh), "mhm_p2_assemble_rows")

    def _large_chunks(self, st, sh, factor_events=None):
        """The large tier, one chunk after another on ``st``: node rows into the workspace,
        then one ragged launch each of the augmented systems (in place over the
        stiffness), the large-order factorization and the checked solve over the chunk's
        cells (largest first).  The responses land in the resident right-hand-side
        layout."""
        torch, P, lib, d = self.torch, _lib.ptr, self.lib, self.d
        for ch in self.chunks:
            n0, n1 = ch["nodes"]
            self._assemble_rows(n0, n1, self.ws_aug, self.ws_factors, sh)
            # the augmented systems of every cell of the chunk, in place over the
            # stiffness, in one ragged launch (largest first)
            _lib.check(lib.mhm_dense_systems_ragged(ch["count"], P(ch["desc"]), P(ch["cpl_off"]), P(ch["tld_of"]), 1,
                                                    P(d["n_of"]), P(d["t_of"]), P(self.ws_aug), P(self.ws_factors),
                                                    P(self.load), P(d["coupling"]), P(self.ws_aug), P(self.rhs),
                                                    P(self.action), P(self.corrected), P(self.cell_status), sh),
                       "mhm_dense_systems_ragged")
            if factor_events is not None:
                factor_events.append(torch.cuda.Event(enable_timing=True))
                factor_events[-1].record(st)
            _lib.check(lib.mhm_batched_factor_large(ch["count"], P(ch["desc"]), ch["max_n"], P(self.ws_aug),
                                                    P(self.ws_factors), P(self.pivots), P(self.row_scale),
                                                    P(self.col_scale), P(self.factor_status), sh),
                       "mhm_batched_factor_large")
            if factor_events is not None:
                factor_events.append(torch.cuda.Event(enable_timing=True))
                factor_events[-1].record(st)
            with torch.cuda.stream(st):
                self.solve_status[ch["s0"]: ch["s1"]].copy_(self.factor_status[ch["s0"]: ch["s1"]])
            _lib.check(lib.mhm_batched_solve_large(ch["count"], P(ch["desc"]), ch["max_n"], ch["max_w"],
                                                   P(self.ws_aug), P(self.ws_factors), P(self.pivots),
                                                   P(self.row_scale), P(self.col_scale), P(self.rhs),
                                                   P(self.solution), P(self.large_work), 1e-10, 0.0, 2,
                                                   P(self.solve_status), sh), "mhm_batched_solve_large")

    def failed_cells(self) -> np.ndarray:
        """Macrocells (global ids) whose local stage failed the reference's contract
        in the last launch (synchronises)."""
        bad = np.flatnonzero(self.cell_status.cpu().numpy() | self.solve_status.cpu().numpy())
        return np.sort(self.order[bad])

    def check(self):
        """Raise the reference's error for any failed stage (synchronises)."""
        for arr in (self.cell_status, self.solve_status):
            stv = arr.cpu().numpy()
            bad = np.flatnonzero(stv)
            if len(bad):
                raise LinearSolveError(f"{_lib.CELL_MESSAGES.get(int(stv[bad[0]]), 'cell failed')} "
                                       f"(macrocell {int(self.order[bad[0]])})")
        return self.general.check()

    def result(self, seconds=0.0) -> PolygonSolution:
        info, stats = self.check()
        x = self.x.cpu().numpy()
        f = self.fields.cpu().numpy()
        fields = [f[self.field_off_h[c]: self.field_off_h[c + 1]] for c in range(self.M)]
        corrected = np.empty(self.M, dtype=bool)
        corrected[self.order] = self.corrected.cpu().numpy().astype(bool)
        return PolygonSolution(trace=x[: self.T].copy(), coarse=x[self.T:].copy(), fields=fields,
                               residual=float(stats[0]), corrected=corrected, global_iterations=int(info[1]),
                               outer_corrections=int(info[2]), seconds=seconds)

    def solve(self, permeability=1.0, source=0.0, stream=None) -> PolygonSolution:
        t0 = time.perf_counter()
        self.set_coefficients(permeability, source)
        self.launch(stream)
        sol = self.result()
        sol.seconds = time.perf_counter() - t0
        return sol

    def cell_block(self, cell: int) -> np.ndarray:
        """The oriented Schur block of a cell (global cell id), for checks."""
        bofs, _ = block_offsets(self.cell_dofs_list)
        t1 = int(self.t_cells[cell]) + 1
        return self.blocks[int(bofs[cell]): int(bofs[cell]) + t1 * t1].cpu().numpy().reshape(t1, t1)

    def matrix(self):
        """Host copy of the assembled skeleton matrix in the reference's CSC form, exact
        zeros dropped (``core/contributions.py:184-185``)."""
        from scipy import sparse

        torch = self.torch
        p = self.pattern
        if getattr(self, "_csc", None) is None:
            self._csc = dict(transpose=torch.as_tensor(transpose_slots(p.indptr, p.indices)).to(self.device),
                             indptr=torch.empty(self.N + 1, dtype=torch.int64, device=self.device),
                             indices=torch.empty(len(p.indices), dtype=torch.int32, device=self.device),
                             data=torch.empty(len(p.indices), dtype=torch.float64, device=self.device))
        c = self._csc
        P = _lib.ptr
        _lib.check(self.lib.mhm_skeleton_export_csc(self.N, P(self.d["indptr"]), P(self.d["indices"]),
                                                    P(c["transpose"]), P(self.values), P(c["indptr"]),
                                                    P(c["indices"]), P(c["data"]), _lib.stream_handle(None)),
                   "mhm_skeleton_export_csc")
        kept = int(c["indptr"][-1])
        return sparse.csc_matrix((c["data"][:kept].cpu().numpy(), c["indices"][:kept].cpu().numpy(),
                                  c["indptr"].cpu().numpy()), shape=(self.N, self.N))


def solve_darcy(mesh: PolygonMesh, *, permeability=1.0, source=0.0, dirichlet=0.0, neumann=None,
                skeleton: EdgeSkeleton | None = None, local_refinement=4, local_meshes=None, quadrature_order=4,
                formulation="primal", degree=1, **_ignored) -> PolygonSolution:
    """GPU counterpart of ``solve_darcy`` (``primal.py:173-344``) on a ``PolygonMesh`` for
    the primal ``degree=2`` or the mixed RT0 / P0 (``formulation="mixed"``,
    ``degree=1``) formulation, homogeneous Dirichlet data, a constant source and a
    constant or ``DiscInclusions`` permeability.  ``local_refinement`` may be one count
    or one per cell (the uneven local sizes of a polygon batch).  Mixed solutions hold
    each cell's fluxes, pressures and boundary multipliers, in that order."""
    if formulation not in ("primal", "mixed"):
        raise ValueError("formulation must be 'primal' or 'mixed'")
    if formulation == "mixed" and int(degree) != 1:
        raise ValueError("RT0 uses degree=1; higher-order primal locals use formulation=primal")
    if formulation == "primal" and int(degree) != 2:
        raise NotImplementedError("the GPU polygon path implements the primal degree-two formulation")
    if local_meshes is not None or neumann:
        raise NotImplementedError("explicit local meshes and Neumann data are not on the GPU polygon path")
    if np.ndim(dirichlet) != 0 or float(dirichlet) != 0.0:
        raise NotImplementedError("the GPU polygon path takes homogeneous Dirichlet data")
    if formulation == "mixed" and skeleton is None:
        from .topology import FaceSpace

        skeleton = EdgeSkeleton(mesh, FaceSpace.uniform(0))
    plan = PolygonP2Plan(mesh, skeleton, local_refinement, order=max(int(quadrature_order), 4),
                         formulation=formulation)
    return plan.solve(permeability, source)
