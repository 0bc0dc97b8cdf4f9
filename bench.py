#!/usr/bin/env python
"""Primal-MHM solves/s on B200: one JSON line per run.

Workload: 64x64 Cartesian macrocells x 16x16 local Q1 (289 local DOFs),
discontinuous P2 traces per macro edge (12 trace + 1 source right-hand sides
per cell), log-normal permeability (Gaussian log-field, exponential covariance,
sigma = 2, correlation length 0.05, PCG64 seed 20261203) on the 1024x1024 fine
cells, f = 1, homogeneous Dirichlet data.  Synthetic, seeded inputs.

A step is one complete MHM solve: local assembly + condensation, ordered
skeleton reduction, global skeleton solve, reconstruction of fields and
fluxes.  ``value`` is solves/s of a serving loop with the permeability already
resident in HBM: independent requests alternate between two plans, so two
solves are in flight and one request's latency-bound global solve (64 of the
148 SMs, high-priority stream) overlaps the next request's local stage
(low-priority stream).  Mixed precision: binary32 local factors + FP64
refinement; the FP64-factor path is reported beside it, and ``sequential``
gives one-solve-at-a-time latency with the per-kernel split (L2 flushed by a
256 MiB write between those steps, outside the timed region).  ``e2e`` runs
the same serving loop through the public API with the permeability copied
from pinned host memory and fields, fluxes, skeleton unknowns and status
copied back for every request.

``--impl reference`` times the CPU restatement of the reference path (the
oracle) on the host cores instead: each step is one whole solve of the same
workload (the 4096 local problems on a spawn process pool of one BLAS thread
per process, then skeleton assembly, the global SuperLU solve and the
reconstruction of fields and fluxes).

Multi-GPU: replicas only (one independent solve per rank, no collective in
the data path); torch.distributed is used for barriers and the max-over-ranks
timing.  ``--gpus N`` without a torchrun environment starts the N ranks itself.
"""

from __future__ import annotations

import argparse
import csv
import io
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MACRO, LOCAL, FACE_DEGREE = 64, 16, 2
SIGMA, ELL, SEED = 2.0, 0.05, 20261203
METRIC = "MHM solves/s (64x64 Q1 Darcy, lognormal kappa), mixed vs FP64 GPU"
CPU_RUNS, SERIAL_SAMPLE_CELLS = 3, 48
# DRAM bytes per launch of this workload's kernels from one ncu capture each, with the
# command that produced them
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "dram_traffic.json")


def triangle_submesh(r):
    """Uniform refinement of the unit right triangle into r^2 triangles:
    (r+1)(r+2)/2 P1 nodes (91 for r = 12, 325 for r = 24)."""
    nodes = [(i, j) for j in range(r + 1) for i in range(r + 1 - j)]
    index = {p: k for k, p in enumerate(nodes)}
    cells = []
    for j in range(r):
        for i in range(r - j):
            cells.append([index[(i, j)], index[(i + 1, j)], index[(i, j + 1)]])
            if i + j < r - 1:
                cells.append([index[(i + 1, j)], index[(i + 1, j + 1)], index[(i, j + 1)]])
    return np.array(nodes, dtype=float) / r, np.array(cells, dtype=np.int64)


def batched_local_campaign(torch, refinement, batch=64, queries=12, repeats=3):
    """The reference's resident batched local-stage benchmark (``gpu_campaign``,
    benchmarks/execution_modes.py:203-290) with this library's kernels: P1 volume
    assembly of ``batch`` copies of a triangle refined ``refinement`` times, the
    mean-constrained dense systems, batched LU, a first solve of the source and three
    trace columns, ``queries`` repeated right-hand sides, download.  Wall clock per
    phase with a device synchronisation at each boundary, one untimed repetition
    first; median over ``repeats``."""
    from pymhm_b200.batched import BatchedFactorization, assemble_p1_batch

    pts, cells = triangle_submesh(refinement)
    n = len(pts)
    coords = np.repeat(pts[None], batch, axis=0)
    dev = torch.device("cuda")
    diffusion = torch.diag(torch.tensor([3.0, 1.0], dtype=torch.float64, device=dev))
    records, error = [], 0.0
    for rep in range(repeats + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p_dev, c_dev = torch.from_numpy(coords).to(dev), torch.from_numpy(cells).to(dev)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        stiffness, mass, forcing = assemble_p1_batch(p_dev, c_dev, diffusion=diffusion, source=1.0)
        constrained = torch.zeros((batch, n + 1, n + 1), dtype=torch.float64, device=dev)
        constrained[:, :n, :n] = stiffness
        c = mass.sum(dim=2)  # constraint M 1, scaled as the condensation contract scales it
        scale = torch.clamp(stiffness.abs().amax(dim=(1, 2)) / c.abs().amax(dim=1), max=1.0)
        means = c * scale[:, None]
        constrained[:, :n, n] = means
        constrained[:, n, :n] = means
        loads = torch.zeros((batch, n + 1, 4), dtype=torch.float64, device=dev)
        loads[:, :n, 0] = forcing
        loads[:, 0, 1] = loads[:, 1, 2] = loads[:, 2, 3] = 1.0  # coupling = the first three unit columns
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        with BatchedFactorization(constrained) as fact:
            torch.cuda.synchronize()
            t3 = time.perf_counter()
            first = fact.solve(loads)
            torch.cuda.synchronize()
            t4 = time.perf_counter()
            for factor in np.linspace(0.5, 1.5, queries):
                repeated = fact.solve(loads * float(factor))
            torch.cuda.synchronize()
            t5 = time.perf_counter()
            host_first = first[:, :n].cpu().numpy()
            host_last = repeated[:, :n].cpu().numpy()
            torch.cuda.synchronize()
            t6 = time.perf_counter()
        if rep == 0:
            a0 = constrained[0].cpu().numpy()
            want = np.linalg.solve(a0, loads[0].cpu().numpy())[:n]
            error = max(float(np.max(np.abs(host_first[0] - want))),
                        float(np.max(np.abs(host_last[-1] - 1.5 * want))))
        else:
            records.append([t1 - t0, t2 - t1, t3 - t2, t4 - t3, t5 - t4, t6 - t5, t6 - t0])
    med = np.median(np.array(records), axis=0) * 1e3
    keys = ["upload", "assembly_and_constrained_systems", "factorization", "first_solve", "repeated_rhs_total",
            "download", "total"]
    out = {k: float(v) for k, v in zip(keys, med)}
    out.update(batch=batch, local_unknowns=n, queries=queries, max_solution_error_vs_numpy=error)
    return out


SERVING_MACRO = (16, 32, 64)
SERVING_LOCAL = (4, 8, 16)


def small_poisson_campaign(torch, steps=200, warmup=10):
    """The 8x8-macrocell Poisson case (4x4 Q1 cells each, P1 faces, kappa = 1,
    f = 2 pi^2 sin(pi x) sin(pi y), homogeneous Dirichlet): 64 local problems of 25
    unknowns.  Launch- and latency-bound; reported as solves/s back to back and the
    latency of one solve at a time (CUDA events), with the error against the
    reference's FP64 solution of the same case (golden fixture)."""
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import sine_source

    mesh = CartesianMacroMesh(8)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(1),) * len(mesh.faces))
    gpath = os.path.join(ROOT, "tests", "golden", "poisson_8x8_r4_p1.npz")
    g = np.load(gpath) if os.path.exists(gpath) else None
    out = {}
    for prec in ("mixed", "fp64"):
        plan = CartesianQ1Plan(mesh, sk, 4, precision=prec)
        plan.set_coefficients(1.0, sine_source)
        st = torch.cuda.Stream()
        for _ in range(warmup):
            plan.launch(st)
        torch.cuda.synchronize()
        lat = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            plan.launch(st)
            e1.record(st)
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(st)
        for _ in range(steps):
            plan.launch(st)
        t1.record(st)
        torch.cuda.synchronize()
        eager_s = t0.elapsed_time(t1)
        # the same fresh solve captured as one CUDA graph (capture("condense"))
        plan.capture("condense", st)
        glat = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            plan.replay("condense", after=st)
            e1.record(st)
            e1.synchronize()
            glat.append(e0.elapsed_time(e1))
        t0.record(st)
        for _ in range(steps):
            plan.replay("condense", after=st)
        t1.record(st)
        torch.cuda.synchronize()
        sol = plan.result()
        lat, glat = np.array(lat), np.array(glat)
        entry = {"solves_per_s": steps * 1000.0 / t0.elapsed_time(t1), "p50_ms": float(np.percentile(glat, 50)),
                 "p99_ms": float(np.percentile(glat, 99)), "global_iterations": sol.global_iterations,
                 "eager": {"solves_per_s": steps * 1000.0 / eager_s, "p50_ms": float(np.percentile(lat, 50)),
                           "p99_ms": float(np.percentile(lat, 99))}}
        if g is not None:
            rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
            entry["error_vs_reference"] = {"lambda": rel(sol.trace, g["trace"]), "u": rel(sol.fields, g["fields"]),
                                           "flux": rel(sol.flux, g["flux"])}
        out[prec] = entry
    out["note"] = ("8x8 macrocells x 4x4 Q1, P1 faces, sine source; one fresh solve (four kernels) per CUDA graph "
                   "replay (capture('condense')); 'eager': the same solve launched from Python each time")
    return out


def cut_material_campaign(torch, steps=5, pixels=1000):
    """The headline workload's mesh (64x64 macrocells x 16x16 Q1, P2 faces) with a
    log-normal pixel field of pixels x pixels cells (sigma 2, ell 0.05) whose lines cut
    the 1024 x 1024 fine cells: every fine cell is integrated on its exact pixel
    intersections (cut-element pre-pass inside the local stage).  One solve at a time,
    per-kernel CUDA events; mixed against FP64 on the same input."""
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from pymhm_b200.workloads import lognormal_permeability

    class Pixels:
        def __init__(self, values):
            self.values, self.spacing, self.origin = values, (1.0 / pixels, 1.0 / pixels), (0.0, 0.0)

    field = Pixels(lognormal_permeability(pixels, pixels, sigma=SIGMA, ell=ELL, seed=SEED + 1))
    mesh = CartesianMacroMesh(MACRO)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(FACE_DEGREE),) * len(mesh.faces))
    out, fields = {}, {}
    for prec in ("mixed", "fp64"):
        plan = CartesianQ1Plan(mesh, sk, LOCAL, precision=prec)
        plan.set_coefficients(field, 1.0)
        st = torch.cuda.Stream()
        plan.launch(st)
        torch.cuda.synchronize()
        per = []
        for _ in range(steps):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            plan.launch(st, events=ev)
            torch.cuda.synchronize()
            per.append([ev[i].elapsed_time(ev[i + 1]) for i in range(4)])
        sol = plan.result()
        per = np.array(per)
        out[prec] = {"ms_per_solve": float(per.sum(1).mean()),
                     "kernels_ms": {"q1_condense_with_cut_prepass": float(per[:, 0].mean()),
                                    "skeleton_scatter": float(per[:, 1].mean()),
                                    "skeleton_pcg": float(per[:, 2].mean()),
                                    "q1_reconstruct": float(per[:, 3].mean())},
                     "global_iterations": sol.global_iterations, "kappa_mode": int(plan.q1.kappa_mode)}
        fields[prec] = sol.fields
        plan.cut_elements = None
    out["mixed_vs_fp64_fields"] = float(np.linalg.norm(fields["mixed"] - fields["fp64"]) /
                                        np.linalg.norm(fields["fp64"]))
    out["note"] = (f"{pixels}x{pixels} pixel field over the 1024x1024 fine grid (pixel lines cut the fine cells); "
                   "the condense time includes the cut-element pre-pass")
    return out


def tetra_campaign(torch, steps=5, warmup=2, cube=8, local=8, cpu_cells=16, preconditioner="cell"):
    """3D Primal-MHM Darcy (config 4): the unit cube split into cube^3 x 6 macro
    tetrahedra (3072 at cube = 8), each red-refined to local^3 fine tetrahedra (165 P1
    nodes at local = 8), Bernstein P1 modes on every macroface (3 per face: the
    constant and the linear modes), 40 horizontal layers of log-normal permeability
    (sigma 3, correlation length 0.1, contrast 1e6, on 64 x 64 pixels), f = 1,
    homogeneous Dirichlet data, FP64.  One solve at a time with CUDA events per stage;
    the oracle's local stage on a sample of cells in this process beside it."""
    from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
    from pymhm_b200.tetra_darcy import TetraP1Plan
    from pymhm_b200.workloads import LayeredField, layered_lognormal_permeability

    t0 = time.perf_counter()
    mesh = TetraMesh.unit_cube(cube)
    sk = TriangularSkeleton(mesh, 1)
    field = LayeredField(layered_lognormal_permeability(40, 64, sigma=3.0, ell=0.1, contrast=1e6, seed=SEED))
    plan = TetraP1Plan(mesh, sk, local, preconditioner=preconditioner)
    plan.set_coefficients(field, 1.0)
    plan_s = time.perf_counter() - t0
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        plan.launch(st)
    torch.cuda.synchronize()
    plan.check()
    per = []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        plan.launch(st, events=ev)
        torch.cuda.synchronize()
        per.append([ev[k].elapsed_time(ev[k + 1]) for k in range(4)])
    sol = plan.result()
    per = np.array(per)
    ms = float(per.sum(axis=1).mean())
    out = {"solves_per_s": 1000.0 / ms, "ms_per_solve": ms,
           "stages_ms": {"local_stage": float(per[:, 0].mean()), "skeleton_scatter": float(per[:, 1].mean()),
                         "general_pcg": float(per[:, 2].mean()), "reconstruct": float(per[:, 3].mean())},
           "macrocells": plan.M, "local_nodes": plan.n, "trace_per_cell": plan.t, "skeleton_unknowns": plan.N,
           "global_iterations": sol.global_iterations, "outer_corrections": sol.outer_corrections,
           "residual": sol.residual, "preconditioner": preconditioner, "plan_build_s": plan_s}
    if cpu_cells:
        from oracle import tetra_mhm as ot
        from oracle.q1_mhm import condense, contribution

        cells = np.linspace(0, plan.M - 1, cpu_cells).astype(int)
        c0 = time.perf_counter()
        for c in cells:
            _, prob = ot.local_problem(mesh, sk, int(c), local, field, 1.0)
            contribution(condense(prob), sk.size + int(c))
        rate = len(cells) / (time.perf_counter() - c0)
        out["cpu_oracle_local_cells_per_s"] = {"value": rate, "cores": 1, "sample": f"{len(cells)} of {plan.M} "
                                               "macrocells, local operators + condensation + contribution"}
    del plan
    torch.cuda.empty_cache()
    return out


def dgemm_peak(torch, n=8192, reps=5):
    """cuBLAS FP64 GEMM throughput on this GPU (TFLOP/s, best of ``reps``): the
    denominator of the FP64 tensor-core kernels' roofline."""
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def polygon_campaign(torch, steps=3, warmup=1, count=2000, cpu_cells=8, preconditioner="cell", inside=30.0,
                     contract_inside=1e4, lo=200, hi=3000):
    """Polygonal P2 Darcy (config 3): the Voronoi cells of 2000 seeded points in the unit
    square, each refined with the largest subdivision count whose P2 space stays within
    a size drawn uniformly in [lo, hi] = [200, 3000], one Legendre P1 face space per edge
    (4-10 edges, 8-20 trace DOFs per cell), 300 seeded discs of radius 0.01-0.03 with
    permeability ``inside`` in a background of 1, f = 1, homogeneous Dirichlet data,
    FP64.  Augmented orders up to 640 run in the small tier (ragged launches of the
    shared-memory-panel LU), larger ones in the large tier (chunks of the windowed-pivot
    LU in HBM).  One solve at a time with CUDA events per stage; the oracle's local
    stage on a sample of cells in this process beside it.

    At the configuration's contrast of 1e4 the reference's own local solves fail its
    columnwise 1e-10 residual test on some of these cells (the same contract here), so
    no solution exists to time; the campaign counts the cells that fail at
    ``contract_inside`` and times the solve at ``inside`` = 30, where every cell passes
    (the oracle's local stage raises on 71 cells at 1e4, 9 at 1e3, 3 at 1e2, none at 30)."""
    from pymhm_b200.polygon import EdgeSkeleton, voronoi_mesh
    from pymhm_b200.polygon_darcy import PolygonP2Plan, refinement_for_sizes
    from pymhm_b200.workloads import DiscInclusions, disc_inclusions

    t0 = time.perf_counter()
    mesh = voronoi_mesh(count, SEED)
    sk = EdgeSkeleton(mesh)
    rs = refinement_for_sizes(mesh, lo, hi, seed=SEED + 1)
    discs = disc_inclusions(300, rmin=0.01, rmax=0.03, seed=SEED + 2)
    field = DiscInclusions(*discs, inside=inside)
    plan = PolygonP2Plan(mesh, sk, rs, preconditioner=preconditioner, workers=min(16, os.cpu_count() or 1))
    plan_s = time.perf_counter() - t0
    failed = []
    if contract_inside:
        plan.set_coefficients(DiscInclusions(*discs, inside=contract_inside), 1.0)
        plan.launch()
        failed = plan.failed_cells()
    plan.set_coefficients(field, 1.0)
    st = torch.cuda.current_stream()
    for _ in range(warmup):
        plan.launch(st)
    torch.cuda.synchronize()
    # cells whose local solve misses the reference's columnwise 1e-10 residual after two
    # corrections: every stage still runs in full for them (the timing is that of the
    # whole workload); the oracle's local solve is run on each to show whether the
    # reference's own path meets the contract there
    edge = plan.failed_cells()
    edge_oracle = {}
    if len(edge):
        from oracle import polygon_mhm as op
        from oracle.q1_mhm import LinearSolveError as OracleError, condense

        for c in edge[:10]:
            prob = op.local_problem(mesh, sk, int(c), mesh.submesh(int(c), int(rs[c])), field, 1.0)
            try:
                condense(prob)
                edge_oracle[int(c)] = "meets the contract"
            except OracleError:
                edge_oracle[int(c)] = "fails the contract"
    per, factor_ms = [], []
    for _ in range(steps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        fev = []
        plan.launch(st, events=ev, factor_events=fev)
        torch.cuda.synchronize()
        per.append([ev[k].elapsed_time(ev[k + 1]) for k in range(4)])
        factor_ms.append(sum(fev[k].elapsed_time(fev[k + 1]) for k in range(0, len(fev), 2)))
    info, stats = plan.general.check()
    per = np.array(per)
    # roofline of the large-tier factorization: 2/3 n^3 flops per matrix of order n (the
    # padded order the kernel factors) against cuBLAS's FP64 GEMM measured here
    large_n = np.array([b["nb"] for b in plan.bins if b["large"] for _ in range(b["k"])], dtype=np.float64)
    flops = float(np.sum(2.0 / 3.0 * large_n ** 3))
    fms = float(np.mean(factor_ms)) if large_n.size else 0.0
    dgemm = dgemm_peak(torch)
    roofline = None
    if large_n.size:
        achieved = flops / (fms * 1e-3) / 1e12
        roofline = {"kernel": "large_factor", "bound": "tensor", "achieved": achieved, "peak": dgemm,
                    "unit": "TFLOP/s", "frac": achieved / dgemm, "ms_per_solve": fms, "flops": flops,
                    "peak_source": "cuBLAS FP64 GEMM (torch.matmul float64, 8192^3) measured in this run",
                    "basis": "2/3 n^3 per large-tier matrix, n its padded order"}
    ms = float(per.sum(axis=1).mean())
    out = {"solves_per_s": 1000.0 / ms, "ms_per_solve": ms,
           "stages_ms": {"local_stage": float(per[:, 0].mean()), "skeleton_scatter": float(per[:, 1].mean()),
                         "general_pcg": float(per[:, 2].mean()), "reconstruct": float(per[:, 3].mean())},
           "macrocells": plan.M, "local_sizes": [int(plan.n_cells.min()), int(plan.n_cells.max())],
           "large_tier": {"cells": int(sum(b["k"] for b in plan.bins if b["large"])), "chunks": len(plan.chunks),
                          "workspace_gb": 2 * (0 if plan.ws_aug is None else plan.ws_aug.numel()) * 8 / 1e9,
                          "roofline": roofline},
           "trace_per_cell": [int(plan.t_cells.min()), int(plan.t_cells.max())], "bins": len(plan.bins),
           "skeleton_unknowns": plan.N, "global_iterations": int(info[1]), "inner_solves": int(info[2]),
           "residual": float(stats[0]), "preconditioner": preconditioner, "disc_permeability": inside,
           "contract_misses": {"cells": len(edge), "oracle_on_them": edge_oracle,
                               "note": "ill-conditioned cells (sliver triangles of short Voronoi edges) whose "
                                       "binary64 residual floor lies at the 1e-10 threshold"},
           "plan_build_s": plan_s}
    if contract_inside:
        out["contract_failures"] = {"disc_permeability": contract_inside, "cells": len(failed),
                                    "first": [int(c) for c in failed[:10]]}
    if cpu_cells:
        from oracle import polygon_mhm as op
        from oracle.q1_mhm import condense, contribution

        from oracle.q1_mhm import LinearSolveError as OracleError

        cells = np.linspace(0, plan.M - 1, cpu_cells).astype(int)
        misses = 0
        c0 = time.perf_counter()
        for c in cells:
            prob = op.local_problem(mesh, sk, int(c), mesh.submesh(int(c), int(rs[c])), field, 1.0)
            try:
                contribution(condense(prob), sk.size + int(c))
            except OracleError:  # a contract miss: the work was done, the reference raises
                misses += 1
        rate = len(cells) / (time.perf_counter() - c0)
        out["cpu_oracle_local_cells_per_s"] = {"value": rate, "cores": 1, "sample": f"{len(cells)} of {plan.M} "
                                               "macrocells, local operators + condensation + contribution",
                                               "contract_misses": misses}
    del plan
    torch.cuda.empty_cache()
    return out


def profile_case(torch, cube=0, count=0):
    """One short run of the 3D or polygon workload for ncu: plan, coefficients, solves,
    status check; returns the global solve's iterations and residual."""
    from pymhm_b200.workloads import DiscInclusions, LayeredField, disc_inclusions, layered_lognormal_permeability

    if cube:
        from pymhm_b200.tetra import TetraMesh, TriangularSkeleton
        from pymhm_b200.tetra_darcy import TetraP1Plan

        mesh = TetraMesh.unit_cube(cube)
        plan = TetraP1Plan(mesh, TriangularSkeleton(mesh, 1), 8)
        plan.set_coefficients(LayeredField(layered_lognormal_permeability(40, 64, sigma=3.0, ell=0.1,
                                                                          contrast=1e6, seed=SEED)), 1.0)
        launches = 2
    else:
        from pymhm_b200.polygon import EdgeSkeleton, voronoi_mesh
        from pymhm_b200.polygon_darcy import PolygonP2Plan, refinement_for_sizes

        mesh = voronoi_mesh(count, SEED)
        plan = PolygonP2Plan(mesh, EdgeSkeleton(mesh), refinement_for_sizes(mesh, 200, 3000, seed=SEED + 1),
                             workers=min(16, os.cpu_count() or 1))
        plan.set_coefficients(DiscInclusions(*disc_inclusions(300, rmin=0.01, rmax=0.03, seed=SEED + 2),
                                             inside=30.0), 1.0)
        launches = 1
    for _ in range(launches):
        plan.launch()
    torch.cuda.synchronize()
    info, stats = plan.check() if cube else plan.general.check()
    return {"case": f"tetra cube {cube}" if cube else f"polygon {count} cells", "launches": launches,
            "global_iterations": int(info[1]), "inner_solves": int(info[2]), "residual": float(stats[0])}


def serving_campaign(torch, lambdas=(100, 500, 2000), requests=150, precisions=("mixed", "fp64"), batch_local=False):
    """Streamed serving (continuous batching with admission by HBM footprint): Poisson
    arrivals at each rate in ``lambdas``; per request a macro grid from {16, 32, 64}^2,
    a local refinement from {4, 8, 16}^2, a seeded log-normal permeability (sigma in
    [1, 2], correlation length 0.05; drawn from a pool of two fields per fine-grid
    size, generated before timing) and 1..8 constant sources, the first solved with
    factors kept, the others through the kept factors.  Before timing, as many slots per
    shape as requests may be in flight (8) are reserved (plans built, both steps
    captured as CUDA graphs), so that no slot is built inside a timed stream, and one
    untimed stream warms them.  With ``batch_local``, requests of one shape admitted
    together share one local-stage launch.  Returns p50/p99 latency (arrival to results
    in pinned host memory) and solves/s per rate and precision."""
    from pymhm_b200.serving import DarcyRequest, ServingEngine, summarize
    from pymhm_b200.workloads import lognormal_permeability

    rng = np.random.default_rng(5)
    pool = {}
    for m in SERVING_MACRO:
        for r in SERVING_LOCAL:
            n = m * r
            if n not in pool:
                pool[n] = [lognormal_permeability(n, n, sigma=float(rng.uniform(1.0, 2.0)), ell=0.05,
                                                  seed=int(rng.integers(1 << 30))) for _ in range(2)]

    def stream(lam, count, seed):
        g = np.random.default_rng(seed)
        t = np.cumsum(g.exponential(1.0 / lam, count)) if lam else np.zeros(count)
        out = []
        for i in range(count):
            m, r = int(g.choice(SERVING_MACRO)), int(g.choice(SERVING_LOCAL))
            kappa = pool[m * r][int(g.integers(2))]
            sources = tuple(float(v) for v in g.uniform(0.5, 2.0, int(g.integers(1, 9))))
            out.append(DarcyRequest(m, r, kappa, sources, arrival=float(t[i])))
        return out

    result = {}
    for prec in precisions:
        engine = ServingEngine(precision=prec, max_in_flight=8, batch_local=batch_local)
        for m in SERVING_MACRO:
            for r in SERVING_LOCAL:
                engine.reserve((m, r, FACE_DEGREE), engine.max_in_flight)
        warm = [DarcyRequest(m, r, pool[m * r][0], (1.0, 2.0)) for m in SERVING_MACRO for r in SERVING_LOCAL] * 2
        engine.run(warm, realtime=False)
        per = {}
        for lam in lambdas:
            before = dict(engine.stats)
            per[f"lambda_{lam}"] = summarize(engine.run(stream(lam, requests, lam)))
            per[f"lambda_{lam}"]["batched_requests"] = (engine.stats.get("batched_requests", 0)
                                                        - before.get("batched_requests", 0))
        per["slots"] = len(engine.slots)
        per["peak_device_bytes"] = int(engine.stats.get("peak_bytes", 0))
        result[prec] = per
        del engine
        torch.cuda.empty_cache()
    result["workload"] = (f"{requests} requests per rate, Poisson arrivals; macro in {SERVING_MACRO}^2, local in "
                          f"{SERVING_LOCAL}^2, P2 faces, 1..8 constant sources per request (kept factors); "
                          "HBM budget 150 GB, 8 requests in flight; same-shape requests admitted together "
                          f"share one local-stage launch: {bool(batch_local)}")
    return result


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true", help="small run for ncu (no baselines, no e2e)")
    ap.add_argument("--profile-extras", action="store_true",
                    help="with --profile: also one refinement step, a P1 batch assembly and a batched LU")
    ap.add_argument("--lu-case", type=int, default=0, metavar="N",
                    help="only factor 64 seeded N x N matrices twice with the batched LU (for ncu)")
    ap.add_argument("--cut-case", type=int, default=0, metavar="P",
                    help="only the 64x64 x 16x16 solve with a P x P pixel field cutting the fine cells, "
                         "mixed and FP64, two timed solves each (for ncu)")
    ap.add_argument("--tetra-case", type=int, default=0, metavar="C",
                    help="only two solves of the 3D workload on the unit cube split into C^3 x 6 macro tetrahedra "
                         "(local refinement 8, the 40-layer field), for ncu")
    ap.add_argument("--polygon-case", type=int, default=0, metavar="M",
                    help="only one solve of the polygon workload with M Voronoi cells (P2 sizes 200-3000, "
                         "disc permeability 30), for ncu")
    ap.add_argument("--serving-full", action="store_true",
                    help="only the streamed-serving workload at its full size: 2000 requests at each of "
                         "50, 100, 200, 500, 1000 and 2000 arrivals/s, mixed and FP64")
    ap.add_argument("--launch-check", action="store_true",
                    help="start the ranks, time an empty step with the barrier and max-over-ranks reduction, "
                         "print the line's rank fields and exit (no GPU work; gloo without a GPU)")
    return ap.parse_args()


def launch_ranks(args):
    """Start ``--gpus`` ranks when this process is not one already (no WORLD_SIZE in the
    environment): re-run this script under torch.distributed.run on 127.0.0.1 and
    exit with its status.  A rank whose WORLD_SIZE differs from ``--gpus`` stops with
    an error.  Returns True when this process only launched the ranks."""
    if args.gpus < 1:
        raise SystemExit("--gpus must be at least 1")
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            raise SystemExit(f"WORLD_SIZE={world} but --gpus {args.gpus}: launch one rank per GPU")
        return False
    if args.gpus == 1:
        return False
    import socket

    with socket.socket() as sock:
        sock.bind(("127.0.0.1", 0))
        port = sock.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    rc = subprocess.call(cmd)
    if rc:
        raise SystemExit(rc)
    return True


def init_dist(world, backend):
    """Process group of the replicas (None for one rank), with a short timeout so that
    ranks waiting on a rank that died end with an error."""
    if world <= 1:
        return None
    import datetime

    import torch.distributed as td

    td.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return td


def launch_check(args):
    """The rank plumbing of a run without GPU work: barrier, a timed empty step per rank
    (one rank sleeps longer), max over ranks, rank 0 prints the rank fields."""
    import torch

    rank, world, _ = dist_env()
    gpu = torch.cuda.is_available()
    dist = init_dist(world, "nccl" if gpu else "gloo")
    device = torch.device("cuda", rank) if gpu else torch.device("cpu")
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    time.sleep(0.01 * (1 + rank))
    mine = (time.perf_counter() - t0) * 1e3
    slowest = max_over_ranks(mine, dist, device)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"launch_check": True, "n_gpus": world, "ms_per_step": slowest,
                          "parallelism": f"replicas x{world}", "rank0_ms": mine}), flush=True)


def lu_case(n, batch=64):
    """The batched dense LU on ``batch`` seeded matrices N(0,1) + n I, factored twice."""
    import torch

    from pymhm_b200 import _lib
    from pymhm_b200.batched import BatchedFactorization

    rng = np.random.default_rng(0)
    a = torch.from_numpy(rng.normal(size=(batch, n, n)) + n * np.eye(n)).to("cuda")
    f = BatchedFactorization(a)
    P = _lib.ptr
    for _ in range(2):
        _lib.check(f.lib.mhm_batched_factor(batch, n, P(f.matrix), P(f.factors), P(f.pivots), P(f.row_scale),
                                            P(f.col_scale), P(f.status), None), "mhm_batched_factor")
    torch.cuda.synchronize()
    print(json.dumps({"lu_case": n, "batch": batch, "ok": bool((f.status == 0).all())}))


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class NvmlClocks:
    """SM clock and clock-event reasons read through NVML every 5 ms on a thread during
    the timed region (read only; the timed region of the default run is tens of ms,
    shorter than nvidia-smi's sampling period).  The GPU is matched by UUID, so a
    remapped CUDA_VISIBLE_DEVICES cannot select another board."""

    PERIOD_S = 0.005

    def __init__(self, device_index):
        import threading

        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        uuid = str(__import__("torch").cuda.get_device_properties(device_index).uuid)
        self.handle = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM))
        self.bits = {
            "hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
            "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
            "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
            "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap,
        }
        self.sm, self.reasons = [], set()
        self.done = threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _sample(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)))
        active = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        self.reasons.update(name for name, bit in self.bits.items() if active & bit)

    def _run(self):
        while True:
            self._sample()
            if self.done.wait(self.PERIOD_S):
                return

    def stop(self):
        self.done.set()
        self.thread.join(timeout=5)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        if not self.sm:
            return None
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": "nvml, 5 ms period"}


def Clocks(index):
    """NVML sampler, or nvidia-smi when NVML is not importable."""
    try:
        return NvmlClocks(index)
    except Exception:
        return SmiClocks(index)


class SmiClocks:
    """nvidia-smi sampling during the timed region (median SM clock, throttle reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.seek(0)
        rows = [r for r in csv.reader(io.StringIO(self.file.read())) if len(r) >= 9]
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms period"}


def workload_kappa():
    from pymhm_b200.workloads import lognormal_permeability

    return lognormal_permeability(MACRO * LOCAL, MACRO * LOCAL, sigma=SIGMA, ell=ELL, seed=SEED)


def cpu_baseline_entry(kappa, runs=CPU_RUNS, serial_cells=SERIAL_SAMPLE_CELLS):
    """The oracle's whole solve of the workload on the host cores, median of ``runs``;
    beside it the local stage in one process with one BLAS thread on a sample of
    cells.  Returns the baseline entry and the median run's solution (the checker of
    the GPU fields)."""
    from oracle.q1_mhm import CartesianSolve, serial_local_rate

    workers = os.cpu_count() or 1
    with CartesianSolve(MACRO, LOCAL, FACE_DEGREE, kappa, 1.0, workers=workers) as solver:
        results = [solver.solve() for _ in range(runs)]
    totals = [r["phases"]["total_s"] for r in results]
    sol = results[int(np.argsort(totals)[len(totals) // 2])]
    sample = np.sort(np.random.default_rng(0).choice(MACRO * MACRO, serial_cells, replace=False))
    rate, seconds = serial_local_rate(MACRO, LOCAL, FACE_DEGREE, kappa, 1.0, sample)
    ph = sol["phases"]
    serial_s = MACRO * MACRO / rate + ph["assembly_s"] + ph["global_solve_s"] + ph["reconstruction_s"]
    entry = {
        "value": 1.0 / ph["total_s"], "unit": "solves/s", "cores": workers, "kind": "port",
        "sample": (f"whole solve of the same workload (4096 local problems on {workers} spawn processes of one "
                   f"BLAS thread, skeleton assembly, global SuperLU solve, reconstruction of fields and fluxes), "
                   f"median of {runs} runs"),
        "runs_s": totals, "phases_s": ph,
        "serial_one_blas_thread": {
            "local_cells_per_s": rate, "sample_cells": serial_cells, "sample_s": seconds,
            "estimated_solve_s": serial_s,
            "note": "local stage of the sampled cells in one process, scaled to 4096 cells, plus the measured "
                    "assembly, global solve and reconstruction phases"},
    }
    return entry, sol


def run_reference(args):
    """Reference arm: the oracle's whole solve per step on all host cores (rank 0)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from oracle.q1_mhm import CartesianSolve

    kappa = workload_kappa()
    workers = os.cpu_count() or 1
    with CartesianSolve(MACRO, LOCAL, FACE_DEGREE, kappa, 1.0, workers=workers) as solver:
        for _ in range(args.warmup):
            solver.solve()
        phases = []
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sol = solver.solve()
            phases.append(sol["phases"])
        elapsed = time.perf_counter() - t0
    ms = 1000.0 * elapsed / args.steps
    value = 1000.0 / ms
    split = {k: float(np.median([p[k] for p in phases])) for k in phases[0]}
    config = workload_config(args)
    config["skeleton_unknowns"] = len(sol["rhs"])
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lognormal kappa, f=1)",
        "config": config, "impl": "reference",
        "phases_median_s": split, "residual": float(sol["residual"]),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "port",
                         "sample": f"whole solve per step: 4096 local problems on {workers} spawn processes of one "
                                   f"BLAS thread (the pool started once, before timing), skeleton assembly, global "
                                   f"SuperLU solve, reconstruction of fields and fluxes"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def workload_config(args):
    return {"workload": f"darcy-q1-{MACRO}x{MACRO}-r{LOCAL}-p{FACE_DEGREE}-lognormal-s{SIGMA:g}-l{ELL:g}",
            "macrocells": MACRO * MACRO, "local_dofs": (LOCAL + 1) ** 2, "rhs_per_cell": 4 * (FACE_DEGREE + 1) + 1,
            "skeleton_unknowns": None, "fine_cells": (MACRO * LOCAL) ** 2, "seed": SEED,
            "parallelism": f"replicas x{int(os.environ.get('WORLD_SIZE', args.gpus))}",
            "serving": "value/e2e: two independent solves in flight per GPU (two plans; local stage on "
                       "low-priority streams, global solve + reconstruction on high-priority streams); "
                       "'sequential': one solve at a time",
            "l2": "sequential: flushed between timed steps (256 MiB write); serving loop: no flush, each "
                  "solve's working set (responses 133 MB + fields/fluxes 26 MB) exceeds the 126 MB L2"}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.lu_case:
        lu_case(args.lu_case)
        return
    if args.cut_case:
        import torch

        print(json.dumps({"cut_case": cut_material_campaign(torch, steps=2, pixels=args.cut_case)}))
        return
    if args.tetra_case or args.polygon_case:
        import torch

        print(json.dumps(profile_case(torch, args.tetra_case, args.polygon_case)))
        return
    if args.serving_full:
        import torch

        print(json.dumps({"serving_stream_full": serving_campaign(torch, lambdas=(50, 100, 200, 500, 1000, 2000),
                                                                  requests=2000)}))
        return
    if launch_ranks(args):
        return
    rank, world, local = dist_env()
    if args.launch_check:
        launch_check(args)
        return
    kappa = workload_kappa()
    # CPU baseline first (spawned pool before any CUDA context exists)
    cpu, ref_sol = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile:
        cpu, ref_sol = cpu_baseline_entry(kappa)
    import torch

    torch.cuda.set_device(local)
    dist = init_dist(world, "nccl")
    from pymhm_b200.darcy import CartesianQ1Plan
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace

    mesh = CartesianMacroMesh(MACRO)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(FACE_DEGREE),) * len(mesh.faces))
    dev = torch.device("cuda", local)
    if args.profile:
        # the bench workload's launches only (mixed precision), for ncu: no baselines,
        # no L2 flush kernels, no host copies
        plan = CartesianQ1Plan(mesh, sk, LOCAL, precision="mixed")
        plan.set_device_coefficients(1, torch.from_numpy(np.ascontiguousarray(kappa)).to(dev), (0.0, 0.0, 0.0),
                                     0, None, 1.0)
        for _ in range(args.warmup + args.steps):
            plan.launch(torch.cuda.current_stream())
        torch.cuda.synchronize()
        info, _ = plan.check()
        extras = {}
        if args.profile_extras:
            # one forced refinement step of this solve, the P1 batch assembly and the
            # batched LU of the 64 x 325 local-stage campaign
            ref = plan.refine(max_steps=1, min_steps=1, rtol=1e-9)
            from pymhm_b200.batched import BatchedFactorization, assemble_p1_batch

            pts, cells = triangle_submesh(24)
            coords = torch.from_numpy(np.repeat(pts[None], 64, axis=0)).to(dev)
            stiff, mass, load = assemble_p1_batch(coords, torch.from_numpy(cells).to(dev),
                                                  diffusion=torch.diag(torch.tensor([3.0, 1.0], device=dev)),
                                                  source=1.0)
            n = stiff.shape[1]
            system = torch.zeros((64, n + 1, n + 1), dtype=torch.float64, device=dev)
            system[:, :n, :n] = stiff
            system[:, :n, n] = system[:, n, :n] = mass.sum(dim=2)
            rhs = torch.zeros((64, n + 1, 4), dtype=torch.float64, device=dev)
            rhs[:, :n, 0] = load
            with BatchedFactorization(system) as fact:
                fact.solve(rhs)
            torch.cuda.synchronize()
            extras = {"refinement_residuals": [float(v) for v in ref.residual_norms], "p1_batch": [64, n]}
        print(json.dumps({"profile": True, "launches": 4 * (args.warmup + args.steps),
                          "global_iterations": int(info[1]), **extras}), flush=True)
        return
    plans = {p: [CartesianQ1Plan(mesh, sk, LOCAL, precision=p) for _ in range(2)] for p in ("mixed", "fp64")}
    kappa_host = torch.from_numpy(np.ascontiguousarray(kappa)).pin_memory()
    kappa_dev = [kappa_host.to(dev) for _ in range(2)]  # one resident copy per plan
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()
    lo, hi = torch.cuda.Stream.priority_range()
    local_st = [torch.cuda.Stream(device=dev, priority=lo) for _ in range(2)]
    global_st = [torch.cuda.Stream(device=dev, priority=hi) for _ in range(2)]

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def fork():
        for st in local_st + global_st:
            st.wait_stream(stream)

    def join():
        for st in local_st + global_st:
            stream.wait_stream(st)

    seq, pipe = {}, {}
    for prec, pl in plans.items():
        for j, plan in enumerate(pl):
            plan.set_device_coefficients(1, kappa_dev[j], (0.0, 0.0, 0.0), 0, None, 1.0)
        # (a) back-to-back single solves on one stream: latency and the per-kernel split,
        #     L2 flushed between steps
        plan = pl[0]
        for _ in range(args.warmup):
            plan.launch(stream)
        torch.cuda.synchronize()
        plan.check()
        steps, kern = [], []
        barrier()
        for _ in range(args.steps):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            plan.launch(stream, events=ev)
            torch.cuda.synchronize()
            steps.append(ev[0].elapsed_time(ev[4]))
            kern.append([ev[k].elapsed_time(ev[k + 1]) for k in range(4)])
        barrier()
        info, stats = plan.check()
        seq[prec] = dict(steps=np.array(steps), kern=np.array(kern), info=info, stats=stats)
        # (b) serving loop: request k on plan k % 2, two solves in flight; the local stage
        #     runs on low-priority streams, the global solve and the reconstruction on
        #     high-priority ones, so each solve's latency-bound global stage overlaps the
        #     next request's local stage
        fork()
        for k in range(args.warmup):
            pl[k % 2].launch(local_st[k % 2], global_stream=global_st[k % 2])
        join()
        torch.cuda.synchronize()
        clocks = Clocks(local) if prec == "mixed" else None
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
        e0.record(stream)
        fork()
        for k in range(args.steps):
            pl[k % 2].launch(local_st[k % 2], global_stream=global_st[k % 2], events=evs[k])
        join()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        clk = clocks.stop() if clocks else None
        for plan in pl:
            plan.check()
        pipe[prec] = dict(total=e0.elapsed_time(e1), lat=np.array([e[0].elapsed_time(e[4]) for e in evs]), clocks=clk)

    # repeated sources on a fixed material (offline / online reuse): the factors of the
    # local problems are kept, each query re-solves the source column only
    online = {}
    for prec, pl in plans.items():
        plan = pl[0]
        plan.prepare_offline(stream)
        for _ in range(args.warmup):
            plan.launch(stream, local="online")
        torch.cuda.synchronize()
        steps_on, kern_on = [], []
        for _ in range(args.steps):
            flush.zero_()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
            plan.launch(stream, events=ev, local="online")
            torch.cuda.synchronize()
            steps_on.append(ev[0].elapsed_time(ev[4]))
            kern_on.append(ev[0].elapsed_time(ev[1]))
        plan.check()
        # the same query captured as a CUDA graph and replayed
        plan.capture_online()
        for _ in range(args.warmup):
            gst = plan.replay_online(1.0)
        torch.cuda.synchronize()
        steps_g = []
        for k in range(args.steps):
            flush.zero_()
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(gst)
            plan.replay_online(1.0 + 0.01 * k, stream=gst)
            g1.record(gst)
            torch.cuda.synchronize()
            steps_g.append(g0.elapsed_time(g1))
        plan.check()
        online[prec] = {"ms_per_solve": float(np.mean(steps_on)), "source_response_ms": float(np.mean(kern_on)),
                        "graph_ms_per_solve": float(np.mean(steps_g))}
        plan._graphs = None
        plan.factors = None

    # original-equation refinement of a mixed-precision solve (refine_hybrid): one
    # forced correction step on the host clock (each step synchronises twice)
    plan = plans["mixed"][0]
    plan.launch(stream)
    torch.cuda.synchronize()
    plan.refine(max_steps=1, min_steps=1, rtol=1e-9, stream=stream)  # first call sizes its buffers
    plan.launch(stream)
    torch.cuda.synchronize()
    t_ref = time.perf_counter()
    ref_out = plan.refine(max_steps=1, min_steps=1, rtol=1e-9, stream=stream)
    refinement = {"ms_one_correction": (time.perf_counter() - t_ref) * 1e3,
                  "residual_norms": [float(v) for v in ref_out.residual_norms], "rhs_norm": ref_out.rhs_norm,
                  "note": "refine_hybrid on the mixed solve: original-equation residual, defect source responses "
                          "with a fresh factorization, correction solve, reconstruction; forced one step"}

    # streamed serving of independent requests (continuous batching, HBM admission)
    serving_stream = serving_campaign(torch)
    small_poisson = small_poisson_campaign(torch)
    cut_material = cut_material_campaign(torch)
    tetra = tetra_campaign(torch)
    polygon = polygon_campaign(torch)

    # the reference's own batched local-stage benchmark, same phases and sizes
    campaigns = {f"batched_local_r{r}": batched_local_campaign(torch, r) for r in (12, 24)}
    campaigns["reference_rtx3060_ms"] = {
        "batched_local_r12": {"factorization": 3.19, "first_solve": 1.31, "repeated_rhs_total": 16.0, "total": 26.6},
        "batched_local_r24": {"factorization": 28.0, "first_solve": 5.15, "repeated_rhs_total": 61.6,
                              "total": 105.6}}
    campaigns["note"] = ("gpu_campaign of benchmarks/execution_modes.py (64 P1 triangle meshes, 12 queries) with "
                         "assemble_p1_batch and BatchedFactorization of this library; reference figures: RTX 3060 "
                         "(benchmarks/results/execution/gpu-r12.json, gpu-r24.json)")

    # end to end through the public API, same serving loop: H2D kappa, solve, D2H
    # fields / flux / x / status / info for every request
    pl = plans["mixed"]
    plan = pl[0]
    n_out = plan.fields.numel() + plan.flux.numel() + plan.x.numel()
    hosts = [dict(fields=torch.empty(plan.fields.shape, dtype=torch.float64).pin_memory(),
                  flux=torch.empty(plan.flux.shape, dtype=torch.float64).pin_memory(),
                  x=torch.empty(plan.x.shape, dtype=torch.float64).pin_memory(),
                  status=torch.empty(plan.cell_status.shape, dtype=torch.int32).pin_memory(),
                  info=torch.empty(4, dtype=torch.int32).pin_memory()) for _ in range(2)]
    # two permeability buffers per plan: request k+2 uploads into the one request k
    # does not read, on an upload stream, while request k computes
    kdev = [[torch.empty_like(kappa_dev[0]) for _ in range(2)] for _ in range(2)]
    for j in range(2):
        pl[j].set_device_coefficients(1, kdev[j][0], (0.0, 0.0, 0.0), 0, None, 1.0)

    # results leave on a copy stream per plan: the plan's next local stage waits for
    # its previous solve's compute only, and its next global stage (which rewrites x,
    # fields and flux) for the copies, which have long finished by then
    copy_st = [torch.cuda.Stream(device=dev) for _ in range(2)]
    upload_st = [torch.cuda.Stream(device=dev) for _ in range(2)]
    copied, status_copied = [None, None], [None, None]
    local_done = [[None, None], [None, None]]  # [plan][buffer]: the local stage that last read it

    def request(k):
        j, b = k % 2, (k // 2) % 2
        p_, ls, gs, cs, h = pl[j], local_st[j], global_st[j], copy_st[j], hosts[j]
        us = upload_st[j]
        if local_done[j][b] is not None:
            us.wait_event(local_done[j][b])
        with torch.cuda.stream(us):
            kdev[j][b].copy_(kappa_host, non_blocking=True)
        uploaded = torch.cuda.Event()
        uploaded.record(us)
        if getattr(p_, "_done", None) is not None:
            ls.wait_event(p_._done)  # the previous solve on this plan still reads its responses
        if status_copied[j] is not None:
            ls.wait_event(status_copied[j])  # the local stage rewrites the cell status words
        if copied[j] is not None:
            gs.wait_event(copied[j])
        ls.wait_event(uploaded)
        p_.set_device_coefficients(1, kdev[j][b], (0.0, 0.0, 0.0), 0, None, 1.0)
        p_.launch(ls, global_stream=gs)  # records p_._done on gs after the reconstruction
        local_done[j][b] = torch.cuda.Event()
        local_done[j][b].record(ls)
        cs.wait_event(p_._done)
        with torch.cuda.stream(cs):
            h["status"].copy_(p_.cell_status, non_blocking=True)
            status_copied[j] = torch.cuda.Event()
            status_copied[j].record(cs)
            h["info"].copy_(p_.info, non_blocking=True)
            h["fields"].copy_(p_.fields, non_blocking=True)
            h["flux"].copy_(p_.flux, non_blocking=True)
            h["x"].copy_(p_.x, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(cs)
        copied[j] = ev

    def fork_all():
        fork()
        for cs in copy_st + upload_st:
            cs.wait_stream(stream)

    def join_all():
        join()
        for cs in copy_st + upload_st:
            stream.wait_stream(cs)

    fork_all()
    for k in range(args.warmup):
        request(k)
    join_all()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fork_all()
    for k in range(args.steps):
        request(k)
    join_all()
    e1.record(stream)
    torch.cuda.synchronize()
    for h in hosts:
        if int(h["status"].numpy().max()) != 0 or int(h["info"][0]) != 0:
            raise RuntimeError("end-to-end solve reported a failure")
    e2e_total = e0.elapsed_time(e1)
    h2d = kappa_host.numel() * 8
    d2h = n_out * 8 + plan.cell_status.numel() * 4 + 16
    host_fields, host_flux, host_x = hosts[(args.steps - 1) % 2]["fields"], hosts[(args.steps - 1) % 2]["flux"], \
        hosts[(args.steps - 1) % 2]["x"]

    # accuracy: lambda and c against the reference's FP64 solution (golden fixture of the
    # same workload); u and the flux, relative L2 over all cells, against the CPU
    # baseline's oracle solve (which reproduces the reference's matrix and unknowns)
    acc = {}
    gpath = os.path.join(ROOT, "tests", "golden", "darcy_64x64_r16_p2_lognormal.npz")
    if os.path.exists(gpath):
        g = np.load(gpath)
        T = plan.T
        rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
        fp64_plan = plans["fp64"][0]
        # the online campaign's replays left another source on this plan
        fp64_plan.set_device_coefficients(1, kappa_dev[0], (0.0, 0.0, 0.0), 0, None, 1.0)
        fp64_plan.launch(stream)
        torch.cuda.synchronize()
        fp64_out = (fp64_plan.x.cpu().numpy(), fp64_plan.fields.cpu().numpy(), fp64_plan.flux.cpu().numpy())
        for name, (x, fields, flux) in (("mixed", (host_x.numpy(), host_fields.numpy(), host_flux.numpy())),
                                        ("fp64", fp64_out)):
            e = {"lambda": rel(x[:T], g["trace"]), "coarse": rel(x[T:], g["coarse"])}
            if ref_sol is not None:
                e["u"] = rel(fields, ref_sol["fields"])
                e["flux"] = rel(flux, ref_sol["flux"])
            acc[name] = e
        acc["note"] = ("relative L2 errors; lambda, coarse: against the reference's solution (fixture); u, flux: "
                       "all 4096 cells against the oracle's solve in the CPU baseline" if ref_sol is not None else
                       "relative L2 errors against the reference's solution (fixture); u and flux need the CPU "
                       "baseline's solve, which this run skipped")

    def agg(v):
        return max_over_ranks(v, dist, dev)

    K = args.steps
    ms = agg(pipe["mixed"]["total"] / K)
    ms64 = agg(pipe["fp64"]["total"] / K)
    ms_e2e = agg(e2e_total / K)
    seq_ms = agg(float(seq["mixed"]["steps"].mean()))
    seq_ms64 = agg(float(seq["fp64"]["steps"].mean()))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    mixed, fp64 = seq["mixed"], seq["fp64"]
    kern = mixed["kern"].mean(axis=0)
    names = ["q1_condense", "skeleton_scatter", "skeleton_pcg", "q1_reconstruct"]
    top = int(np.argmax(kern))
    roof = roofline(plan, names[top], kern[top], int(mixed["info"][1]), int(mixed["info"][2]))

    def pct(v, q):
        return float(np.percentile(v, q))

    line = {
        "metric": METRIC, "value": world * 1000.0 / ms, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded lognormal kappa, f=1)", "config": workload_config(args),
        "latency_ms": {"p50": pct(pipe["mixed"]["lat"], 50), "p99": pct(pipe["mixed"]["lat"], 99)},
        "fp64": {"value": world * 1000.0 / ms64, "ms_per_step": ms64,
                 "p50": pct(pipe["fp64"]["lat"], 50), "p99": pct(pipe["fp64"]["lat"], 99),
                 "sequential_ms": seq_ms64,
                 "kernels_ms": dict(zip(names, map(float, fp64["kern"].mean(axis=0)))),
                 "global_iterations": int(fp64["info"][1])},
        "mixed_over_fp64": ms64 / ms,
        "sequential": {"ms_per_solve": seq_ms, "p50": pct(mixed["steps"], 50), "p99": pct(mixed["steps"], 99),
                       "fp64_ms_per_solve": seq_ms64},
        "kernels_ms": dict(zip(names, map(float, kern))),
        "online_new_source": {"mixed": online["mixed"], "fp64": online["fp64"],
                              "note": "OfflineQ1System: kept local factors, one query = source responses + "
                                      "right-hand-side reduction + global solve + reconstruction, one at a time"},
        "refinement": refinement,
        "reference_campaigns": campaigns,
        "serving_stream": serving_stream,
        "poisson_8x8_r4_p1": small_poisson,
        "cut_material": cut_material,
        "tetra_3d": tetra,
        "polygon_p2": polygon,
        "global_iterations": int(mixed["info"][1]), "outer_corrections": int(mixed["info"][2]),
        "residual": float(mixed["stats"][0]), "certificate": float(mixed["stats"][1]),
        "error_vs_reference": acc,
        "e2e": {"value": world * 1000.0 / ms_e2e, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e},
        "gpu_launches": 4 * args.steps,
        "roofline": roof, "cpu_baseline": cpu, "clocks": pipe["mixed"]["clocks"],
    }
    line["config"]["skeleton_unknowns"] = plan.N
    print(json.dumps(line), flush=True)


def max_over_ranks(value, dist, device):
    """Max of a per-rank scalar (the job's time is its slowest replica)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def profile_traffic(kernel):
    """DRAM bytes per launch (read + write) of ``kernel`` from the committed ncu summary,
    with the command that measured them; None when that kernel was not captured."""
    if not os.path.exists(TRAFFIC_FILE):
        return None, None
    with open(TRAFFIC_FILE) as f:
        entry = json.load(f).get(kernel)
    if not entry:
        return None, None
    return float(entry["dram_bytes_read"]) + float(entry["dram_bytes_write"]), entry


def roofline(plan, kernel, ms, inner_iters, outer):
    """Algorithmic bytes of the dominant kernel per launch over its measured time.

    Global CG: per inner iteration one sweep of the CSR matrix (12 bytes per stored
    entry: value and column index) and six vectors of N doubles, nnz*12 + 6*N*8, times
    the measured inner iterations.  The kernel's own model of what it moves (cell
    blocks and tables once, per iteration the exchanged face partials and coarse row
    data, one CSR sweep per outer correction) is reported beside it."""
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, source = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak, source = float(json.load(f)["hbm_gbs"]), "measured"
    p = plan.pattern
    nnz = len(p.indices)
    M, n, w, T, N = plan.cells, plan.n, plan.w, plan.T, plan.N
    model = None
    if kernel == "skeleton_pcg":
        t = plan.t
        per_iter = nnz * 12 + 6 * N * 8
        bytes_ = inner_iters * per_iter
        setup = M * (t + 1) * (t + 1) * 8 + M * t * (8 + 8 + 4) + T * 16
        kernel_iter = 2 * (M * t * 8 + 2 * T * 8) + 2 * (2 * 3 * M * 8 + M * 8 + 3 * M * 8)
        model = setup + inner_iters * kernel_iter + (outer + 2) * (nnz * 12 + 2 * N * 8)
        basis = f"{inner_iters} inner iterations x (nnz*12 + 6*N*8) = {inner_iters} x {per_iter} bytes"
    elif kernel == "q1_condense":
        bytes_ = plan.nxf * plan.nyf * 8 + M * w * (n + 1) * 8 + M * (plan.t + 1) * (plan.t + 2) * 8
        basis = "kappa read + responses and Schur blocks / loads written"
    elif kernel == "q1_reconstruct":
        bytes_ = M * w * (n + 1) * 8 + plan.nxf * plan.nyf * 8 + M * n * 8 + M * plan.nfine * 16
        basis = "responses and kappa read + fields and fluxes written"
    else:
        bytes_ = nnz * 24 + N * 24
        basis = "contributor maps and blocks read + values written"
    achieved = bytes_ / (ms * 1e-3) / 1e9
    traffic, prof = profile_traffic(kernel)
    out = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "traffic": traffic, "algorithmic_bytes": int(bytes_), "basis": basis,
           "ms_per_launch": float(ms),
           "peak_source": source + " (MEASURED_PEAKS.json hbm_gbs)" if source == "measured" else source}
    if model is not None:
        out["kernel_model_bytes"] = int(model)
    if prof is not None:
        out["traffic_source"] = {k: prof[k] for k in ("command", "case") if k in prof}
    return out


if __name__ == "__main__":
    main()
