"""3D Primal-MHM Darcy on tetrahedral macro meshes with P1 local spaces, on the GPU.

GPU counterpart of ``solve_darcy_3d`` (PyMHM 1.3.2, ``src/pymhm/_legacy/models/darcy/
primal_3d.py:68-147``) for degree-one local spaces, uniform red refinement of every
macrocell, a ``TriangularSkeleton`` of Bernstein degree 0 or 1 per face, homogeneous
Dirichlet data and a constant source.  One launch sequence per solve, all on the
device, no host synchronisation:

1. ``mhm_tet_kappa``: the Duffy-rule average of the permeability over every fine
   tetrahedron (a ``LayeredField``; a constant permeability skips it);
2. ``mhm_p1_batch_assemble``: dense P1 stiffness, mass and load of every macrocell
   (all macrocells share the refined connectivity);
3. ``mhm_dense_systems``: the local contract and the augmented systems;
4. ``mhm_batched_factor_large`` / ``mhm_batched_solve_large``: equilibrated LU with
   the row search of each 32-column panel kept to its diagonal window (exact for these
   bordered semi-definite systems; 20 % faster here than full partial pivoting, which
   ``lu="partial"`` selects: ``mhm_batched_factor`` / ``mhm_batched_solve``) and the
   checked, refined multi-RHS solve (``BatchedFactorization``'s contract);
5. ``mhm_dense_contributions``: Schur blocks and loads on the tensor cores;
6. ``mhm_skeleton_scatter``: the ordered reduction into the skeleton system;
7. ``mhm_general_solve``: the global solve (projected PCG, outer FP64 correction);
8. ``mhm_dense_reconstruct``: the nodal fields.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import _lib
from .batched import _node_incidence
from .errors import LinearSolveError
from .general import GeneralSkeleton
from .tetra import TetraMesh, TriangularSkeleton, duffy_tetrahedron, reference_refinement, trace_coupling
from .topology import skeleton_pattern, transpose_slots
from .workloads import LayeredField

UNIT_TET = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


@dataclass
class Tetra3DSolution:
    trace: np.ndarray
    coarse: np.ndarray
    fields: np.ndarray  # (cells, local nodes)
    residual: float
    corrected: np.ndarray
    global_iterations: int
    outer_corrections: int
    seconds: float = 0.0


class TetraP1Plan:
    """Device-resident plan of one tetrahedral problem shape (mesh, skeleton, local
    refinement): topology, tables, sparsity and every buffer of the launch sequence."""

    def __init__(self, mesh: TetraMesh, skeleton: TriangularSkeleton | None = None, local_refinement: int = 2, *,
                 device=None, global_rtol=1e-13, inner_rtol=1e-10, max_inner=20000, max_outer=16,
                 preconditioner="cell", lu="windowed"):
        import torch

        if lu not in ("windowed", "partial"):
            raise ValueError("lu must be 'windowed' (the bordered systems' panel-window pivoting) or 'partial'")
        self.lu = lu

        self.torch = torch
        self.lib = _lib.lib()
        self.device = torch.device("cuda" if device is None else device)
        self.mesh = mesh
        self.skeleton = TriangularSkeleton(mesh, 1) if skeleton is None else skeleton
        if self.skeleton.mesh is not mesh:
            raise ValueError("skeleton must belong to the supplied tetrahedral mesh")
        self.r = int(local_refinement)
        self.global_rtol, self.inner_rtol = float(global_rtol), float(inner_rtol)
        self.max_inner, self.max_outer = int(max_inner), int(max_outer)
        if preconditioner not in ("cell", "face"):
            raise ValueError("preconditioner must be 'cell' (the cells' D S^-1 D) or 'face' (face blocks)")
        self.preconditioner = preconditioner
        bary, conn = reference_refinement(self.r)
        fine_cells = TetraMesh(bary @ UNIT_TET, conn).cells  # oriented as in every positive macrocell
        self.n, self.E = len(bary), len(fine_cells)
        sk = self.skeleton
        self.t = 4 * sk.modes
        self.M = len(mesh.cells)
        self.T, self.N = sk.size, sk.size + self.M
        if self.t > 12:
            raise NotImplementedError("at most 12 trace DOFs per cell")
        macro = mesh.points[mesh.cells]  # (cells, 4, 3), positively oriented
        # the submeshes' vertices, each computed as TetraMesh.submesh does (bary @ X):
        # the material pre-pass must see the same coordinates as the reference
        points = np.stack([bary @ X for X in macro])
        coupling = trace_coupling(mesh, sk, self.r)
        self.cell_dofs_h = sk.cell_dof_array
        self.pattern = skeleton_pattern(self.cell_dofs_h, self.T)
        node_ptr, node_contrib = _node_incidence(fine_cells.astype(np.int32), self.n)
        qbary, qw = duffy_tetrahedron(5)
        dev, f64 = self.device, dict(dtype=torch.float64, device=self.device)

        def up(a, dtype):
            return torch.as_tensor(np.array(a, order="C", copy=True), dtype=dtype).to(dev)

        self.d_fine_cells = up(fine_cells, torch.int32)
        self.d_qbary, self.d_qw = up(qbary, torch.float64), up(qw, torch.float64)
        self.d_points = up(points, torch.float64)
        self.d_coupling = up(coupling, torch.float64)
        self.d_node_ptr, self.d_node_contrib = up(node_ptr, torch.int64), up(node_contrib, torch.int32)
        self.d_cell_dofs = up(self.cell_dofs_h, torch.int64)
        p = self.pattern
        self.d_slot_ptr, self.d_contrib = up(p.slot_ptr, torch.int64), up(p.contrib, torch.int64)
        self.d_load_ptr, self.d_load_contrib = up(p.load_ptr, torch.int64), up(p.load_contrib, torch.int64)
        self.d_indptr, self.d_indices = up(p.indptr, torch.int64), up(p.indices, torch.int32)
        self.d_boundary = torch.zeros(self.T, **f64)
        self.general = GeneralSkeleton(list(self.cell_dofs_h), list(sk.geometric_constraint()), sk.offsets, self.T,
                                       p.indptr, p.indices, device=dev)
        M, n, E, t = self.M, self.n, self.E, self.t
        n1, w = n + 1, t + 2
        self.diffusion = torch.empty((M, E, 3, 3), **f64)
        nbytes = int(self.lib.mhm_p1_batch_scratch_bytes(M, 3, E))
        self.scratch = torch.empty(max(nbytes // 8, 1), **f64)
        self.stiffness = torch.empty((M, n, n), **f64)
        self.mass = torch.empty((M, n, n), **f64)
        self.load = torch.empty((M, n), **f64)
        self.p1_status = torch.zeros(4, dtype=torch.int32, device=dev)
        self.aug = torch.empty((M, n1, n1), **f64)
        self.rhs = torch.empty((M, n1, w), **f64)
        self.action = torch.empty((M, 3, n1), **f64)
        self.n_of = torch.full((M,), n, dtype=torch.int32, device=dev)
        self.t_of = torch.full((M,), t, dtype=torch.int32, device=dev)
        cells = torch.arange(M, dtype=torch.int64, device=dev)
        self.block_off, self.load_off = cells * (t + 1) * (t + 1), cells * (t + 1)
        self.dof_off, self.field_off = cells * t, cells * n
        self.cell_id = cells.to(torch.int32)
        self.corrected = torch.empty(M, dtype=torch.uint8, device=dev)
        self.cell_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.factors = torch.empty_like(self.aug)
        self.pivots = torch.empty((M, n1), dtype=torch.int32, device=dev)
        self.row_scale = torch.empty((M, n1), **f64)
        self.col_scale = torch.empty((M, n1), **f64)
        self.factor_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.solve_status = torch.empty(M, dtype=torch.int32, device=dev)
        self.solution = torch.empty((M, n1, w), **f64)
        self.work = torch.empty((M, n1, w), **f64)
        if self.lu == "windowed":
            # every local system is bordered semi-definite (P1 stiffness, the mass
            # constraint): the large-order LU's panel-window pivoting factors it exactly
            rec = np.array([(k * n1 * n1, k * n1, k * n1 * w, n1, w, k, 0) for k in range(M)],
                           dtype=[("mat_off", "<i8"), ("vec_off", "<i8"), ("rhs_off", "<i8"), ("n", "<i4"),
                                  ("nrhs", "<i4"), ("slot", "<i4"), ("reserved", "<i4")])
            self.d_desc = torch.as_tensor(rec.view(np.uint8).copy()).to(dev)
            self.large_work = torch.empty(66 * M * n1, **f64)
        self.blocks = torch.empty((M, t + 1, t + 1), **f64)
        self.loads = torch.empty((M, t + 1), **f64)
        self.values = torch.empty(len(p.indices), **f64)
        self.grhs = torch.empty(self.N, **f64)
        self.load_scale = torch.empty(self.N, **f64)
        self.x = torch.empty(self.N, **f64)
        self.fields = torch.empty((M, n), **f64)
        self.kappa = None
        self.kconst = torch.eye(3, dtype=torch.float64, device=dev)
        self.source = torch.ones(1, **f64)

    def set_coefficients(self, permeability=1.0, source=1.0):
        """A ``LayeredField`` (voxel values uploaded) or a positive constant permeability;
        a constant source."""
        torch = self.torch
        if isinstance(permeability, LayeredField):
            self.kappa = torch.as_tensor(permeability.values).to(self.device)
        elif np.ndim(permeability) == 0 and float(permeability) > 0:
            self.kappa = None
            self.kconst = float(permeability) * torch.eye(3, dtype=torch.float64, device=self.device)
        else:
            raise NotImplementedError("permeability: a LayeredField or a positive constant")
        if np.ndim(source) != 0 or not np.isfinite(float(source)):
            raise NotImplementedError("the GPU tetrahedral path takes a constant source")
        self.source = torch.full((1,), float(source), dtype=torch.float64, device=self.device)

    def launch(self, stream=None, *, events=None):
        """Enqueue one complete solve on ``stream`` (no host synchronisation).  ``events``:
        five CUDA events recorded before the local stage, the reduction, the global
        solve, the reconstruction and after it."""
        P, lib, sh = _lib.ptr, self.lib, _lib.stream_handle(stream)
        M, n, E, t = self.M, self.n, self.E, self.t
        st = self.torch.cuda.current_stream() if stream is None else stream

        def mark(k):
            if events is not None:
                events[k].record(st)

        mark(0)
        if self.kappa is not None:
            L, px, py = self.kappa.shape
            _lib.check(lib.mhm_tet_kappa(M, P(self.d_points), n, E, P(self.d_fine_cells), len(self.d_qw),
                                         P(self.d_qbary), P(self.d_qw), L, px, py, P(self.kappa), P(self.diffusion),
                                         sh), "mhm_tet_kappa")
            kbase, kb, kc = self.diffusion, E, 1
        else:
            kbase, kb, kc = self.kconst, 0, 0
        _lib.check(lib.mhm_p1_batch_assemble(M, n, 3, P(self.d_points), E, P(self.d_fine_cells), P(kbase), kb, kc,
                                             P(self.source), 0, 0, P(self.d_node_ptr), P(self.d_node_contrib),
                                             P(self.scratch), P(self.stiffness), P(self.mass), P(self.load),
                                             P(self.p1_status), sh), "mhm_p1_batch_assemble")
        n1, w = n + 1, t + 2
        _lib.check(lib.mhm_dense_systems(M, n, t, n1, w, 0, P(self.n_of), P(self.t_of), P(self.stiffness),
                                         P(self.mass), P(self.load), P(self.d_coupling), P(self.aug), P(self.rhs),
                                         P(self.action), P(self.corrected), P(self.cell_status), sh),
                   "mhm_dense_systems")
        if self.lu == "windowed":
            _lib.check(lib.mhm_batched_factor_large(M, P(self.d_desc), n1, P(self.aug), P(self.factors),
                                                    P(self.pivots), P(self.row_scale), P(self.col_scale),
                                                    P(self.factor_status), sh), "mhm_batched_factor_large")
        else:
            _lib.check(lib.mhm_batched_factor(M, n1, P(self.aug), P(self.factors), P(self.pivots), P(self.row_scale),
                                              P(self.col_scale), P(self.factor_status), sh), "mhm_batched_factor")
        with self.torch.cuda.stream(st):
            self.solve_status.copy_(self.factor_status)  # the solve adds its failures to the factor's
        if self.lu == "windowed":
            _lib.check(lib.mhm_batched_solve_large(M, P(self.d_desc), n1, w, P(self.aug), P(self.factors),
                                                   P(self.pivots), P(self.row_scale), P(self.col_scale), P(self.rhs),
                                                   P(self.solution), P(self.large_work), 1e-10, 0.0, 2,
                                                   P(self.solve_status), sh), "mhm_batched_solve_large")
        else:
            _lib.check(lib.mhm_batched_solve(M, n1, w, P(self.aug), P(self.factors), P(self.pivots),
                                             P(self.row_scale), P(self.col_scale), P(self.rhs), P(self.solution),
                                             P(self.work), 1e-10, 0.0, 2, P(self.solve_status), sh),
                       "mhm_batched_solve")
        _lib.check(lib.mhm_dense_contributions(M, n, t, n1, w, t, P(self.n_of), P(self.t_of), P(self.solution),
                                               P(self.d_coupling), P(self.action), P(self.load), P(self.block_off),
                                               P(self.load_off), P(self.blocks), P(self.loads), sh),
                   "mhm_dense_contributions")
        p = self.pattern
        mark(1)
        _lib.check(lib.mhm_skeleton_scatter(len(p.indices), P(self.d_slot_ptr), P(self.d_contrib), P(self.blocks),
                                            P(self.values), self.N, self.T, P(self.d_load_ptr),
                                            P(self.d_load_contrib), P(self.loads), P(self.d_boundary), P(self.grhs),
                                            P(self.load_scale), sh), "mhm_skeleton_scatter")
        mark(2)
        self.general.launch(self.values, self.grhs, self.x, rtol=self.global_rtol, inner_rtol=self.inner_rtol,
                            max_inner=self.max_inner, max_outer=self.max_outer, stream=stream,
                            blocks=self.blocks if self.preconditioner == "cell" else None)
        mark(3)
        _lib.check(lib.mhm_dense_reconstruct(M, n1, w, P(self.n_of), P(self.t_of), P(self.solution),
                                             P(self.d_cell_dofs), P(self.dof_off), P(self.cell_id), self.T, P(self.x),
                                             P(self.field_off), P(self.fields), sh), "mhm_dense_reconstruct")
        mark(4)

    def check(self):
        """Raise the reference's error for any failed stage (synchronises)."""
        flags = self.p1_status.cpu().numpy()
        if flags.any():
            raise ValueError(["points must be finite", "degenerate simplex in resident geometry",
                              "diffusion must be finite real symmetric positive definite",
                              "source must be real finite cell values"][int(np.flatnonzero(flags)[0])])
        for arr in (self.cell_status, self.solve_status):
            st = arr.cpu().numpy()
            bad = np.flatnonzero(st)
            if len(bad):
                raise LinearSolveError(f"{_lib.CELL_MESSAGES.get(int(st[bad[0]]), 'cell failed')} "
                                       f"(macrocell {int(bad[0])})")
        return self.general.check()

    def result(self, seconds=0.0) -> Tetra3DSolution:
        info, stats = self.check()
        x = self.x.cpu().numpy()
        return Tetra3DSolution(trace=x[: self.T].copy(), coarse=x[self.T:].copy(), fields=self.fields.cpu().numpy(),
                               residual=float(stats[0]), corrected=self.corrected.cpu().numpy().astype(bool),
                               global_iterations=int(info[1]), outer_corrections=int(info[2]), seconds=seconds)

    def solve(self, permeability=1.0, source=1.0, stream=None) -> Tetra3DSolution:
        t0 = time.perf_counter()
        self.set_coefficients(permeability, source)
        self.launch(stream)
        sol = self.result()
        sol.seconds = time.perf_counter() - t0
        return sol

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
        _lib.check(self.lib.mhm_skeleton_export_csc(self.N, P(self.d_indptr), P(self.d_indices), P(c["transpose"]),
                                                    P(self.values), P(c["indptr"]), P(c["indices"]), P(c["data"]),
                                                    _lib.stream_handle(None)), "mhm_skeleton_export_csc")
        kept = int(c["indptr"][-1])
        return sparse.csc_matrix((c["data"][:kept].cpu().numpy(), c["indices"][:kept].cpu().numpy(),
                                  c["indptr"].cpu().numpy()), shape=(self.N, self.N))


def solve_darcy_3d(mesh: TetraMesh, *, permeability=1.0, source=0.0, dirichlet=0.0, neumann=None,
                   skeleton: TriangularSkeleton | None = None, local_refinement: int = 2, local_meshes=None,
                   degree: int = 2, quadrature_order: int = 5, mean_pressure: float = 0.0, solver="scipy",
                   local_solver="scipy", backend="serial", workers=None) -> Tetra3DSolution:
    """GPU counterpart of ``solve_darcy_3d`` (``primal_3d.py:68-147``) for ``degree=1``,
    homogeneous Dirichlet data, uniform local refinement, a constant source and a
    constant or ``LayeredField`` permeability.  ``solver``, ``local_solver``,
    ``backend``, ``workers`` and ``mean_pressure`` are accepted for signature
    compatibility; other values of the rest raise ``NotImplementedError``."""
    del solver, local_solver, backend, workers, mean_pressure
    if int(degree) != 1:
        raise NotImplementedError("the GPU tetrahedral path implements degree-one local spaces")
    if local_meshes is not None or neumann:
        raise NotImplementedError("explicit local meshes and Neumann data are not on the GPU tetrahedral path")
    if np.ndim(dirichlet) != 0 or float(dirichlet) != 0.0:
        raise NotImplementedError("the GPU tetrahedral path takes homogeneous Dirichlet data")
    if int(quadrature_order) != 5:
        raise NotImplementedError("the permeability average uses the reference's default order 5")
    plan = TetraP1Plan(mesh, skeleton, local_refinement)
    return plan.solve(permeability, source)
