"""NumPy/SciPy restatement of PyMHM's primal P2 Darcy path on polygon macro meshes
(config 3; the oracle).

Test infrastructure only: imported by ``tests/`` and ``bench.py``'s CPU arm, never by
``pymhm_b200``.  It follows PyMHM 1.3.2 (paths relative to ``src/pymhm/``):

* local operators   ``fem/scalar/triangle.py:208-257`` (``scalar_operators``: Duffy
                    rule ``triangle_quadrature``, the material sampled at the points,
                    compensated diffusion blocks), ``fem/scalar/operators.py:63-78``
* driver            ``_legacy/models/darcy/primal.py:28-106, 173-344``
                    (``_DarcyLocalFactory``: kernel 1, constraint M 1 / (1^T M 1),
                    quadrature count max(4, degree + 2), homogeneous Dirichlet data)
* mixed RT0 / P0  ``fem/scalar/operators.py:324-364`` (``rt0_operators``: the face
                    basis sign (x - opposite vertex) / (2 area), the inverse
                    permeability at the Duffy points), ``fem/hdiv/mixed.py:77-112``
                    (``normal_flux_blocks``), ``primal.py:80-103`` (kernel zero on the
                    fluxes and one on the pressures and multipliers, constraint the
                    cell areas over their total, coupling minus the flux map)
* condensation, contributions, assembly and the global SuperLU solve: the generic
  functions of ``oracle/q1_mhm.py``.

The macro and local topology, the P2 node numbering and the trace coupling come from
``pymhm_b200.polygon``, whose arrays the tests pin against the reference's own
(``tests/test_oracle_polygon.py``).
"""

from __future__ import annotations

import numpy as np
from scipy import sparse

from oracle import q1_mhm as q
from oracle.tetra_mhm import diffusion_blocks, triangle_quadrature
from pymhm_b200.polygon import (EdgeSkeleton, PolygonMesh, TriangleMesh, p2_nodal_space, p2_trace_coupling,
                                rt0_coupling)


def p1_geometry(mesh: TriangleMesh):
    """``p1_geometry`` (``operators.py:72-77``): barycentric gradients (cells, 3, 2)."""
    v = mesh.points[mesh.cells]
    mats = np.concatenate((np.ones((len(v), 3, 1)), v), axis=2)
    return np.linalg.inv(mats)[:, 1:, :].swapaxes(1, 2), mesh.areas


def p2_basis(bary):
    """P2 Lagrange values in PyMHM's node order (vertices, edges (0,1), (1,2), (2,0)) and
    their derivatives with respect to the three barycentric coordinates."""
    l0, l1, l2 = bary[:, 0], bary[:, 1], bary[:, 2]
    vals = np.column_stack((l0 * (2 * l0 - 1), l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), 4 * l0 * l1, 4 * l1 * l2,
                            4 * l2 * l0))
    d = np.zeros((len(bary), 6, 3))
    d[:, 0, 0] = 4 * l0 - 1
    d[:, 1, 1] = 4 * l1 - 1
    d[:, 2, 2] = 4 * l2 - 1
    d[:, 3, 0], d[:, 3, 1] = 4 * l1, 4 * l0
    d[:, 4, 1], d[:, 4, 2] = 4 * l2, 4 * l1
    d[:, 5, 2], d[:, 5, 0] = 4 * l0, 4 * l2
    return vals, d


def p2_operators(fine: TriangleMesh, permeability=1.0, source=0.0, order=4):
    """``scalar_operators`` for degree two with a scalar permeability and source."""
    bary, weights = triangle_quadrature(max(order, 4))
    dofs, nodes = p2_nodal_space(fine)
    grads_l, areas = p1_geometry(fine)
    vals, dl = p2_basis(bary)
    gradients = np.einsum("qna,tap->tqnp", dl, grads_l)  # (cells, q, 6, 2)
    physical = np.einsum("tqi,tij->tqj", np.broadcast_to(bary, (len(fine.cells), *bary.shape)),
                         fine.points[fine.cells])
    flat = physical.reshape(-1, 2)
    raw = permeability(flat) if callable(permeability) else permeability
    kap = np.broadcast_to(np.asarray(raw, dtype=float), (len(flat),)).reshape(physical.shape[:2])
    tensors = kap[:, :, None, None] * np.eye(2)
    stiffness = diffusion_blocks(weights, gradients, tensors, areas)
    mass = np.einsum("q,qi,qj,t->tij", weights, vals, vals, areas)
    rawf = source(flat) if callable(source) else source
    force = np.broadcast_to(np.asarray(rawf, dtype=float), (len(flat),)).reshape(physical.shape[:2])
    load = np.einsum("q,qi,tq,t->ti", weights, vals, force, areas)
    rows = np.repeat(dofs, 6, axis=1).ravel()
    cols = np.tile(dofs, (1, 6)).ravel()
    n = len(nodes)
    A = sparse.coo_matrix((stiffness.ravel(), (rows, cols)), shape=(n, n)).tocsc()
    M = sparse.coo_matrix((mass.ravel(), (rows, cols)), shape=(n, n)).tocsc()
    return A, M, np.bincount(dofs.ravel(), weights=load.ravel(), minlength=n)


def local_problem(coarse: PolygonMesh, skeleton: EdgeSkeleton, cell: int, fine: TriangleMesh, permeability, source):
    """``_DarcyLocalFactory.__call__``, primal, degree two (``primal.py:45-78``)."""
    A, M, f = p2_operators(fine, permeability, source)
    B = p2_trace_coupling(coarse, cell, fine, skeleton)
    mean = np.asarray(M @ np.ones((A.shape[0], 1)))
    constraints = mean / float(np.ones(A.shape[0]) @ mean[:, 0])
    return q.LocalProblem(A, B, f, skeleton.cell_dofs(cell), constraints)


def _samples(field, flat, shape):
    raw = field(flat) if callable(field) else field
    return np.broadcast_to(np.asarray(raw, dtype=float), (len(flat),)).reshape(shape)


def rt0_operators(fine: TriangleMesh, permeability=1.0, source=0.0, order=4):
    """``rt0_operators`` for a scalar permeability and source: the flux mass (faces x
    faces, K^-1 weighted), the signed divergence (cells x faces) and the P0 source
    moments."""
    bary, weights = triangle_quadrature(order)
    v = fine.points[fine.cells]
    physical = np.einsum("qi,tij->tqj", bary, v)
    flat = physical.reshape(-1, 2)
    kap = _samples(permeability, flat, physical.shape[:2])
    areas = fine.areas
    opposite = v[:, [2, 0, 1]]  # face s runs from vertex s to s + 1
    basis = (fine.signs[:, None, :, None] * (physical[:, :, None, :] - opposite[:, None, :, :])
             / (2 * areas)[:, None, None, None])
    blocks = np.einsum("q,tqia,tq,tqja,t->tij", weights, basis, 1.0 / kap, basis, areas)
    nf, nt = len(fine.faces), len(fine.cells)
    mass = sparse.coo_matrix((blocks.ravel(), (np.repeat(fine.cell_faces, 3, axis=1).ravel(),
                                               np.tile(fine.cell_faces, (1, 3)).ravel())), shape=(nf, nf)).tocsc()
    divergence = sparse.coo_matrix((fine.signs.ravel().astype(float),
                                    (np.repeat(np.arange(nt), 3), fine.cell_faces.ravel())), shape=(nt, nf)).tocsc()
    load = np.sum(_samples(source, flat, physical.shape[:2]) * weights, axis=1) * areas
    return mass, divergence, load


def mixed_local_problem(coarse: PolygonMesh, skeleton: EdgeSkeleton, cell: int, fine: TriangleMesh, permeability,
                        source):
    """``_DarcyLocalFactory.__call__``, mixed (``primal.py:80-103``) with
    ``normal_flux_blocks``: unknowns (fluxes, pressures, boundary multipliers)."""
    mass, div, force = rt0_operators(fine, permeability, source)
    nq, npres = len(fine.faces), len(fine.cells)
    bfaces = fine.boundary_faces
    nb = len(bfaces)
    sel = sparse.coo_matrix((np.ones(nb), (bfaces, np.arange(nb))), shape=(nq, nb)).tocsc()
    zero = sparse.csc_matrix((npres, nb))
    matrix = sparse.bmat([[mass, -div.T, sel], [-div, None, zero], [sel.T, zero.T, None]], format="csc")
    load = np.r_[np.zeros(nq), -force, np.zeros(nb)]
    kernel = np.r_[np.zeros(nq), np.ones(npres + nb)]
    mean = np.r_[np.zeros(nq), fine.areas, np.zeros(nb)]
    constraints = (mean / (kernel @ mean))[:, None]
    return q.LocalProblem(matrix, rt0_coupling(coarse, cell, fine, skeleton), load, skeleton.cell_dofs(cell),
                          constraints, kernel)


def solve_darcy_p2(coarse: PolygonMesh, skeleton: EdgeSkeleton, fines, permeability=1.0, source=0.0,
                   keep_responses=False, formulation="primal"):
    """``solve_darcy`` (``primal.py:173-344``) for degree two (or, ``formulation="mixed"``,
    RT0 / P0 with its negated boundary load, zero here), the given local meshes and
    homogeneous Dirichlet data.  Returns trace, coarse unknowns and fields per cell."""
    build = mixed_local_problem if formulation == "mixed" else local_problem
    responses, contribs = [], []
    for cell, fine in enumerate(fines):
        resp = q.condense(build(coarse, skeleton, cell, fine, permeability, source))
        contribs.append(q.contribution(resp, skeleton.size + cell))
        responses.append(resp)
    matrix, rhs, scale = q.assemble_global(contribs, skeleton.size, np.zeros(skeleton.size))
    x, residual = q.solve_global(matrix, rhs, scale)
    trace, coarse_u = x[: skeleton.size], x[skeleton.size:]
    fields = [r.source - r.lifts @ trace[r.problem.trace_dofs] + r.retained @ coarse_u[c: c + 1]
              for c, r in enumerate(responses)]
    corrected = np.array([r.coarse_vectors is not None for r in responses])
    return dict(trace=trace, coarse=coarse_u, fields=fields, matrix=matrix, rhs=rhs, residual=residual,
                corrected=corrected, responses=responses if keep_responses else [])
