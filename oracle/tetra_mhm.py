"""NumPy/SciPy restatement of PyMHM's 3D Primal-MHM path for P1 tetrahedra (the oracle).

Test infrastructure only: imported by ``tests/`` and ``bench.py``'s CPU arm, never by
``pymhm_b200``.  It follows PyMHM 1.3.2 (paths relative to ``src/pymhm/``):

* local operators     ``fem/scalar/tetrahedron.py:41-52, 157-190`` (Duffy rule of order
                      5, compensated diffusion blocks ``fem/scalar/_integration.py:43-88``)
* trace coupling      ``fem/traces/triangle_3d.py:221-273`` (3-point-per-direction Duffy
                      rule on every fine boundary triangle, Bernstein face modes)
* driver              ``_legacy/models/darcy/primal_3d.py:32-147`` (``_DarcyFactory``,
                      kernel 1, constraint M 1, homogeneous Dirichlet data)
* condensation, contributions, assembly and the global SuperLU solve: the generic
  functions of ``oracle/q1_mhm.py``.

The macro and fine topology (``TetraMesh``, its red refinement, the skeleton numbering)
is taken from ``pymhm_b200.tetra``, whose arrays the tests pin against the reference's
own (``tests/test_oracle_tetra.py``).
"""

from __future__ import annotations

import numpy as np
from scipy import sparse

from oracle import q1_mhm as q
from pymhm_b200.tetra import TetraMesh, TriangularSkeleton, duffy_tetrahedron


def _neumaier(total, corr, value):
    combined = total + value
    corr = corr + np.where(np.abs(total) >= np.abs(value), (total - combined) + value, (value - combined) + total)
    return combined, corr


def diffusion_blocks(weights, gradients, tensors, measures):
    """``diffusion_blocks`` (``_integration.py:43-88``) vectorised over cells, with a
    measure per cell.  gradients (cells, q, width, dim), tensors (cells, q, dim, dim)."""
    cells, count, width, dim = gradients.shape
    transformed = np.empty((cells, count, width, dim))
    for k in range(count):
        for j in range(width):
            for a in range(dim):
                t = np.zeros(cells)
                c = np.zeros(cells)
                for b in range(dim):
                    t, c = _neumaier(t, c, tensors[:, k, a, b] * gradients[:, k, j, b])
                transformed[:, k, j, a] = t + c
    out = np.empty((cells, width, width))
    for i in range(width):
        for j in range(width):
            t = np.zeros(cells)
            c = np.zeros(cells)
            for k in range(count):
                s = np.zeros(cells)
                sc = np.zeros(cells)
                for a in range(dim):
                    s, sc = _neumaier(s, sc, gradients[:, k, i, a] * transformed[:, k, j, a])
                t, c = _neumaier(t, c, (s + sc) * weights[k] * measures)
            out[:, i, j] = t + c
    return out


def barycentric_gradients(mesh: TetraMesh) -> np.ndarray:
    """``tetra_barycentric_gradients`` (``meshes/tetrahedron.py:161-166``): (cells, 4, 3)."""
    inverse = np.linalg.inv((mesh.points[mesh.cells[:, 1:]] - mesh.points[mesh.cells[:, :1]]).transpose(0, 2, 1))
    return np.concatenate((-inverse.sum(axis=1)[:, None], inverse), axis=1)


def p1_operators(fine: TetraMesh, permeability=1.0, source=0.0, order=5):
    """``tetra_operators`` for degree one (``tetrahedron.py:157-190``)."""
    bary, weights = duffy_tetrahedron(max(order, 3))
    grads = barycentric_gradients(fine)  # the P1 basis is the barycentric coordinates
    x = np.einsum("qi,tij->tqj", bary, fine.points[fine.cells])
    pts = x.reshape(-1, 3)
    raw = permeability(pts) if callable(permeability) else permeability
    kap = np.broadcast_to(np.asarray(raw, dtype=float), (len(pts),)).reshape(x.shape[:2])
    tensors = kap[:, :, None, None] * np.eye(3)
    g = np.broadcast_to(grads[:, None], (len(fine.cells), len(weights), 4, 3))
    stiffness = diffusion_blocks(weights, g, tensors, fine.volumes)
    mass = np.einsum("t,q,qi,qj->tij", fine.volumes, weights, bary, bary)
    rawf = source(pts) if callable(source) else source
    force = np.broadcast_to(np.asarray(rawf, dtype=float), (len(pts),)).reshape(x.shape[:2])
    load = np.einsum("t,q,qi,tq->ti", fine.volumes, weights, bary, force)
    dofs = fine.cells
    rows = np.broadcast_to(dofs[:, :, None], stiffness.shape).ravel()
    cols = np.broadcast_to(dofs[:, None, :], stiffness.shape).ravel()
    n = len(fine.points)
    A = sparse.coo_matrix((stiffness.ravel(), (rows, cols)), shape=(n, n)).tocsc()
    M = sparse.coo_matrix((mass.ravel(), (rows, cols)), shape=(n, n)).tocsc()
    f = np.zeros(n)
    np.add.at(f, dofs, load)
    return A, M, f


def triangle_quadrature(order):
    """``triangle_quadrature`` (``fem/scalar/operators.py:63-69``)."""
    t, w = np.polynomial.legendre.leggauss(order)
    t, w = (t + 1) / 2, w / 2
    bary = np.array([(1 - a - (1 - a) * b, a, (1 - a) * b) for a in t for b in t])
    weights = np.array([2 * wa * wb * (1 - a) for a, wa in zip(t, w) for wb in w])
    return bary, weights


def trace_coupling(coarse: TetraMesh, cell: int, fine: TetraMesh, skeleton: TriangularSkeleton):
    """``tetra_trace_coupling`` for P1 nodes, one subtriangle per face, Bernstein modes
    of degree 0 or 1 (``triangle_3d.py:221-273``)."""
    deg = skeleton.degree
    matrix = np.zeros((len(fine.points), 4 * skeleton.modes))
    verts = coarse.points[coarse.cells[cell]]
    jac = (verts[1:] - verts[:1]).T
    coords = (fine.points - verts[0]) @ np.linalg.inv(jac).T
    macro_bary = np.column_stack((1 - coords.sum(axis=1), coords))
    order = max(3, 2, (1 + deg + 3) // 2)
    bface, weights = triangle_quadrature(order)
    for side, face in enumerate(coarse.cell_faces[cell]):
        macro_vertices = [int(np.flatnonzero(coarse.cells[cell] == node)[0]) for node in coarse.faces[face]]
        for ff in fine.boundary_faces:
            ids = fine.faces[ff]
            if np.max(np.abs(macro_bary[ids, side])) > 1e-10:
                continue
            face_bary = macro_bary[ids][:, macro_vertices]  # (3 fine vertices, 3 face coordinates)
            # fine P1 values at the points: the fine face's own barycentric coordinates
            values = bface
            pts_face = bface @ face_bary  # macro face barycentric coordinates of the points
            if deg == 0:
                basis = np.ones((len(weights), 1))
            else:
                basis = pts_face  # Bernstein degree 1 = the barycentric coordinates
            block = coarse.signs[cell, side] * fine.areas[ff] * np.einsum("q,qi,qj->ij", weights, values, basis)
            matrix[np.ix_(ids, skeleton.modes * side + np.arange(skeleton.modes))] += block
    return matrix


def local_problem(coarse, skeleton, cell, refinement, permeability, source):
    """``_DarcyFactory.__call__`` for degree one (``primal_3d.py:45-66``)."""
    fine = coarse.submesh(cell, refinement)
    A, M, f = p1_operators(fine, permeability, source)
    B = trace_coupling(coarse, cell, fine, skeleton)
    constraints = np.asarray(M @ np.ones((A.shape[0], 1)))
    return fine, q.LocalProblem(A, B, f, skeleton.cell_dofs(cell), constraints)


def solve_darcy_p1(coarse, skeleton, refinement, permeability=1.0, source=0.0, keep_responses=False):
    """``solve_darcy_3d`` with degree one and homogeneous Dirichlet data
    (``primal_3d.py:68-147``).  Returns trace, coarse unknowns, fields per cell."""
    responses, contribs = [], []
    for cell in range(len(coarse.cells)):
        _, prob = local_problem(coarse, skeleton, cell, refinement, permeability, source)
        resp = q.condense(prob)
        contribs.append(q.contribution(resp, skeleton.size + cell))
        responses.append(resp)
    matrix, rhs, scale = q.assemble_global(contribs, skeleton.size, np.zeros(skeleton.size))
    x, residual = q.solve_global(matrix, rhs, scale)
    trace, coarse_u = x[: skeleton.size], x[skeleton.size:]
    fields = np.array([r.source - r.lifts @ trace[r.problem.trace_dofs] + r.retained @ coarse_u[c: c + 1]
                       for c, r in enumerate(responses)])
    corrected = np.array([r.coarse_vectors is not None for r in responses])
    return dict(trace=trace, coarse=coarse_u, fields=fields, matrix=matrix, rhs=rhs, residual=residual,
                corrected=corrected, responses=responses if keep_responses else [])
