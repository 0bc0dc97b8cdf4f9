"""NumPy/SciPy restatement of PyMHM's Cartesian Q1 Primal-MHM path (the oracle).

Test infrastructure only: imported by ``tests/``, ``__graft_entry__.smoke`` and
the CPU arm of ``bench.py``.  It is the checker for the CUDA path and is never
called by ``pymhm_b200``.

Every function follows the reference algorithm of PyMHM 1.3.2; paths below are
relative to ``src/pymhm/`` of that project:

* topology            ``meshes/cartesian.py:31-144``
* skeleton spaces     ``fem/traces/interval.py:13-161``
* Q1 tables/operators ``fem/scalar/quadrilateral.py:25-113, 191-298``
* diffusion Gram      ``fem/scalar/_integration.py:32-88`` (Neumaier sums)
* boundary data       ``fem/scalar/operators.py:247-321``
* local contract      ``core/contracts.py:37-211``
* condensation        ``core/condensation.py:118-191``
* equilibrated LU     ``linalg/linear.py:98-152, 262-310, 400-422``
* contributions       ``core/contributions.py:14-195``, ``core/_assembly.py``
* reduced load        ``core/reconstruction.py:91-141``
* global solve        ``core/system.py:355-528``
* flux samples        ``postprocessing/solutions.py:278-324``

Parity is pinned against fixtures written by the reference itself; see
``tests/test_oracle_golden.py``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import fsum

import numpy as np
from numpy.polynomial.legendre import leggauss
from scipy import sparse
from scipy.sparse import linalg as splinalg

EPS = np.finfo(float).eps


class LinearSolveError(RuntimeError):
    """Mirror of ``linalg/linear.py:32`` (factorization or residual failure)."""


# --------------------------------------------------------------------------------------
# Topology: meshes/cartesian.py:31-108 (face IDs by first encounter in ccw row-major cells)
# --------------------------------------------------------------------------------------
@dataclass
class CartesianMesh:
    nx: int
    ny: int
    bounds: tuple
    points: np.ndarray = field(repr=False)
    cells: np.ndarray = field(repr=False)
    faces: np.ndarray = field(repr=False)
    cell_faces: np.ndarray = field(repr=False)
    signs: np.ndarray = field(repr=False)
    face_cells: np.ndarray = field(repr=False)

    @property
    def spacing(self):
        x0, x1, y0, y1 = self.bounds
        return np.array([(x1 - x0) / self.nx, (y1 - y0) / self.ny])

    @property
    def lengths(self):
        return np.linalg.norm(self.points[self.faces[:, 1]] - self.points[self.faces[:, 0]], axis=1)

    @property
    def boundary_faces(self):
        return np.flatnonzero(self.face_cells[:, 1] == -1)

    def submesh(self, cell, subdivisions):
        """``meshes/cartesian.py:137-144``."""
        rx, ry = (subdivisions, subdivisions) if np.isscalar(subdivisions) else subdivisions
        lower, upper = self.points[self.cells[cell, [0, 2]]]
        return cartesian_mesh(rx, ry, (lower[0], upper[0], lower[1], upper[1]))


def cartesian_mesh(nx, ny=None, bounds=(0.0, 1.0, 0.0, 1.0)):
    """Restates ``CartesianMacroMesh.__post_init__`` (``meshes/cartesian.py:31-108``).

    Faces are numbered by first encounter while visiting cells row-major, each
    cell's sides counterclockwise (bottom, right, top, left); a face is oriented
    along its first cell's counterclockwise traversal and carries sign +1 there
    and -1 in the second cell.
    """
    ny = nx if ny is None else ny
    x0, x1, y0, y1 = (float(v) for v in bounds)
    x, y = np.linspace(x0, x1, nx + 1), np.linspace(y0, y1, ny + 1)
    points = np.column_stack((np.tile(x, ny + 1), np.repeat(y, nx + 1)))
    cells = np.empty((nx * ny, 4), dtype=np.int64)
    nfaces = (ny + 1) * nx + (nx + 1) * ny
    faces = np.empty((nfaces, 2), dtype=np.int64)
    face_cells = np.full((nfaces, 2), -1, dtype=np.int64)
    cell_faces = np.empty((nx * ny, 4), dtype=np.int64)
    signs = np.empty((nx * ny, 4), dtype=np.int64)
    seen = {}
    for j in range(ny):
        for i in range(nx):
            c = j * nx + i
            a = j * (nx + 1) + i
            ring = (a, a + 1, a + nx + 2, a + nx + 1)
            cells[c] = ring
            for side in range(4):
                u, v = ring[side], ring[(side + 1) % 4]
                key = (min(u, v), max(u, v))
                if key in seen:
                    f = seen[key]
                    face_cells[f, 1] = c
                    signs[c, side] = -1
                else:
                    f = len(seen)
                    seen[key] = f
                    faces[f] = (u, v)
                    face_cells[f, 0] = c
                    signs[c, side] = 1
                cell_faces[c, side] = f
    return CartesianMesh(nx, ny, (x0, x1, y0, y1), points, cells, faces, cell_faces, signs,
                         face_cells)


# --------------------------------------------------------------------------------------
# Skeleton: fem/traces/interval.py:13-161 (discontinuous Legendre / continuous nodal faces)
# --------------------------------------------------------------------------------------
def legendre_values(x, degree):
    """Conventional Legendre L_0..L_degree with L_j(1)=1 (three-term recurrence).

    Stands in for ``fem/reference.py:596-625`` (Basix orthonormal set rescaled).
    """
    x = np.asarray(x, dtype=float)
    out = np.empty((*x.shape, degree + 1))
    out[..., 0] = 1.0
    if degree >= 1:
        out[..., 1] = x
    for j in range(1, degree):
        out[..., j + 1] = ((2 * j + 1) * x * out[..., j] - j * out[..., j - 1]) / (j + 1)
    return out


def lagrange_interval(degree, points, nodes):
    """Nodal interval basis on declared ``nodes`` with Kronecker rows at literal nodes.

    Stands in for ``simplex_lagrange_tabulation("interval", ...)``
    (``fem/reference.py:497-540``); derivatives are returned as a second array.
    """
    x = np.asarray(points, dtype=float)
    c = np.asarray(nodes, dtype=float)
    vals = np.ones((len(x), len(c)))
    ders = np.zeros((len(x), len(c)))
    for i in range(len(c)):
        others = [m for m in range(len(c)) if m != i]
        denom = np.prod([c[i] - c[m] for m in others])
        for m in others:
            vals[:, i] *= (x - c[m])
        vals[:, i] /= denom
        for skip in others:
            term = np.ones(len(x))
            for m in others:
                if m != skip:
                    term *= (x - c[m])
            ders[:, i] += term / denom
    rows, cols = np.nonzero(x[:, None] == c[None, :])
    vals[rows] = 0.0
    vals[rows, cols] = 1.0
    return vals, ders


@dataclass(frozen=True)
class FaceSpace:
    """``fem/traces/interval.py:13-116``."""

    breaks: tuple = (0.0, 1.0)
    degrees: tuple = (0,)
    continuous: bool = False

    @classmethod
    def uniform(cls, degree=0, subdivisions=1, continuous=False):
        return cls(tuple(float(v) for v in np.linspace(0, 1, subdivisions + 1)),
                   (degree,) * subdivisions, continuous)

    @property
    def size(self):
        return 1 + sum(self.degrees) if self.continuous else sum(p + 1 for p in self.degrees)

    def evaluate(self, parameter):
        """``interval.py:54-89``."""
        t = np.atleast_1d(np.asarray(parameter, dtype=float))
        values = np.zeros((len(t), self.size))
        offset = 0
        for i, degree in enumerate(self.degrees):
            lo, hi = self.breaks[i: i + 2]
            mask = (t >= lo) & ((t < hi) | ((i == len(self.degrees) - 1) & (t <= hi)))
            local = (t[mask] - lo) / (hi - lo)
            if self.continuous:
                nodes = np.r_[0.0, 1.0, np.arange(1, degree) / degree]
                basis, _ = lagrange_interval(degree, local, nodes)
                ids = np.r_[i, i + 1, len(self.breaks) + offset + np.arange(degree - 1)]
                values[np.ix_(mask, ids)] = basis
                offset += degree - 1
            else:
                values[mask, offset: offset + degree + 1] = legendre_values(2 * local - 1, degree)
                offset += degree + 1
        return values

    def quadrature(self, order=4):
        """``interval.py:99-116`` (weights renormalised to mass two in long double)."""
        x, w = leggauss(order)
        w = np.asarray(w, dtype=np.longdouble)
        w *= np.longdouble(2) / np.sum(w)
        points, weights = [], []
        for lo, hi in zip(self.breaks[:-1], self.breaks[1:]):
            points.extend(lo + (x + 1) * (hi - lo) / 2)
            weights.extend(w * (hi - lo) / 2)
        return np.asarray(points), np.asarray(weights, dtype=float)


@dataclass
class Skeleton:
    """``SkeletonSpace`` (``interval.py:119-161``) for scalar traces."""

    mesh: CartesianMesh
    faces: tuple
    offsets: np.ndarray = field(init=False)

    def __post_init__(self):
        self.offsets = np.r_[0, np.cumsum([f.size for f in self.faces])].astype(np.int64)

    @property
    def size(self):
        return int(self.offsets[-1])

    def dofs(self, face):
        return np.arange(self.offsets[face], self.offsets[face + 1])

    def cell_dofs(self, cell):
        return np.concatenate([self.dofs(int(f)) for f in self.mesh.cell_faces[cell]])


# --------------------------------------------------------------------------------------
# Q1 operators: fem/scalar/quadrilateral.py:25-113, 191-298
# --------------------------------------------------------------------------------------
def quadrature(order=4):
    """``quadrilateral_quadrature`` (``quadrilateral.py:25-32``)."""
    p, w = leggauss(order)
    p, w = (p + 1) / 2, w / 2
    return (np.array([(x, y) for y in p for x in p]),
            np.array([wx * wy for wy in w for wx in w]))


def q1_basis(points):
    """``qk_basis`` for degree one (``quadrilateral.py:71-94``), x-fastest ordering."""
    x, dx = lagrange_interval(1, points[:, 0], [0.0, 1.0])
    y, dy = lagrange_interval(1, points[:, 1], [0.0, 1.0])
    basis = np.einsum("qi,qj->qij", y, x).reshape(len(points), 4)
    grad = np.stack((np.einsum("qi,qj->qij", y, dx), np.einsum("qi,qj->qij", dy, x)), axis=-1)
    return basis, grad.reshape(len(points), 4, 2)


def q1_space(mesh):
    """``qk_space`` for degree one (``quadrilateral.py:97-113``)."""
    nx, ny = mesh.nx, mesh.ny
    x0, x1, y0, y1 = mesh.bounds
    nodes = np.array([(x, y) for y in np.linspace(y0, y1, ny + 1) for x in np.linspace(x0, x1, nx + 1)])
    local = np.array([0, 1, nx + 1, nx + 2])
    origin = np.array([j * (nx + 1) + i for j in range(ny) for i in range(nx)])
    return (origin[:, None] + local).astype(np.int64), nodes


def _neumaier(total, corr, value):
    """``_compensated_add`` (``_integration.py:32-40``), vectorised."""
    combined = total + value
    corr = corr + np.where(np.abs(total) >= np.abs(value), (total - combined) + value,
                           (value - combined) + total)
    return combined, corr


def diffusion_blocks(weights, gradients, tensors, measure):
    """``diffusion_blocks`` (``_integration.py:43-88``), vectorised over cells.

    Shapes: weights (q,) or per cell (cells,q), gradients (q,4,2) or (cells,q,4,2),
    tensors (cells,q,2,2), measure scalar.
    """
    cells, count = tensors.shape[:2]
    weights = np.broadcast_to(weights, (cells, count))
    gradients = np.broadcast_to(gradients, (cells, *gradients.shape[-3:]))
    width, dim = gradients.shape[2:]
    transformed = np.empty((cells, count, width, dim))
    for q in range(count):
        for j in range(width):
            for a in range(dim):
                t = np.zeros(cells)
                c = np.zeros(cells)
                for b in range(dim):
                    t, c = _neumaier(t, c, tensors[:, q, a, b] * gradients[:, q, j, b])
                transformed[:, q, j, a] = t + c
    result = np.empty((cells, width, width))
    for i in range(width):
        for j in range(width):
            t = np.zeros(cells)
            c = np.zeros(cells)
            for q in range(count):
                s = np.zeros(cells)
                sc = np.zeros(cells)
                for a in range(dim):
                    s, sc = _neumaier(s, sc, gradients[:, q, i, a] * transformed[:, q, j, a])
                t, c = _neumaier(t, c, (s + sc) * weights[:, q] * measure)
            result[:, i, j] = t + c
    return result


def tensor_at(permeability, pts):
    """Scalar or callable permeability as (n,2,2) tensors (``materials/evaluation.py:43``)."""
    raw = permeability(pts) if callable(permeability) else permeability
    value = np.asarray(raw, dtype=float)
    if value.ndim == 0 or value.shape == (len(pts),):
        return np.broadcast_to(value, (len(pts),))[:, None, None] * np.eye(2)
    return np.broadcast_to(value, (len(pts), 2, 2)).copy()


def scalar_at(source, pts):
    raw = source(pts) if callable(source) else source
    return np.broadcast_to(np.asarray(raw, dtype=float), (len(pts),)).copy()


class PixelField:
    """Grid-aligned piecewise-constant field (``materials/cartesian.py:14-72``).

    ``values[ix, iy]`` holds the value of pixel (ix, iy); points on a pixel
    boundary take the pixel on their positive side, clipped at the upper edge.
    """

    def __init__(self, values, spacing, origin=(0.0, 0.0)):
        self.values = np.asarray(values, dtype=float)
        self.spacing = np.asarray(spacing, dtype=float)
        self.origin = np.asarray(origin, dtype=float)

    def __call__(self, pts):
        coords = (np.asarray(pts) - self.origin) / self.spacing
        levels = np.rint(coords)
        coords = np.where(np.abs(coords - levels) <= 4 * EPS * np.maximum(1, np.abs(coords)),
                          levels, coords)
        shape = np.asarray(self.values.shape[:2])
        idx = np.minimum(np.maximum(coords, 0).astype(np.int64), shape - 1)
        return self.values[idx[:, 0], idx[:, 1]]


def grid_resolves_material(fine, field):
    """``grid_resolves_material`` (``quadrilateral.py:116-132``): every pixel line lies on a
    fine-grid line (pixel spacing an integer multiple of the fine spacing, origin offset
    an integer number of fine cells), to 64 eps of the compared values."""
    spacing = np.asarray(fine.spacing, dtype=float)
    intervals = np.asarray(field.spacing, dtype=float) / spacing
    bounds = np.asarray(fine.bounds, dtype=float)
    offsets = (bounds[[0, 2]] - np.asarray(field.origin, dtype=float)) / spacing
    values = np.r_[intervals, offsets]
    tolerance = 64 * EPS * max(1.0, float(np.max(np.abs(values))))
    return bool(np.all(np.abs(values - np.rint(values)) <= tolerance))


def rectangle_intersection_quadrature(origins, spacing, field, order):
    """``rectangle_intersection_quadrature`` (``quadrilateral.py:136-188``): per fine cell,
    tensor Gauss rules on its exact intersections with the pixels, in the cell's
    reference coordinates; zero-weight padding to a common point count."""
    pixel_spacing = np.asarray(field.spacing, dtype=float)
    pixel_origin = np.asarray(field.origin, dtype=float)
    shape = np.asarray(field.values.shape[:2])
    lower = (origins - pixel_origin) / pixel_spacing
    upper = (origins + spacing - pixel_origin) / pixel_spacing
    tolerance = 64 * EPS * shape
    if np.any(lower < -tolerance) or np.any(upper > shape + tolerance):
        raise ValueError("a fine rectangle lies outside the Cartesian material field")
    lower = np.where(np.isclose(lower, np.rint(lower), rtol=0, atol=tolerance), np.rint(lower), lower)
    upper = np.where(np.isclose(upper, np.rint(upper), rtol=0, atol=tolerance), np.rint(upper), upper)
    first = np.floor(lower).astype(int)
    last = np.ceil(upper).astype(int) - 1
    parts = np.max(last - first + 1, axis=0)
    gauss, weights = leggauss(order)
    gauss, weights = (gauss + 1) / 2, weights / 2
    axes, axis_weights = [], []
    for axis in range(2):
        indices = first[:, axis, None] + np.arange(parts[axis])
        physical_lo = pixel_origin[axis] + indices * pixel_spacing[axis]
        physical_hi = pixel_origin[axis] + (indices + 1) * pixel_spacing[axis]
        end = origins[:, axis, None] + spacing[axis]
        lo = np.minimum(np.maximum(physical_lo, origins[:, axis, None]), end)
        hi = np.maximum(np.minimum(physical_hi, end), lo)
        a = (lo - origins[:, axis, None]) / spacing[axis]
        width = (hi - lo) / spacing[axis]
        axes.append(a[..., None] + width[..., None] * gauss)
        axis_weights.append(width[..., None] * weights)
    count = len(origins)
    x = np.broadcast_to(axes[0][:, None, None, :, :], (count, parts[1], order, parts[0], order))
    y = np.broadcast_to(axes[1][:, :, :, None, None], x.shape)
    combined = axis_weights[1][:, :, :, None, None] * axis_weights[0][:, None, None, :, :]
    reference = np.stack((x, y), axis=-1).reshape(count, -1, 2)
    return np.clip(reference, 0, 1), combined.reshape(count, -1)


def q1_operators(fine, permeability=1.0, source=0.0, order=4):
    """``quadrilateral_operators`` (``quadrilateral.py:191-253``): the uniform rule, or the
    cut rule when the pixel lines of a ``PixelField`` cross the fine cells."""
    reference, weights = quadrature(order)
    dofs, nodes = q1_space(fine)
    basis, gradient = q1_basis(reference)
    gradient = gradient / fine.spacing
    area = float(np.prod(fine.spacing))
    n = len(nodes)
    cuts = isinstance(permeability, PixelField) and not grid_resolves_material(fine, permeability)
    blocks, loads = [], []
    for begin in range(0, len(fine.cells), 256):
        origins = fine.points[fine.cells[begin: begin + 256, 0]]
        if cuts:
            cref, cw = rectangle_intersection_quadrature(origins, np.asarray(fine.spacing, float), permeability,
                                                         order)
            cb, cg = q1_basis(cref.reshape(-1, 2))
            cb = cb.reshape(len(origins), -1, 4)
            cg = cg.reshape(len(origins), -1, 4, 2) / fine.spacing
            pts = origins[:, None, :] + cref * fine.spacing
            tensors = tensor_at(permeability, pts.reshape(-1, 2)).reshape(len(origins), -1, 2, 2)
            force = scalar_at(source, pts.reshape(-1, 2)).reshape(len(origins), -1)
            blocks.append(diffusion_blocks(cw, cg, tensors, area))
            loads.append(area * np.einsum("tq,tqi,tq->ti", cw, cb, force))
            continue
        pts = origins[:, None, :] + reference[None, :, :] * fine.spacing
        tensors = tensor_at(permeability, pts.reshape(-1, 2)).reshape(len(origins), len(weights), 2, 2)
        force = scalar_at(source, pts.reshape(-1, 2)).reshape(len(origins), len(weights))
        blocks.append(diffusion_blocks(weights, gradient, tensors, area))
        loads.append(area * np.einsum("q,qi,tq->ti", weights, basis, force))
    row = np.repeat(dofs, 4, axis=1).ravel()
    col = np.tile(dofs, (1, 4)).ravel()
    matrix = sparse.coo_matrix((np.concatenate(blocks).ravel(), (row, col)), shape=(n, n)).tocsc()
    mass_block = area * np.einsum("q,qi,qj->ij", weights, basis, basis)
    mass = sparse.coo_matrix((np.tile(mass_block.ravel(), len(dofs)), (row, col)), shape=(n, n)).tocsc()
    load = np.bincount(dofs.ravel(), weights=np.concatenate(loads).ravel(), minlength=n)
    return matrix, mass, load


def side_parameters(coarse, cell, fine):
    """Fine boundary node ids per side and their oriented face coordinates.

    Follows the geometry of ``quadrilateral_trace_coupling`` (``quadrilateral.py:256-278``).
    """
    _, nodes = q1_space(fine)
    nx, ny = fine.nx, fine.ny
    edge_nodes = (np.arange(nx + 1), np.arange(ny + 1) * (nx + 1) + nx,
                  ny * (nx + 1) + np.arange(nx + 1), np.arange(ny + 1) * (nx + 1))
    out = []
    for side, face in enumerate(coarse.cell_faces[cell]):
        ids = edge_nodes[side]
        start, end = coarse.points[coarse.faces[face]]
        tangent = end - start
        length = coarse.lengths[face]
        out.append((ids, (nodes[ids] - start) @ tangent / length ** 2, length))
    return out


def trace_coupling(coarse, cell, fine, skeleton):
    """``quadrilateral_trace_coupling`` for degree one (``quadrilateral.py:256-298``)."""
    _, nodes = q1_space(fine)
    width = sum(skeleton.faces[f].size for f in coarse.cell_faces[cell])
    matrix = np.zeros((len(nodes), width))
    offset = 0
    for side, (face, (ids, tnodes, length)) in enumerate(
            zip(coarse.cell_faces[cell], side_parameters(coarse, cell, fine))):
        space = skeleton.faces[face]
        gauss, w = leggauss(max(space.degrees) + 1 + 1)
        for begin in range(0, len(ids) - 1):
            idx = ids[begin: begin + 2]
            t0, t1 = tnodes[begin], tnodes[begin + 1]
            lo, hi = sorted((float(t0), float(t1)))
            cuts = sorted({lo, hi, *(b for b in space.breaks if lo < b < hi)})
            for left, right in zip(cuts[:-1], cuts[1:]):
                parameter = left + (gauss + 1) * (right - left) / 2
                s = (parameter - t0) / (t1 - t0)
                local_basis, _ = lagrange_interval(1, s, [0.0, 1.0])
                weights = w * (right - left) / 2 * length * coarse.signs[cell, side]
                matrix[idx, offset: offset + space.size] += local_basis.T @ (
                    weights[:, None] * space.evaluate(parameter))
        offset += space.size
    return matrix


def boundary_data(skeleton, dirichlet=0.0, neumann=None, order=4):
    """``boundary_data`` for scalar skeletons (``fem/scalar/operators.py:247-321``)."""
    neumann = {} if neumann is None else neumann
    load = np.zeros(skeleton.size)
    fixed = {}
    mesh = skeleton.mesh
    for face in mesh.boundary_faces:
        space = skeleton.faces[face]
        parameter, weights = space.quadrature(max(order, max(space.degrees) + 2))
        start, end = mesh.points[mesh.faces[face]]
        pts = start + parameter[:, None] * (end - start)
        basis = space.evaluate(parameter)
        values = scalar_at(neumann[face] if face in neumann else dirichlet, pts)
        moments = np.empty(basis.shape[1])
        for i in range(basis.shape[1]):  # boundary_moments (_integration.py:91-108)
            t = np.zeros(())
            c = np.zeros(())
            for q in range(len(weights)):
                t, c = _neumaier(t, c, basis[q, i] * weights[q] * values[q])
            moments[i] = t + c
        dofs = skeleton.dofs(int(face))
        if face in neumann:
            coef = np.linalg.solve(basis.T @ (weights[:, None] * basis), moments)
            fixed.update(zip(dofs.tolist(), coef.tolist()))
        else:
            load[dofs] = moments * mesh.lengths[face]
    return load, fixed


# --------------------------------------------------------------------------------------
# Local contract, condensation and checked LU: core/contracts.py, core/condensation.py,
# linalg/linear.py
# --------------------------------------------------------------------------------------
def accurate_residual(matrix, rhs, solution):
    """``accurate_residual`` (``linalg/linear.py:98-126``), long-double branch."""
    prec = np.longdouble
    return np.asarray(rhs, dtype=prec) - matrix.astype(prec) @ np.asarray(solution, dtype=prec)


def matrix_action(matrix, values):
    """``_matrix_action`` (``core/contracts.py:37-52``)."""
    return np.asarray(-accurate_residual(matrix.tocsr(), np.zeros((matrix.shape[0], *values.shape[1:])),
                                         values), dtype=float)


class ResidualFailure(LinearSolveError):
    pass


def checked(matrix, rhs, result, rtol=1e-10, atol=0.0):
    """``_checked`` (``linalg/linear.py:132-152``)."""
    solution = np.asarray(result)
    if solution.shape != rhs.shape or not np.all(np.isfinite(solution)):
        raise LinearSolveError("solver returned a nonfinite solution or an incompatible shape")
    difference = matrix @ solution - rhs
    scale = np.maximum(atol, np.max(np.abs(rhs), axis=0))
    scale = np.where(scale > 0, scale, 1.0)
    residual = np.linalg.norm(difference / scale, axis=0)
    threshold = np.maximum(atol / scale, rtol * np.linalg.norm(rhs / scale, axis=0))
    if np.any(residual > threshold):
        residual = np.linalg.norm(np.asarray(accurate_residual(matrix, rhs, solution), dtype=float) / scale,
                                  axis=0)
    if np.any(residual > threshold):
        raise ResidualFailure(f"residual criterion failed: scaled ||Ax-b||={residual}, allowed={threshold}")
    return solution


class EquilibratedLU:
    """``factorize(solver='scipy')`` + ``LinearFactorization.solve`` (``linalg/linear.py:240-331, 400-422``)."""

    def __init__(self, matrix, rtol=1e-10):
        op = sparse.csr_matrix(matrix, dtype=float, copy=True)
        op.sum_duplicates()
        op.sort_indices()
        self.matrix = op
        self.rtol = rtol
        row = np.asarray(abs(op).max(axis=1).toarray()).ravel()
        if np.any(row == 0):
            raise LinearSolveError("SuperLU factorization failed: matrix has a zero row")
        bal = op.copy()
        bal.data /= np.repeat(row, np.diff(bal.indptr))
        col = np.asarray(abs(bal).max(axis=0).toarray()).ravel()
        if np.any(col == 0):
            raise LinearSolveError("SuperLU factorization failed: matrix has a zero column")
        bal.data /= col[bal.indices]
        try:
            self.lu = splinalg.splu(bal.tocsc())
        except RuntimeError as exc:
            raise LinearSolveError(f"SuperLU factorization failed: {exc}") from exc
        piv = np.abs(self.lu.U.diagonal())
        if np.min(piv) <= EPS * op.shape[0] * np.max(np.abs(self.lu.U.data)):
            raise LinearSolveError("SuperLU factorization has insufficient numerical rank after equilibration")
        self.row, self.col = row, col

    def _apply(self, rhs):
        r = self.row[:, None] if rhs.ndim == 2 else self.row
        c = self.col[:, None] if rhs.ndim == 2 else self.col
        return np.asarray(self.lu.solve(rhs / r) / c)

    def solve(self, rhs, steps=2):
        forcing = np.asarray(rhs, dtype=float)
        result = self._apply(forcing)
        for _ in range(steps):
            try:
                return checked(self.matrix, forcing, result, self.rtol)
            except ResidualFailure:
                residual = np.asarray(accurate_residual(self.matrix, forcing, result), dtype=float)
                result = result + self._apply(residual)
        return checked(self.matrix, forcing, result, self.rtol)


@dataclass
class LocalProblem:
    """``LocalProblem`` (``core/contracts.py:92-211``) with one declared kernel vector Z
    (``kernel``; default the ones vector, the primal problems; the mixed RT0 problems
    declare zero fluxes and unit pressures) and C = M Z scaled as the driver gives it."""

    matrix: sparse.csc_matrix
    coupling: np.ndarray
    load: np.ndarray
    trace_dofs: np.ndarray
    constraints: np.ndarray
    kernel: np.ndarray | None = None
    action: np.ndarray = field(init=False)
    test_action: np.ndarray = field(init=False)
    corrected: bool = field(init=False)

    def __post_init__(self):
        n = self.matrix.shape[0]
        self.kernel = np.ones((n, 1)) if self.kernel is None else np.asarray(self.kernel, dtype=float).reshape(n, 1)
        kernel = self.kernel
        scale = float(np.max(np.abs(self.matrix.data), initial=0.0))
        if scale:
            normalized = self.matrix.copy()
            normalized.data /= scale
            norm = float(splinalg.norm(normalized))
            kernel = kernel / np.max(np.abs(kernel), axis=0)
            ref = norm * np.linalg.norm(kernel, axis=0)
            for op in (normalized, normalized.T):
                if np.any(np.linalg.norm(op @ kernel, axis=0) > 1e-10 * ref):
                    raise ValueError("declared kernel is not a left and right nullspace")
        self.action = matrix_action(self.matrix, self.kernel)
        self.test_action = matrix_action(self.matrix.T, self.kernel)
        self.corrected = bool(np.any(self.action) or np.any(self.test_action))

    def condensation_system(self):
        """``local_condensation_system`` / ``local_condensation_matrix`` (``condensation.py:125-174``)."""
        n = self.matrix.shape[0]
        scale = float(np.max(np.abs(self.matrix.data), initial=0.0)) or 1.0
        c = self.constraints * np.minimum(1.0, scale / np.max(np.abs(self.constraints), axis=0))
        aug = sparse.bmat([[self.matrix, sparse.csc_matrix(c)], [sparse.csc_matrix(c.T), None]],
                          format="csc")
        width = self.coupling.shape[1] + 1
        rhs = np.zeros((n + 1, width + (1 if self.corrected else 0)))
        rhs[:n, 0] = self.load
        rhs[:n, 1:width] = self.coupling
        if self.corrected:
            rhs[:n, width:] = self.action
        return aug, rhs


@dataclass
class LocalResponse:
    problem: LocalProblem
    source: np.ndarray
    lifts: np.ndarray
    coarse_vectors: np.ndarray | None

    @property
    def retained(self):
        return self.problem.kernel if self.coarse_vectors is None else self.coarse_vectors


def condense(problem: LocalProblem):
    """``condense_local`` direct branch + ``local_response_from_solution`` (``condensation.py:118-191``)."""
    aug, rhs = problem.condensation_system()
    sol = EquilibratedLU(aug).solve(rhs)
    n = problem.matrix.shape[0]
    width = problem.coupling.shape[1] + 1
    x = sol[:n]
    coarse = problem.kernel - x[:, width:] if problem.corrected else None
    return LocalResponse(problem, x[:, 0], x[:, 1:width], coarse)


def contribution(resp: LocalResponse, coarse_dof: int):
    """``local_global_contribution`` + ``local_condensed_load`` (``contributions.py:14-74``, ``reconstruction.py:91-127``)."""
    p = resp.problem
    z = p.kernel
    e = resp.retained
    g = p.coupling.T @ e
    if resp.coarse_vectors is None:
        coarse_trace = z.T @ p.coupling
        coarse_matrix = np.zeros((1, 1))
        coarse_rhs = -z.T @ p.load
    else:
        coarse_trace = z.T @ p.coupling - p.test_action.T @ resp.lifts
        coarse_matrix = p.test_action.T @ e
        coarse_rhs = p.test_action.T @ resp.source - z.T @ p.load
    block = np.block([[p.coupling.T @ resp.lifts, -g], [-coarse_trace, -coarse_matrix]])
    load = np.concatenate((p.coupling.T @ resp.source, coarse_rhs))
    return np.r_[p.trace_dofs, coarse_dof].astype(np.int64), block, load


def assemble_global(contribs, trace_size, boundary_load=None):
    """``assemble_hybrid_contributions`` (``contributions.py:77-195``, ``_assembly.py``)."""
    size = trace_size + len(contribs)
    rhs = np.zeros(size)
    scale = np.zeros(size)
    rows, cols, vals = [], [], []
    for idx, block, load in contribs:
        rows.append(np.repeat(idx, len(idx)))
        cols.append(np.tile(idx, len(idx)))
        vals.append(block.ravel())
        for i in range(len(idx)):  # accumulate_load, ordered
            rhs[idx[i]] += load[i]
            scale[idx[i]] += abs(load[i])
    matrix = sparse.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                               shape=(size, size)).tocsc()
    matrix.eliminate_zeros()
    if boundary_load is not None:
        rhs[:trace_size] -= boundary_load
        scale[:trace_size] += np.abs(boundary_load)
    return matrix, rhs, scale


def mean_constraint(responses, trace_size, weights, value):
    """``hybrid_mean_constraint`` (``core/system.py:531-566``): the row r and target b
    of sum_cells w_c . u_c = value, u_c = source - lifts lambda + retained c."""
    row = np.zeros(trace_size + len(responses))
    target = float(value)
    for c, (r, w) in enumerate(zip(responses, weights)):
        np.add.at(row, r.problem.trace_dofs, -r.lifts.T @ w)
        row[trace_size + c] = (r.retained.T @ w)[0]
        target -= w @ r.source
    return row, target


def solve_global(matrix, rhs, load_scale, rtol=1e-10, fixed=None, constraints=None):
    """``solve_hybrid_system`` (``core/system.py:355-528``): fixed trace DOFs take their
    prescribed values and leave the system, whose other rows lose the prescribed
    action (``:421-447``); constraint rows r.x = b border it with multipliers
    (``:448-457``), the residual check reading the physical rows only."""
    fixed = {} if fixed is None else fixed
    n = len(rhs)
    x = np.zeros(n)
    idx = np.array(sorted(fixed), dtype=np.int64)
    x[idx] = [fixed[i] for i in idx]
    free = np.setdiff1d(np.arange(n), idx)
    reduced = matrix[free][:, free] if len(idx) else matrix
    action = (matrix @ x)[free]
    rrhs = rhs[free] - action
    if constraints:
        rows = np.array([row for row, _ in constraints])
        targets = np.array([t for _, t in constraints]) - rows @ x
        bordered = sparse.bmat([[sparse.csc_matrix(reduced), sparse.csc_matrix(rows[:, free].T)],
                                [sparse.csc_matrix(rows[:, free]), None]], format="csc")
        x[free] = EquilibratedLU(bordered, rtol).solve(np.r_[rrhs, targets])[: len(free)]
    else:
        x[free] = EquilibratedLU(sparse.csc_matrix(reduced), rtol).solve(rrhs)
    defect = reduced @ x[free] - rrhs
    scale = abs(reduced) @ np.abs(x[free])
    phys = max(np.linalg.norm(rhs[free]), np.linalg.norm(load_scale[free]), np.linalg.norm(action),
               np.linalg.norm(rrhs), np.linalg.norm(scale), np.finfo(float).tiny)
    residual = float(np.linalg.norm(defect) / phys)
    if residual > 1e-8:
        raise ValueError("incompatible data: gauge changed physical equations")
    return x, residual


def cell_flux(fine, u, permeability):
    """Flux ``-K grad u`` at fine-cell centres (``postprocessing/solutions.py:278-324``)."""
    dofs, _ = q1_space(fine)
    h = fine.spacing
    coef = u[dofs]
    gx = (-coef[:, 0] + coef[:, 1] - coef[:, 2] + coef[:, 3]) * 0.5 / h[0]
    gy = (-coef[:, 0] - coef[:, 1] + coef[:, 2] + coef[:, 3]) * 0.5 / h[1]
    centres = fine.points[fine.cells[:, 0]] + 0.5 * h
    k = tensor_at(permeability, centres)
    grad = np.column_stack((gx, gy))
    return -np.einsum("qab,qb->qa", k, grad)


# --------------------------------------------------------------------------------------
# Driver: _legacy/models/darcy/cartesian.py:69-168
# --------------------------------------------------------------------------------------
@dataclass
class Q1Solution:
    trace: np.ndarray
    coarse: np.ndarray
    fields: np.ndarray
    flux: np.ndarray
    residual: float
    matrix: sparse.csc_matrix
    rhs: np.ndarray
    corrected: np.ndarray
    responses: list


def local_problem(mesh, skeleton, cell, refinement, permeability, source, order=4):
    """``_assemble_quad`` (``cartesian.py:69-83``)."""
    fine = mesh.submesh(cell, refinement)
    matrix, mass, load = q1_operators(fine, permeability, source, order)
    coupling = trace_coupling(mesh, cell, fine, skeleton)
    constraints = mass @ np.ones((matrix.shape[0], 1))
    return fine, LocalProblem(matrix, coupling, load, skeleton.cell_dofs(cell), constraints)


def solve_darcy_q1(mesh, skeleton, refinement, permeability=1.0, source=0.0, dirichlet=0.0,
                   order=4, keep_responses=False, cells=None, neumann=None, mean_pressure=0.0):
    """``solve_darcy_quadrilateral`` for degree one (``cartesian.py:86-168``); Neumann
    faces fix their trace DOFs, and with every boundary face Neumann the mean of the
    pressure is ``mean_pressure`` (``:136-142``)."""
    boundary, fixed = boundary_data(skeleton, dirichlet, neumann, order)
    responses, contribs, fines = [], [], []
    for cell in range(len(mesh.cells)):
        fine, problem = local_problem(mesh, skeleton, cell, refinement, permeability, source, order)
        resp = condense(problem)
        contribs.append(contribution(resp, skeleton.size + cell))
        responses.append(resp)
        fines.append(fine)
    matrix, rhs, scale = assemble_global(contribs, skeleton.size, boundary)
    constraints = None
    if neumann and set(neumann) == set(int(f) for f in mesh.boundary_faces):
        x0, x1, y0, y1 = mesh.bounds
        weights = [r.problem.constraints[:, 0] for r in responses]
        constraints = [mean_constraint(responses, skeleton.size, weights, mean_pressure * (x1 - x0) * (y1 - y0))]
    x, residual = solve_global(matrix, rhs, scale, fixed=fixed, constraints=constraints)
    trace = x[: skeleton.size]
    coarse = x[skeleton.size:]
    fields = np.array([r.source - r.lifts @ trace[r.problem.trace_dofs] + r.retained @ coarse[c: c + 1]
                       for c, r in enumerate(responses)])
    flux = np.array([cell_flux(fines[c], fields[c], permeability) for c in range(len(responses))])
    corrected = np.array([r.coarse_vectors is not None for r in responses])
    return Q1Solution(trace, coarse, fields, flux, residual, matrix, rhs, corrected,
                      responses if keep_responses else [])


# --------------------------------------------------------------------------------------
# Original-equation refinement: core/refinement.py:612-800 (no fixed DOFs, no moments)
# --------------------------------------------------------------------------------------
def refine_q1(mesh, skeleton, refinement, trace, coarse, fields, permeability=1.0, source=0.0, dirichlet=0.0,
              max_steps=2, min_steps=0, rtol=1e-10, atol=0.0, order=4):
    """``refine_hybrid`` for the Cartesian Q1 system (``refinement.py:612-800``).

    Residual of the uncondensed equations (``:718-738``): local defects
    ``f - B lambda - A u`` (accurate residuals, ``:721-727``) and the weak trace rows
    ``boundary - sum B^T u`` (``:729-731``); acceptance at ``max(atol, rtol ||rhs||)``
    (``:687-690, :739-765``); each correction solves every cell with its defect as the
    source, assembles the correction system with the weak residual as boundary load
    and adds its solution (``:772-800``).
    """
    boundary, _ = boundary_data(skeleton, dirichlet, None, order)
    probs = [local_problem(mesh, skeleton, c, refinement, permeability, source, order)[1]
             for c in range(len(mesh.cells))]
    trace = np.array(trace, dtype=float)
    coarse = np.array(coarse, dtype=float)
    fields = [np.array(u, dtype=float) for u in fields]
    rhs_norm = float(np.linalg.norm(np.concatenate([p.load for p in probs] + [boundary])))
    threshold = max(atol, rtol * rhs_norm)
    history, step = [], 0
    while True:
        defects = []
        weak = boundary.copy()
        for p, u in zip(probs, fields):
            forcing = accurate_residual(sparse.csr_matrix(p.coupling), p.load, trace[p.trace_dofs])
            defects.append(accurate_residual(p.matrix.tocsr(), forcing, u))
            np.add.at(weak, p.trace_dofs, -p.coupling.T @ u)
        residual = float(np.linalg.norm(np.concatenate([*defects, weak])))
        history.append(residual)
        if step >= min_steps and np.isfinite(residual) and residual <= threshold:
            retained = [np.sum(np.asarray(d, dtype=float)) for d in defects]
            return dict(trace=trace, coarse=coarse, fields=np.array(fields), residual_norms=tuple(history),
                        rhs_norm=rhs_norm, reduced=float(np.linalg.norm(np.r_[weak, retained])))
        if step == max_steps or not np.isfinite(residual):
            raise LinearSolveError(f"original hybrid residual {residual:.6e} exceeds {threshold:.6e} "
                                   f"after {step} corrections")
        contribs, responses = [], []
        for c, (p, d) in enumerate(zip(probs, defects)):
            resp = condense(LocalProblem(p.matrix, p.coupling, np.asarray(d, dtype=float), p.trace_dofs,
                                         p.constraints))
            contribs.append(contribution(resp, skeleton.size + c))
            responses.append(resp)
        matrix, rhs, scale = assemble_global(contribs, skeleton.size, weak)
        x, _ = solve_global(matrix, rhs, scale)
        dtrace, dcoarse = x[: skeleton.size], x[skeleton.size:]
        trace += dtrace
        coarse += dcoarse
        fields = [u + r.source - r.lifts @ dtrace[r.problem.trace_dofs] + r.retained @ dcoarse[c: c + 1]
                  for c, (u, r) in enumerate(zip(fields, responses))]
        step += 1


# --------------------------------------------------------------------------------------
# The whole Cartesian solve with the local stage on a process pool (checker at full size
# and the timed CPU baseline)
# --------------------------------------------------------------------------------------
_POOL_STATE = {}


def _pool_init(macro, local, face_degree, kappa, source, blas_threads):
    """Worker set-up: one BLAS thread (the reference's process-backend policy,
    ``execution/cpu.py:97-101``) and the mesh, skeleton and coefficients."""
    from threadpoolctl import threadpool_limits

    _POOL_STATE["limits"] = threadpool_limits(blas_threads)
    mesh = cartesian_mesh(macro)
    sk = Skeleton(mesh, (FaceSpace.uniform(face_degree),) * len(mesh.faces))
    nf = macro * local
    perm = PixelField(kappa, (1.0 / nf, 1.0 / nf)) if kappa is not None else 1.0
    _POOL_STATE.update(mesh=mesh, sk=sk, local=local, perm=perm, source=source)


def _pool_cells(cells):
    """Assembly, condensation and contribution of the given macrocells (the per-cell
    loop of ``solve_darcy_q1``); returns what the parent assembles and reconstructs."""
    st = _POOL_STATE
    out = []
    for cell in cells:
        _, problem = local_problem(st["mesh"], st["sk"], int(cell), (st["local"], st["local"]), st["perm"],
                                   st["source"])
        resp = condense(problem)
        idx, block, load = contribution(resp, st["sk"].size + int(cell))
        out.append((idx, block, load, resp.source, resp.lifts, resp.retained[:, 0]))
    return out


def cartesian_flux(mesh, refinement, fields, permeability):
    """``cell_flux`` of every macrocell at once: the same gradient formula and
    fine-cell centres (``postprocessing/solutions.py:278-324``) over all cells."""
    r = refinement
    lower = mesh.points[mesh.cells[:, 0]]
    upper = mesh.points[mesh.cells[:, 2]]
    xs = np.linspace(lower[:, 0], upper[:, 0], r + 1)  # (r+1, cells), as each submesh's linspace
    ys = np.linspace(lower[:, 1], upper[:, 1], r + 1)
    hx = (upper[:, 0] - lower[:, 0]) / r
    hy = (upper[:, 1] - lower[:, 1]) / r
    ix, iy = np.tile(np.arange(r), r), np.repeat(np.arange(r), r)  # fine cells x-fastest
    origin = iy * (r + 1) + ix
    u = np.asarray(fields)
    c0, c1, c2, c3 = (u[:, origin + k] for k in (0, 1, r + 1, r + 2))
    gx = (-c0 + c1 - c2 + c3) * 0.5 / hx[:, None]
    gy = (-c0 - c1 + c2 + c3) * 0.5 / hy[:, None]
    cx = xs[ix].T + 0.5 * hx[:, None]
    cy = ys[iy].T + 0.5 * hy[:, None]
    k = tensor_at(permeability, np.column_stack((cx.ravel(), cy.ravel())))
    grad = np.column_stack((gx.ravel(), gy.ravel()))
    return -np.einsum("qab,qb->qa", k, grad).reshape(len(u), r * r, 2)


class CartesianSolve:
    """``solve_darcy_q1`` of a uniform Cartesian workload (``macro`` x ``macro`` cells,
    ``local`` x ``local`` Q1, uniform Legendre faces of ``face_degree``, pixel
    permeability ``kappa`` on the fine cells or 1, constant or callable ``source``,
    homogeneous Dirichlet data) with the per-cell local stage on ``workers`` spawn
    processes of one BLAS thread each.  Assembly, the global SuperLU solve and the
    reconstruction run in the calling process.  ``solve()`` times each phase.

    Start it before any CUDA context exists in the calling process, or keep the
    default spawn context: a pool forked from a CUDA process can hang.
    """

    def __init__(self, macro, local, face_degree, kappa=None, source=1.0, workers=None, chunks_per_worker=4):
        import multiprocessing as mp
        import os

        self.workers = int(workers or os.cpu_count() or 1)
        self.macro, self.local = macro, local
        self.mesh = cartesian_mesh(macro)
        self.sk = Skeleton(self.mesh, (FaceSpace.uniform(face_degree),) * len(self.mesh.faces))
        nf = macro * local
        self.perm = PixelField(kappa, (1.0 / nf, 1.0 / nf)) if kappa is not None else 1.0
        self.boundary, _ = boundary_data(self.sk, 0.0, None, 4)
        cells = len(self.mesh.cells)
        self.dofs = np.array([self.sk.cell_dofs(c) for c in range(cells)])
        self.chunks = [c for c in np.array_split(np.arange(cells), self.workers * chunks_per_worker) if len(c)]
        self.pool = mp.get_context("spawn").Pool(self.workers, initializer=_pool_init,
                                                 initargs=(macro, local, face_degree, kappa, source, 1))
        self.pool.map(_pool_cells, [[0]] * self.workers)  # imports and caches, untimed

    def close(self):
        self.pool.close()
        self.pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self):
        import time

        t0 = time.perf_counter()
        parts = self.pool.map(_pool_cells, self.chunks)
        t1 = time.perf_counter()
        res = [r for p in parts for r in p]
        matrix, rhs, scale = assemble_global([r[:3] for r in res], self.sk.size, self.boundary)
        t2 = time.perf_counter()
        x, residual = solve_global(matrix, rhs, scale)
        t3 = time.perf_counter()
        T = self.sk.size
        trace, coarse = x[:T], x[T:]
        fields = np.array([src - lifts @ trace[self.dofs[c]] + ret * coarse[c]
                           for c, (_, _, _, src, lifts, ret) in enumerate(res)])
        flux = cartesian_flux(self.mesh, self.local, fields, self.perm)
        t4 = time.perf_counter()
        phases = {"local_stage_s": t1 - t0, "assembly_s": t2 - t1, "global_solve_s": t3 - t2,
                  "reconstruction_s": t4 - t3, "total_s": t4 - t0}
        return dict(trace=trace, coarse=coarse, fields=fields, flux=flux, matrix=matrix, rhs=rhs,
                    residual=residual, phases=phases)


def serial_local_rate(macro, local, face_degree, kappa, source, cells):
    """Macrocells per second of the local stage in this process with one BLAS thread
    (the reference's ``backend="serial"`` policy), over the given cell ids."""
    import time

    from threadpoolctl import threadpool_limits

    mesh = cartesian_mesh(macro)
    sk = Skeleton(mesh, (FaceSpace.uniform(face_degree),) * len(mesh.faces))
    nf = macro * local
    perm = PixelField(kappa, (1.0 / nf, 1.0 / nf)) if kappa is not None else 1.0
    with threadpool_limits(1):
        local_problem(mesh, sk, int(cells[0]), (local, local), perm, source)  # warm caches
        t0 = time.perf_counter()
        for cell in cells:
            _, problem = local_problem(mesh, sk, int(cell), (local, local), perm, source)
            contribution(condense(problem), sk.size + int(cell))
        dt = time.perf_counter() - t0
    return len(cells) / dt, dt
