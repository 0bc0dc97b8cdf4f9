"""Host-side topology, trace spaces and index maps of the Cartesian MHM path.

Everything here is integer bookkeeping or once-per-mesh tabulation; it is
computed on the host once and uploaded.  The numbering is bit-exact with
PyMHM 1.3.2 (paths relative to its ``src/pymhm/``):

* ``CartesianMacroMesh``  ``meshes/cartesian.py:11-144``: points x-fastest,
  counterclockwise cells, faces numbered by first encounter in row-major cells
  (sides bottom, right, top, left), each face oriented along its first cell's
  counterclockwise traversal, sign +1 in that cell and -1 in the other.
* ``FaceSpace`` / ``SkeletonSpace``  ``fem/traces/interval.py:13-161``:
  discontinuous unnormalised Legendre modes per segment or continuous nodal
  bases, global offsets, cell DOFs in side order.
* ``coupling_tables``  ``fem/scalar/quadrilateral.py:256-298``: the integral of
  each fine boundary hat against each face basis, split at fine nodes and face
  breaks, with the reference's Gauss order ``max(face degree) + 2``.
* ``boundary_data``  ``fem/scalar/operators.py:247-321`` (weak Dirichlet moments).
* ``skeleton_pattern``  the CSR pattern that ``assemble_hybrid_contributions``
  (``core/contributions.py:77-195``) produces, with per-slot contributor lists
  in cell order so that the device reduction adds shared-face entries in the
  reference's order.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from functools import cached_property

import numpy as np
from numpy.polynomial.legendre import leggauss


# ----------------------------------------------------------------------------------------
# Macro mesh
# ----------------------------------------------------------------------------------------
@dataclass(frozen=True)
class CartesianMacroMesh:
    """Uniform rectangle mesh with the reference's numbering (see module docstring)."""

    nx: int = 1
    ny: int | None = None
    bounds: tuple[float, float, float, float] = (0.0, 1.0, 0.0, 1.0)
    points: np.ndarray = field(init=False, repr=False)
    cells: np.ndarray = field(init=False, repr=False)
    faces: np.ndarray = field(init=False, repr=False)
    cell_faces: np.ndarray = field(init=False, repr=False)
    signs: np.ndarray = field(init=False, repr=False)
    face_cells: np.ndarray = field(init=False, repr=False)

    def __post_init__(self) -> None:
        nx = int(self.nx)
        ny = nx if self.ny is None else int(self.ny)
        if nx < 1 or ny < 1:
            raise ValueError("nx and ny must be positive integers")
        x0, x1, y0, y1 = (float(v) for v in self.bounds)
        if not (x1 > x0 and y1 > y0) or not np.isfinite([x0, x1, y0, y1]).all():
            raise ValueError("bounds must have positive width and height")
        x, y = np.linspace(x0, x1, nx + 1), np.linspace(y0, y1, ny + 1)
        points = np.column_stack((np.tile(x, ny + 1), np.repeat(y, nx + 1)))
        j, i = np.divmod(np.arange(nx * ny), nx)
        a = j * (nx + 1) + i
        cells = np.column_stack((a, a + 1, a + nx + 2, a + nx + 1)).astype(np.int64)
        # first-encounter face ids: row 0 gives 4 + 3 (nx - 1) new faces, every later
        # row 3 + 2 (nx - 1); see the module docstring for the visiting order.
        row_start = np.where(j == 0, 0, 3 * nx + 1 + (j - 1) * (2 * nx + 1))
        bottom = np.where(j == 0, np.where(i == 0, 0, 3 * i + 1), -1)
        right = np.where(j == 0, np.where(i == 0, 1, 3 * i + 2),
                         row_start + np.where(i == 0, 0, 2 * i + 1))
        top = np.where(j == 0, np.where(i == 0, 2, 3 * i + 3),
                       row_start + np.where(i == 0, 1, 2 * i + 2))
        left = np.where(i == 0, np.where(j == 0, 3, row_start + 2), -1)
        cell_ids = np.arange(nx * ny)
        # faces seen before: bottom = top of the cell below, left = right of the cell to the left
        below = np.where(j > 0, cell_ids - nx, 0)
        leftc = np.where(i > 0, cell_ids - 1, 0)
        bottom = np.where(j > 0, top[below], bottom)
        left = np.where(i > 0, right[leftc], left)
        cell_faces = np.column_stack((bottom, right, top, left)).astype(np.int64)
        first = np.column_stack((j == 0, np.ones_like(i, bool), np.ones_like(i, bool), i == 0))
        ends = np.stack((cells, np.roll(cells, -1, axis=1)), axis=-1)  # (cells, side, 2)
        nfaces = (ny + 1) * nx + (nx + 1) * ny
        faces = np.empty((nfaces, 2), dtype=np.int64)
        face_cells = np.full((nfaces, 2), -1, dtype=np.int64)
        faces[cell_faces[first]] = ends[first]
        cidx = np.broadcast_to(cell_ids[:, None], (nx * ny, 4))
        face_cells[cell_faces[first], 0] = cidx[first]
        face_cells[cell_faces[~first], 1] = cidx[~first]
        signs = np.where(first, 1, -1).astype(np.int64)
        object.__setattr__(self, "nx", nx)
        object.__setattr__(self, "ny", ny)
        object.__setattr__(self, "bounds", (x0, x1, y0, y1))
        for name, value in (("points", points), ("cells", cells), ("faces", faces),
                            ("cell_faces", cell_faces), ("signs", signs),
                            ("face_cells", face_cells)):
            value.setflags(write=False)
            object.__setattr__(self, name, value)

    @property
    def spacing(self) -> np.ndarray:
        x0, x1, y0, y1 = self.bounds
        return np.array([(x1 - x0) / self.nx, (y1 - y0) / self.ny])

    @property
    def lengths(self) -> np.ndarray:
        return np.linalg.norm(self.points[self.faces[:, 1]] - self.points[self.faces[:, 0]], axis=1)

    @property
    def areas(self) -> np.ndarray:
        return np.full(len(self.cells), float(np.prod(self.spacing)))

    @property
    def boundary_faces(self) -> np.ndarray:
        return np.flatnonzero(self.face_cells[:, 1] == -1)


def mesh_arrays(mesh) -> CartesianMacroMesh:
    """Accept this package's mesh or any object with the reference's mesh attributes."""
    if isinstance(mesh, CartesianMacroMesh):
        return mesh
    for name in ("nx", "ny", "bounds", "faces", "cell_faces", "signs"):
        if not hasattr(mesh, name):
            raise TypeError("a CartesianMacroMesh (or an object with its attributes) is required")
    own = CartesianMacroMesh(mesh.nx, mesh.ny, tuple(mesh.bounds))
    if not (np.array_equal(own.cell_faces, mesh.cell_faces) and np.array_equal(own.signs, mesh.signs)
            and np.array_equal(own.faces, mesh.faces)):
        raise ValueError("mesh numbering differs from the Cartesian macro-mesh convention")
    return own


# ----------------------------------------------------------------------------------------
# Face and skeleton spaces
# ----------------------------------------------------------------------------------------
def legendre(x: np.ndarray, degree: int) -> np.ndarray:
    """Conventional Legendre L_0..L_degree (L_j(1) = 1), three-term recurrence."""
    x = np.asarray(x, dtype=float)
    out = np.empty((*x.shape, degree + 1))
    out[..., 0] = 1.0
    if degree >= 1:
        out[..., 1] = x
    for j in range(1, degree):
        out[..., j + 1] = ((2 * j + 1) * x * out[..., j] - j * out[..., j - 1]) / (j + 1)
    return out


def lagrange(x: np.ndarray, nodes: np.ndarray) -> np.ndarray:
    """Nodal interval basis on ``nodes`` with exact Kronecker rows at literal nodes."""
    x = np.asarray(x, dtype=float)
    c = np.asarray(nodes, dtype=float)
    vals = np.ones((len(x), len(c)))
    for i in range(len(c)):
        for m in range(len(c)):
            if m != i:
                vals[:, i] *= (x - c[m]) / (c[i] - c[m])
    rows, cols = np.nonzero(x[:, None] == c[None, :])
    vals[rows] = 0.0
    vals[rows, cols] = 1.0
    return vals


@dataclass(frozen=True)
class FaceSpace:
    """Trace space on one macro face (``fem/traces/interval.py:13-116``)."""

    breaks: tuple[float, ...] = (0.0, 1.0)
    degrees: tuple[int, ...] = (0,)
    continuous: bool = False

    def __post_init__(self) -> None:
        breaks = tuple(float(v) for v in self.breaks)
        degrees = tuple(int(p) for p in self.degrees)
        if len(breaks) != len(degrees) + 1 or not degrees:
            raise ValueError("one degree is required per face segment")
        if breaks[0] != 0 or breaks[-1] != 1 or not np.all(np.diff(breaks) > 0):
            raise ValueError("face breaks must increase strictly from 0 to 1")
        if min(degrees) < 0 or (self.continuous and min(degrees) < 1):
            raise ValueError("invalid face degrees")
        object.__setattr__(self, "breaks", breaks)
        object.__setattr__(self, "degrees", degrees)

    @classmethod
    def uniform(cls, degree: int = 0, subdivisions: int = 1, *, continuous: bool = False) -> "FaceSpace":
        return cls(tuple(np.linspace(0, 1, subdivisions + 1)), (degree,) * subdivisions, continuous)

    @classmethod
    def of(cls, space) -> "FaceSpace":
        if isinstance(space, FaceSpace):
            return space
        return cls(tuple(space.breaks), tuple(space.degrees), bool(space.continuous))

    @property
    def size(self) -> int:
        return 1 + sum(self.degrees) if self.continuous else sum(p + 1 for p in self.degrees)

    def evaluate(self, parameter) -> np.ndarray:
        """Basis values at oriented face coordinates (``interval.py:54-89``)."""
        t = np.atleast_1d(np.asarray(parameter, dtype=float))
        values = np.zeros((len(t), self.size))
        offset = 0
        for i, degree in enumerate(self.degrees):
            lo, hi = self.breaks[i: i + 2]
            mask = (t >= lo) & ((t < hi) | ((i == len(self.degrees) - 1) & (t <= hi)))
            local = (t[mask] - lo) / (hi - lo)
            if self.continuous:
                nodes = np.r_[0.0, 1.0, np.arange(1, degree) / degree]
                ids = np.r_[i, i + 1, len(self.breaks) + offset + np.arange(degree - 1)]
                values[np.ix_(mask, ids)] = lagrange(local, nodes)
                offset += degree - 1
            else:
                values[mask, offset: offset + degree + 1] = legendre(2 * local - 1, degree)
                offset += degree + 1
        return values

    def quadrature(self, order: int = 4) -> tuple[np.ndarray, np.ndarray]:
        """Per-segment Gauss rule (``interval.py:99-116``)."""
        x, w = leggauss(order)
        w = np.asarray(w, dtype=np.longdouble)
        w *= np.longdouble(2) / np.sum(w)
        points, weights = [], []
        for lo, hi in zip(self.breaks[:-1], self.breaks[1:]):
            points.extend(lo + (x + 1) * (hi - lo) / 2)
            weights.extend(w * (hi - lo) / 2)
        return np.asarray(points), np.asarray(weights, dtype=float)

    def moments(self) -> np.ndarray:
        """Exact integrals of each basis function over [0, 1]."""
        order = max(self.degrees) + 2
        t, w = self.quadrature(order)
        return w @ self.evaluate(t)


class SkeletonSpace:
    """Scalar skeleton over a Cartesian mesh (``interval.py:119-161``)."""

    def __init__(self, mesh, faces=None):
        self.mesh = mesh_arrays(mesh)
        nf = len(self.mesh.faces)
        faces = tuple(FaceSpace() for _ in range(nf)) if faces is None else tuple(FaceSpace.of(f) for f in faces)
        if len(faces) != nf:
            raise ValueError("provide exactly one FaceSpace per mesh face")
        self.faces = faces
        self.offsets = np.r_[0, np.cumsum([f.size for f in faces])].astype(np.int64)
        self.offsets.setflags(write=False)

    @classmethod
    def of(cls, skeleton, mesh=None) -> "SkeletonSpace":
        if isinstance(skeleton, SkeletonSpace):
            return skeleton
        if getattr(skeleton, "components", 1) != 1:
            raise ValueError("a scalar skeleton is required")
        return cls(skeleton.mesh if mesh is None else mesh, skeleton.faces)

    @property
    def size(self) -> int:
        return int(self.offsets[-1])

    def dofs(self, face: int) -> np.ndarray:
        return np.arange(self.offsets[face], self.offsets[face + 1])

    @cached_property
    def cell_dof_array(self) -> np.ndarray:
        """(cells, t) trace DOFs in side order; requires equal cell widths."""
        m = self.mesh
        sizes = np.diff(self.offsets)
        widths = sizes[m.cell_faces].sum(axis=1)
        if not np.all(widths == widths[0]):
            raise ValueError("cells must have equal trace widths")
        out = np.concatenate([self.offsets[m.cell_faces[:, s], None] + np.arange(sizes[m.cell_faces[0, s]])
                              for s in range(4)], axis=1)
        return out.astype(np.int64)

    def cell_dofs(self, cell: int) -> np.ndarray:
        return np.concatenate([self.dofs(int(f)) for f in self.mesh.cell_faces[cell]])

    def uniform_by_orientation(self) -> tuple[FaceSpace, FaceSpace]:
        """The shared horizontal and vertical face spaces (GPU path requirement)."""
        m = self.mesh
        hfaces = m.cell_faces[:, [0, 2]].ravel()
        vfaces = m.cell_faces[:, [1, 3]].ravel()
        h = {self.faces[f] for f in np.unique(hfaces)}
        v = {self.faces[f] for f in np.unique(vfaces)}
        if len(h) != 1 or len(v) != 1:
            raise NotImplementedError("the GPU path requires one FaceSpace per face orientation")
        return h.pop(), v.pop()


# ----------------------------------------------------------------------------------------
# Tables and boundary data
# ----------------------------------------------------------------------------------------
def coupling_tables(space_h: FaceSpace, space_v: FaceSpace, rx: int, ry: int, hx_macro: float,
                    hy_macro: float) -> np.ndarray:
    """``[kind][orient][k][j]`` integrals of fine boundary hats against face bases.

    kind 0: horizontal side with rx+1 nodes and face length hx_macro; kind 1:
    vertical side, ry+1 nodes, length hy_macro.  orient 0: the face coordinate
    grows with the side coordinate; orient 1: it decreases.  Follows the
    segment/breakpoint quadrature of ``quadrilateral.py:279-297``.
    """
    kmax = max(rx, ry) + 1
    jmax = max(space_h.size, space_v.size)
    table = np.zeros((2, 2, kmax, jmax))
    for kind, (space, r, length) in enumerate(((space_h, rx, hx_macro), (space_v, ry, hy_macro))):
        gauss, w = leggauss(max(space.degrees) + 1 + 1)
        for orient in range(2):
            tn = np.arange(r + 1) / r
            if orient:
                tn = 1.0 - tn
            for k in range(r):
                t0, t1 = tn[k], tn[k + 1]
                lo, hi = sorted((float(t0), float(t1)))
                cuts = sorted({lo, hi, *(b for b in space.breaks if lo < b < hi)})
                for left, right in zip(cuts[:-1], cuts[1:]):
                    parameter = left + (gauss + 1) * (right - left) / 2
                    s = (parameter - t0) / (t1 - t0)
                    local = np.column_stack((1 - s, s))
                    weights = w * (right - left) / 2 * length
                    table[kind, orient, k: k + 2, : space.size] += local.T @ (
                        weights[:, None] * space.evaluate(parameter))
    return table


def side_orientation(mesh: CartesianMacroMesh) -> np.ndarray:
    """(cells, 4) 1 where the face coordinate decreases along the side's coordinate."""
    p = mesh.points
    f = mesh.faces[mesh.cell_faces]  # (cells, 4, 2)
    dx = p[f[..., 1], 0] - p[f[..., 0], 0]
    dy = p[f[..., 1], 1] - p[f[..., 0], 1]
    horizontal = np.array([True, False, True, False])
    return np.where(horizontal[None, :], dx < 0, dy < 0).astype(np.int8)


def _neumaier_moments(basis: np.ndarray, weights: np.ndarray, values: np.ndarray) -> np.ndarray:
    """``boundary_moments`` (``fem/scalar/_integration.py:91-108``)."""
    out = np.empty(basis.shape[1])
    for i in range(basis.shape[1]):
        total = 0.0
        corr = 0.0
        for q in range(len(weights)):
            v = basis[q, i] * weights[q] * values[q]
            s = total + v
            corr += (total - s) + v if abs(total) >= abs(v) else (v - s) + total
            total = s
        out[i] = total + corr
    return out


def _neumann_faces(skeleton: SkeletonSpace, neumann) -> dict:
    neumann = {} if neumann is None else neumann
    if not isinstance(neumann, dict):
        raise ValueError("Neumann data must map boundary faces to prescribed fields")
    boundary = set(int(f) for f in skeleton.mesh.boundary_faces)
    faces = {}
    for face, data in neumann.items():
        if isinstance(face, bool) or not isinstance(face, (int, np.integer)) or int(face) not in boundary:
            raise ValueError("Neumann data may only be imposed on boundary faces")
        faces[int(face)] = data
    return faces


def boundary_data(skeleton: SkeletonSpace, dirichlet=0.0, order: int = 4, neumann=None) -> np.ndarray:
    """Weak Dirichlet trace load on the faces without Neumann data
    (``fem/scalar/operators.py:247-321``)."""
    load = np.zeros(skeleton.size)
    neumann = _neumann_faces(skeleton, neumann)
    if not callable(dirichlet) and float(dirichlet) == 0.0:
        return load
    mesh = skeleton.mesh
    lengths = mesh.lengths
    for face in mesh.boundary_faces:
        if int(face) in neumann:
            continue
        space = skeleton.faces[face]
        t, w = space.quadrature(max(order, max(space.degrees) + 2))
        start, end = mesh.points[mesh.faces[face]]
        pts = start + t[:, None] * (end - start)
        vals = dirichlet(pts) if callable(dirichlet) else dirichlet
        vals = np.broadcast_to(np.asarray(vals, dtype=float), (len(pts),))
        load[skeleton.dofs(int(face))] = _neumaier_moments(space.evaluate(t), w, vals) * lengths[face]
    return load


def neumann_fixed(skeleton: SkeletonSpace, neumann, order: int = 4) -> tuple[np.ndarray, np.ndarray]:
    """Prescribed trace coefficients of the Neumann faces (``boundary_data``'s ``fixed``,
    ``fem/scalar/operators.py:286-316``): the L2 projection of the outward normal flux
    onto each face's trace basis, with the compensated boundary moments."""
    neumann = _neumann_faces(skeleton, neumann)
    dofs, values = [], []
    mesh = skeleton.mesh
    for face in mesh.boundary_faces:
        if int(face) not in neumann:
            continue
        space = skeleton.faces[face]
        t, w = space.quadrature(max(order, max(space.degrees) + 2))
        start, end = mesh.points[mesh.faces[face]]
        pts = start + t[:, None] * (end - start)
        data = neumann[int(face)]
        vals = np.broadcast_to(np.asarray(data(pts) if callable(data) else data, dtype=float), (len(pts),))
        if not np.all(np.isfinite(vals)):
            raise ValueError("scalar coefficient must be finite")
        basis = space.evaluate(t)
        moments = _neumaier_moments(basis, w, vals)
        coef = np.linalg.solve(basis.T @ (w[:, None] * basis), moments)
        dofs.append(skeleton.dofs(int(face)))
        values.append(coef)
    if not dofs:
        return np.zeros(0, dtype=np.int64), np.zeros(0)
    return np.concatenate(dofs).astype(np.int64), np.concatenate(values)


def neumann_layout(mesh, neumann) -> tuple[int, list]:
    """(bits, partial): the whole sides the Neumann faces cover (bit 0 the bottom
    y = y0, bit 1 the top, bit 2 the left x = x0, bit 3 the right) and the Neumann
    faces left over, on sides they cover only in part."""
    faces = set(int(f) for f in (neumann or {}))
    if not faces:
        return 0, []
    x0, x1, y0, y1 = mesh.bounds
    pts = mesh.points[mesh.faces[mesh.boundary_faces]]
    xs, ys = pts[:, :, 0], pts[:, :, 1]
    sides = [set(int(f) for f in mesh.boundary_faces[np.all(c == v, axis=1)])
             for c, v in ((ys, y0), (ys, y1), (xs, x0), (xs, x1))]
    bits, covered = 0, set()
    for bit, side in enumerate(sides):
        if side <= faces:
            bits |= 1 << bit
            covered |= side
    return bits, sorted(faces - covered)


def coarse_partial_correction(mesh, bits: int, partial, ax: float, ay: float) -> tuple[np.ndarray, np.ndarray]:
    """Woodbury factor of the coarse operator with Neumann faces on part of a side.

    A_sep = ay (T_y (x) I) + ax (I (x) T_x) takes the whole Neumann sides in ``bits``
    as Neumann ends and every other side as Dirichlet; each face in ``partial`` takes
    its a_y (horizontal face) or a_x (vertical face) off its cell's diagonal:
    A = A_sep - E D E^T.  Returns the m affected cells and R = A_sep^-1 E
    (D^-1 - E^T A_sep^-1 E)^-1 (cells x m), so that A^-1 r = y + R (E^T y) with
    y = A_sep^-1 r."""
    from scipy import sparse
    from scipy.sparse import linalg as splinalg

    nx, ny = mesh.nx, mesh.ny

    def factor(n, lo, hi):
        t = sparse.diags([-np.ones(n - 1), 2.0 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], format="lil")
        if lo:
            t[0, 0] -= 1.0
        if hi:
            t[n - 1, n - 1] -= 1.0
        return t.tocsr()

    tx = factor(nx, bits & 4, bits & 8)
    ty = factor(ny, bits & 1, bits & 2)
    a_sep = (ay * sparse.kron(ty, sparse.identity(nx)) + ax * sparse.kron(sparse.identity(ny), tx)).tocsc()
    weight = {}
    for f in partial:
        c = int(mesh.face_cells[f, 0])
        p = mesh.points[mesh.faces[f]]
        horizontal = p[0, 1] == p[1, 1]
        weight[c] = weight.get(c, 0.0) + (ay if horizontal else ax)
    cells = np.array(sorted(weight), dtype=np.int32)
    d = np.array([weight[c] for c in cells])
    e = np.zeros((nx * ny, len(cells)))
    e[cells, np.arange(len(cells))] = 1.0
    z = splinalg.splu(a_sep).solve(e)
    cap = np.diag(1.0 / d) - z[cells]
    return cells, np.ascontiguousarray(np.linalg.solve(cap.T, z.T).T)


def coarse_x_basis(nx: int, bits: int) -> tuple[np.ndarray, np.ndarray]:
    """Eigenvectors [cell][mode] and eigenvalues of the coarse operator's x factor
    tridiag(-1, 2, -1) of order nx whose end rows lose a neighbour on a Neumann left
    (bit 2) or right (bit 3) side."""
    t = 2.0 * np.eye(nx) - np.eye(nx, k=1) - np.eye(nx, k=-1)
    if bits & 4:
        t[0, 0] -= 1.0
    if bits & 8:
        t[-1, -1] -= 1.0
    lam, vec = np.linalg.eigh(t)
    lam = np.maximum(lam, 0.0)
    if bits & 12 == 12:  # both ends Neumann: the constant mode, exactly
        lam[0] = 0.0
        vec[:, 0] = 1.0 / np.sqrt(nx)
    return np.ascontiguousarray(vec), lam


def coarse_mode0_pinv(ny: int, ay: float) -> np.ndarray:
    """Pseudo-inverse of ay tridiag(-1, 2, -1) of order ny with both end rows Neumann
    (the coarse operator's constant x mode when every side is fixed): the constant
    vector spans its kernel."""
    t = 2.0 * np.eye(ny) - np.eye(ny, k=1) - np.eye(ny, k=-1)
    t[0, 0] -= 1.0
    t[-1, -1] -= 1.0
    lam, vec = np.linalg.eigh(t)
    keep = np.arange(ny) > 0  # the smallest eigenvalue is the constant mode's zero
    return np.ascontiguousarray((vec[:, keep] / lam[keep]) @ vec[:, keep].T / ay)


def fixed_coarse_data(mesh, skeleton: SkeletonSpace, fixed_faces, ax: float, ay: float) -> dict:
    """Host data of a skeleton solve whose trace DOFs on ``fixed_faces`` (boundary
    faces) are prescribed: the DOF mask, the whole fixed sides (``neumann_layout``
    bits), the x eigenbasis when the left or right side is fixed, the mode-0
    pseudo-inverse when every side is, and the Woodbury factor of faces on parts of
    sides (None where not needed)."""
    faces = sorted(set(int(f) for f in fixed_faces))
    bits, partial = neumann_layout(mesh, {f: 0.0 for f in faces})
    mask = np.zeros(skeleton.size, dtype=np.uint8)
    for f in faces:
        mask[skeleton.dofs(f)] = 1
    out = dict(mask=mask, bits=bits, qx=None, lamx=None, pinv0=None, wb_cells=None, wb_R=None)
    if bits & 12:
        out["qx"], out["lamx"] = coarse_x_basis(mesh.nx, bits)
    if bits == 15 and not partial:
        out["pinv0"] = coarse_mode0_pinv(mesh.ny, ay)
    if partial:
        out["wb_cells"], out["wb_R"] = coarse_partial_correction(mesh, bits, partial, ax, ay)
    return out


# ----------------------------------------------------------------------------------------
# Global pattern and solver maps
# ----------------------------------------------------------------------------------------
@dataclass
class SkeletonPattern:
    size: int
    trace_size: int
    indptr: np.ndarray
    indices: np.ndarray
    slot_ptr: np.ndarray
    contrib: np.ndarray
    load_ptr: np.ndarray
    load_contrib: np.ndarray
    trace_end: np.ndarray


def skeleton_pattern(cell_dofs: np.ndarray, trace_size: int) -> SkeletonPattern:
    """Structural CSR of the reduced system with cell-ordered contributor lists.

    Cell K contributes the dense block over ``I_K = [cell_dofs[K], T + K]``; the
    flat contributor index of entry (a, b) is ``K (t+1)^2 + a (t+1) + b``.
    Slots are row-major with sorted columns (SciPy CSC of a symmetric pattern
    has the same index arrays).
    """
    cells, t = cell_dofs.shape
    t1 = t + 1
    idx = np.concatenate((cell_dofs, trace_size + np.arange(cells)[:, None]), axis=1)
    rows = np.repeat(idx, t1, axis=1).ravel()
    cols = np.tile(idx, (1, t1)).ravel()
    flat = np.arange(cells * t1 * t1, dtype=np.int64)
    order = np.lexsort((flat, cols, rows))  # by row, col, then cell order
    r, c, f = rows[order], cols[order], flat[order]
    new = np.ones(len(r), dtype=bool)
    new[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    slot_start = np.flatnonzero(new)
    size = trace_size + cells
    slot_rows = r[slot_start]
    indices = c[slot_start].astype(np.int32)
    indptr = np.zeros(size + 1, dtype=np.int64)
    np.add.at(indptr, slot_rows + 1, 1)
    indptr = np.cumsum(indptr)
    slot_ptr = np.r_[slot_start, len(r)].astype(np.int64)
    # load contributors
    lrows = idx.ravel()
    lflat = np.arange(cells * t1, dtype=np.int64)
    lorder = np.lexsort((lflat, lrows))
    load_ptr = np.zeros(size + 1, dtype=np.int64)
    np.add.at(load_ptr, lrows + 1, 1)
    load_ptr = np.cumsum(load_ptr)
    trace_end = np.empty(trace_size, dtype=np.int64)
    for_row = indices < trace_size
    counts = np.add.reduceat(for_row.astype(np.int64), indptr[:-1]) if len(indices) else np.zeros(size, np.int64)
    trace_end[:] = indptr[:trace_size] + counts[:trace_size]
    return SkeletonPattern(size, trace_size, indptr, indices, slot_ptr, f.astype(np.int64), load_ptr,
                           lflat[lorder], trace_end)


def block_offsets(cell_dofs) -> tuple[np.ndarray, np.ndarray]:
    """Flat offsets of every cell's (t_K + 1)^2 block and (t_K + 1) load when the
    cells' contributions are stored one after another (cells may differ in size)."""
    t1 = np.array([len(d) + 1 for d in cell_dofs], dtype=np.int64)
    bofs = np.zeros(len(t1) + 1, dtype=np.int64)
    bofs[1:] = np.cumsum(t1 * t1)
    lofs = np.zeros(len(t1) + 1, dtype=np.int64)
    lofs[1:] = np.cumsum(t1)
    return bofs, lofs


def skeleton_pattern_ragged(cell_dofs, trace_size: int) -> SkeletonPattern:
    """``skeleton_pattern`` for cells with different numbers of trace DOFs (polygons):
    cell K's block over ``[cell_dofs[K], T + K]`` is stored at ``block_offsets`` and
    its entry (a, b) is ``offset_K + a (t_K + 1) + b``."""
    bofs, lofs = block_offsets(cell_dofs)
    cells = len(cell_dofs)
    idx = [np.r_[np.asarray(d, dtype=np.int64), trace_size + k] for k, d in enumerate(cell_dofs)]
    rows = np.concatenate([np.repeat(i, len(i)) for i in idx]) if cells else np.zeros(0, np.int64)
    cols = np.concatenate([np.tile(i, len(i)) for i in idx]) if cells else np.zeros(0, np.int64)
    flat = np.arange(bofs[-1], dtype=np.int64)
    order = np.lexsort((flat, cols, rows))
    r, c, f = rows[order], cols[order], flat[order]
    new = np.ones(len(r), dtype=bool)
    new[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    slot_start = np.flatnonzero(new)
    size = trace_size + cells
    indices = c[slot_start].astype(np.int32)
    indptr = np.zeros(size + 1, dtype=np.int64)
    np.add.at(indptr, r[slot_start] + 1, 1)
    indptr = np.cumsum(indptr)
    slot_ptr = np.r_[slot_start, len(r)].astype(np.int64)
    lrows = np.concatenate(idx) if cells else np.zeros(0, np.int64)
    lflat = np.arange(lofs[-1], dtype=np.int64)
    lorder = np.lexsort((lflat, lrows))
    load_ptr = np.zeros(size + 1, dtype=np.int64)
    np.add.at(load_ptr, lrows + 1, 1)
    load_ptr = np.cumsum(load_ptr)
    for_row = indices < trace_size
    counts = np.add.reduceat(for_row.astype(np.int64), indptr[:-1]) if len(indices) else np.zeros(size, np.int64)
    trace_end = indptr[:trace_size] + counts[:trace_size]
    return SkeletonPattern(size, trace_size, indptr, indices, slot_ptr, f, load_ptr, lflat[lorder], trace_end)


def transpose_slots(indptr: np.ndarray, indices: np.ndarray) -> np.ndarray:
    """For a CSR pattern that is symmetric, ``out[k]`` = the slot of (i, j) for the slot
    k of (j, i).  Sorting the slots by (column, row) lists them in the CSR order of the
    transpose, which is the same pattern."""
    rows = np.repeat(np.arange(len(indptr) - 1, dtype=np.int64), np.diff(indptr))
    order = np.lexsort((rows, indices.astype(np.int64)))
    if not (np.array_equal(indices[order], rows) and np.array_equal(rows[order], indices)):
        raise ValueError("the pattern is not symmetric")
    return order.astype(np.int64)


def dof_cell_maps(cell_dofs: np.ndarray, trace_size: int) -> tuple[np.ndarray, np.ndarray]:
    """(T, 2) cells containing each trace DOF (cell order, -1 padded) and the DOF's slot."""
    cells, t = cell_dofs.shape
    dof_cells = np.full((trace_size, 2), -1, dtype=np.int32)
    dof_slot = np.zeros((trace_size, 2), dtype=np.int32)
    flat = cell_dofs.ravel()
    cell_of = np.repeat(np.arange(cells), t)
    slot_of = np.tile(np.arange(t), cells)
    order = np.lexsort((cell_of, flat))
    flat, cell_of, slot_of = flat[order], cell_of[order], slot_of[order]
    first = np.ones(len(flat), dtype=bool)
    first[1:] = flat[1:] != flat[:-1]
    if np.any(np.bincount(flat, minlength=trace_size) > 2):
        raise ValueError("a trace DOF is shared by more than two cells")
    k = np.where(first, 0, 1)
    dof_cells[flat, k] = cell_of
    dof_slot[flat, k] = slot_of
    return dof_cells, dof_slot


def geometric_constraint(mesh: CartesianMacroMesh, space_h: FaceSpace, space_v: FaceSpace) -> np.ndarray:
    """(cells, t) exact net-flux columns G0 = B^T 1 = sign * length * int psi_j."""
    mh, mv = space_h.moments(), space_v.moments()
    hx, hy = mesh.spacing
    sides = []
    for s in range(4):
        m, length = (mh, hx) if s % 2 == 0 else (mv, hy)
        sides.append(mesh.signs[:, s, None] * (length * m)[None, :])
    return np.concatenate(sides, axis=1)


def sine_transform(n: int) -> np.ndarray:
    k = np.arange(1, n + 1)
    return np.sqrt(2.0 / (n + 1)) * np.sin(np.pi * np.outer(k, k) / (n + 1))


def coarse_coefficients(mesh: CartesianMacroMesh, space_h: FaceSpace, space_v: FaceSpace) -> tuple[float, float]:
    """(ax, ay) with G0^T G0 = ay (T_y (x) I) + ax (I (x) T_x), T = tridiag(-1, 2, -1).

    A vertical face couples x-neighbours with weight hy^2 |int psi|^2 summed over its
    basis, a horizontal face couples y-neighbours with hx^2 |int psi|^2.
    """
    mh2 = float(np.sum(space_h.moments() ** 2))
    mv2 = float(np.sum(space_v.moments() ** 2))
    hx, hy = mesh.spacing
    return hy * hy * mv2, hx * hx * mh2


def coarse_eigenvalues(mesh: CartesianMacroMesh, space_h: FaceSpace, space_v: FaceSpace) -> np.ndarray:
    """Eigenvalues (ny, nx) of G0^T G0 in the sine basis."""
    ax, ay = coarse_coefficients(mesh, space_h, space_v)
    lx = 2 - 2 * np.cos(np.pi * np.arange(1, mesh.nx + 1) / (mesh.nx + 1))
    ly = 2 - 2 * np.cos(np.pi * np.arange(1, mesh.ny + 1) / (mesh.ny + 1))
    return ay * ly[:, None] + ax * lx[None, :]
