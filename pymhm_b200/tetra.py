"""Tetrahedral macro meshes and triangular skeletons for the 3D Primal-MHM path.

Host-side topology, built once per mesh: it fixes the global numbering of the trace
unknowns, so it follows the reference's construction exactly (PyMHM 1.3.2,
``src/pymhm/``):

* ``TetraMesh``: ``meshes/tetrahedron.py:23-96``.  Cells are reoriented to a positive
  determinant (vertices 1 and 2 swapped); side i of a cell is the face opposite its
  vertex i; faces are the sorted vertex triples numbered by first encounter over
  (cell, side) in order; a face's normal points out of its first cell, which carries
  sign +1 and the second cell -1.
* ``TetraMesh.unit_cube``: ``:98-112`` (six Freudenthal tetrahedra per cube, one per
  permutation of the axes, cubes in C order).
* ``reference_refinement`` / ``TetraMesh.submesh``: ``:114-158`` (red refinement with
  the fixed octahedron diagonal; the new vertices are edge midpoints numbered by
  first use).
* ``TriangularSkeleton``: ``fem/traces/triangle_3d.py:53-200`` for the uniform,
  unsubdivided, discontinuous case: Bernstein modes of degree 0 or 1 per macroface
  (degree 1: the face's barycentric coordinates in its sorted vertex order), the
  four faces' blocks in side order per cell.

The trace coupling of a local P1 space is tabulated here in closed form: on a fine
boundary triangle, two linear functions integrate exactly as
area / 12 (sum_k f_k g_k + sum_k f_k sum_k g_k), which the reference evaluates with
a 3-point-per-direction Duffy rule (``triangle_3d.py:221-273``); both are exact, so
the tables agree to rounding.
"""

from __future__ import annotations

from itertools import combinations, permutations

import numpy as np

EPS = np.finfo(float).eps


class TetraMesh:
    """Oriented tetrahedra with signed triangular face incidence (see the module docstring)."""

    def __init__(self, points, cells):
        pts = np.array(points, dtype=float)
        raw = np.asarray(cells)
        if pts.ndim != 2 or pts.shape[1] != 3 or len(pts) < 4 or not np.isfinite(pts).all():
            raise ValueError("points must have shape (n, 3), n >= 4")
        if raw.ndim != 2 or raw.shape[1] != 4 or not len(raw) or not np.issubdtype(raw.dtype, np.integer):
            raise ValueError("cells must have shape (n, 4), n >= 1")
        cells = np.array(raw, dtype=np.int64)
        if np.any(cells < 0) or np.any(cells >= len(pts)):
            raise ValueError("cell vertex outside points")
        if len(np.unique(np.sort(cells, axis=1), axis=0)) != len(cells):
            raise ValueError("duplicate tetrahedron")
        edges = pts[cells[:, 1:]] - pts[cells[:, :1]]
        det = np.linalg.det(edges)
        scale = np.prod(np.linalg.norm(edges, axis=2), axis=1)
        if np.any(np.abs(det) <= 32 * EPS * scale):
            raise ValueError("degenerate tetrahedron")
        neg = det < 0
        cells[neg, 1], cells[neg, 2] = cells[neg, 2].copy(), cells[neg, 1].copy()
        self.points, self.cells = pts, cells
        self.volumes = np.abs(det) / 6
        M = len(cells)
        keys = np.sort(np.stack([np.delete(cells, s, axis=1) for s in range(4)], axis=1), axis=2).reshape(-1, 3)
        uniq, first, inv = np.unique(keys, axis=0, return_index=True, return_inverse=True)
        order = np.argsort(first, kind="stable")
        rank = np.empty_like(order)
        rank[order] = np.arange(len(order))
        face_of = rank[inv.ravel()]
        self.faces = uniq[order]
        self.cell_faces = face_of.reshape(M, 4)
        counts = np.bincount(face_of, minlength=len(self.faces))
        if np.any(counts > 2):
            raise ValueError("nonmanifold triangular face")
        self.face_cells = np.full((len(self.faces), 2), -1, dtype=np.int64)
        occ = np.argsort(face_of, kind="stable")  # per face, its (cell, side) slots in encounter order
        ptr = np.r_[0, np.cumsum(counts)]
        self.face_cells[:, 0] = occ[ptr[:-1]] // 4
        two = counts == 2
        self.face_cells[two, 1] = occ[ptr[:-1][two] + 1] // 4
        fp = pts[self.faces]
        cross = np.cross(fp[:, 1] - fp[:, 0], fp[:, 2] - fp[:, 0])
        self.areas = np.linalg.norm(cross, axis=1) / 2
        self.normals = cross / (2 * self.areas[:, None])
        centres = pts[cells].mean(axis=1)
        mid = fp.mean(axis=1)
        out = np.einsum("fi,fi->f", self.normals, mid - centres[self.face_cells[:, 0]]) < 0
        self.normals[out] *= -1
        self.signs = np.where(np.arange(M)[:, None] == self.face_cells[self.cell_faces, 0], 1, -1).astype(np.int64)
        second = self.face_cells[:, 1] >= 0
        check = np.einsum("fi,fi->f", self.normals[second], mid[second] - centres[self.face_cells[second, 1]])
        if np.any(check > 0):
            raise ValueError("nonmanifold cells overlap across their shared face")
        self.boundary_faces = np.flatnonzero(self.face_cells[:, 1] < 0)

    @classmethod
    def unit_cube(cls, subdivisions: int = 1) -> "TetraMesh":
        """Six conforming Freudenthal tetrahedra per cube of an n^3 grid."""
        n = int(subdivisions)
        if n < 1:
            raise ValueError("subdivisions must be positive")
        points = np.indices((n + 1,) * 3).reshape(3, -1).T / n
        corners = np.array(list(np.ndindex((n,) * 3)), dtype=np.int64)
        cells = []
        for corner in corners:
            for perm in permutations(range(3)):
                node = corner.copy()
                verts = [np.ravel_multi_index(tuple(node), (n + 1,) * 3)]
                for axis in perm:
                    node[axis] += 1
                    verts.append(np.ravel_multi_index(tuple(node), (n + 1,) * 3))
                cells.append(verts)
        return cls(points, np.asarray(cells, dtype=np.int64))

    def submesh(self, cell: int, refinement: int = 2) -> "TetraMesh":
        """Red refinement of one macrocell into refinement^3 tetrahedra."""
        if not 0 <= int(cell) < len(self.cells):
            raise ValueError("cell outside mesh")
        bary, cells = reference_refinement(refinement)
        return TetraMesh(bary @ self.points[self.cells[cell]], cells)


_REFINEMENTS: dict = {}


def reference_refinement(refinement: int) -> tuple[np.ndarray, np.ndarray]:
    """Barycentric points and cells of the red refinement of the reference tetrahedron
    into refinement^3 children (refinement a power of two); new vertices are the edge
    midpoints in order of first use, and each tetrahedron splits into its four corner
    children and four children around the interior octahedron's (ab, cd) diagonal."""
    r = int(refinement)
    if r < 1 or r & (r - 1):
        raise ValueError("refinement must be a power of two")
    if r not in _REFINEMENTS:
        points = [row for row in np.eye(4)]
        cells = [[0, 1, 2, 3]]
        for _ in range(r.bit_length() - 1):
            mids: dict = {}
            out = []
            for a, b, c, d in cells:
                m = []
                for i, j in combinations((a, b, c, d), 2):
                    key = (min(i, j), max(i, j))
                    if key not in mids:
                        mids[key] = len(points)
                        points.append((points[i] + points[j]) / 2)
                    m.append(mids[key])
                ab, ac, ad, bc, bd, cd = m
                out += [[a, ab, ac, ad], [ab, b, bc, bd], [ac, bc, c, cd], [ad, bd, cd, d],
                        [ab, ac, ad, cd], [ab, ac, bc, cd], [ab, ad, bd, cd], [ab, bc, bd, cd]]
            cells = out
        pts, conn = np.asarray(points), np.asarray(cells, dtype=np.int64)
        pts.setflags(write=False)
        conn.setflags(write=False)
        _REFINEMENTS[r] = (pts, conn)
    return _REFINEMENTS[r]


class TriangularSkeleton:
    """Discontinuous Bernstein modes of degree 0 or 1 on every macroface (one
    subtriangle per face): (degree+1)(degree+2)/2 DOFs per face, numbered face by face."""

    def __init__(self, mesh: TetraMesh, degree: int = 1):
        if int(degree) not in (0, 1):
            raise NotImplementedError("the GPU tetrahedral path takes face degrees 0 and 1")
        self.mesh = mesh
        self.degree = int(degree)
        self.modes = (self.degree + 1) * (self.degree + 2) // 2
        self.offsets = np.arange(len(mesh.faces) + 1, dtype=np.int64) * self.modes
        self.size = int(self.offsets[-1])

    def dofs(self, face: int) -> np.ndarray:
        return np.arange(self.offsets[face], self.offsets[face + 1])

    def cell_dofs(self, cell: int) -> np.ndarray:
        return np.concatenate([self.dofs(int(f)) for f in self.mesh.cell_faces[cell]])

    @property
    def cell_dof_array(self) -> np.ndarray:
        f = self.mesh.cell_faces
        return (self.offsets[f][:, :, None] + np.arange(self.modes)[None, None, :]).reshape(len(f), -1)

    def geometric_constraint(self) -> np.ndarray:
        """(cells, 4 modes) G0 = B^T 1: sign * area * (integral of each mode over the
        unit-area face), 1 for degree 0 and 1/3 for each barycentric mode."""
        m = self.mesh
        per = np.full(self.modes, 1.0 if self.degree == 0 else 1.0 / 3.0)
        return (m.signs[:, :, None] * m.areas[m.cell_faces][:, :, None] * per[None, None, :]).reshape(len(m.cells), -1)


def fine_boundary_table(refinement: int, degree: int) -> np.ndarray:
    """Geometry-free trace coupling of the refined reference tetrahedron:
    R[s, a, v] = sum over the fine boundary triangles on side s that contain node a of
    (lambda_v(a) + sum_k lambda_v(k)) / 12 (v a local vertex of the macrocell, lambda
    its barycentric coordinate; degree 0: 1/3 in slot v = s).  The coupling of a cell
    with face area A on side s is sign * A / refinement^2 * R[s, a, vertex of mode j]."""
    bary, cells = reference_refinement(refinement)
    ref = TetraMesh(bary @ np.array([[0.0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]]), cells)
    R = np.zeros((4, len(bary), 4))
    for fface in ref.boundary_faces:
        ids = ref.faces[fface]
        lam = bary[ids]  # (3 nodes, 4 coordinates)
        sides = np.flatnonzero(np.all(lam == 0.0, axis=0))
        if len(sides) != 1:
            raise ValueError("fine boundary face is not on one macro side")
        s = int(sides[0])
        for k, a in enumerate(ids):
            if degree == 0:
                R[s, a, s] += 1.0 / 3.0
            else:
                R[s, a, :] += (lam[k] + lam.sum(axis=0)) / 12.0
    return R


def trace_coupling(mesh: TetraMesh, skeleton: TriangularSkeleton, refinement: int) -> np.ndarray:
    """(cells, nodes, t) coupling of each cell's local P1 nodes with its trace modes
    (``tetra_trace_coupling``, ``fem/traces/triangle_3d.py:221-273``)."""
    R = fine_boundary_table(refinement, skeleton.degree)
    M, n = len(mesh.cells), R.shape[1]
    B = np.zeros((M, n, 4 * skeleton.modes))
    r2 = float(refinement) ** 2
    for s in range(4):
        faces = mesh.cell_faces[:, s]
        scale = mesh.signs[:, s] * mesh.areas[faces] / r2
        if skeleton.degree == 0:
            B[:, :, s] = scale[:, None] * R[s, :, s][None, :]
            continue
        # mode j of the face is the barycentric coordinate of the face's j-th sorted
        # vertex, which is the cell's local vertex `local[:, j]`
        local = np.argmax(mesh.cells[:, None, :] == mesh.faces[faces][:, :, None], axis=2)
        for j in range(3):
            B[:, :, 3 * s + j] = scale[:, None] * R[s][:, local[:, j]].T
    return B


def duffy_tetrahedron(order: int = 5) -> tuple[np.ndarray, np.ndarray]:
    """``tetrahedron_quadrature`` (``fem/scalar/tetrahedron.py:41-52``): a collapsed
    Gauss product rule, barycentric points and weights summing to one."""
    x, w = np.polynomial.legendre.leggauss(order)
    x, w = (x + 1) / 2, w / 2
    a, b, c = np.meshgrid(x, x, x, indexing="ij")
    wa, wb, wc = np.meshgrid(w, w, w, indexing="ij")
    xyz = np.array([a, (1 - a) * b, (1 - a) * (1 - b) * c]).reshape(3, -1).T
    bary = np.column_stack((1 - xyz.sum(axis=1), xyz))
    weights = (6 * wa * wb * wc * (1 - a) ** 2 * (1 - b)).ravel()
    return bary, weights
