"""Polygonal macro meshes, their local triangulations and P2 nodal spaces (config 3).

Host-side topology, built once per mesh.  It fixes the global numbering of the trace
unknowns and the local node numbering, so it follows the reference's construction
(PyMHM 1.3.2, ``src/pymhm/``):

* ``TriangleMesh``: ``meshes/triangle.py:13-84``.  Clockwise cells are reoriented
  (vertices 1 and 2 swapped); side s of a cell is the edge from its vertex s to vertex
  s+1; edges are numbered by first encounter over (cell, side) and keep the first
  cell's orientation, which carries sign +1 and the second cell -1.
* ``PolygonMesh``: ``meshes/polygonal.py:60-265``.  Cells are reoriented
  counterclockwise; each cell is ear-clipped (``_triangulate``); with
  ``local_triangulation="boundary"`` the cell is instead fanned from its area centroid
  when every edge sees it, else every ear is fanned from its own centroid; macrofaces
  are the polygon edges, numbered and signed like the triangle mesh's.
  ``submesh(cell, r)`` refines every base triangle into r^2 triangles, nodes keyed by
  their exact barycentric weights on the base vertices so shared edges share nodes.
* ``nodal_space``: ``fem/scalar/triangle.py:65-92`` for degree 2: the vertices, then
  one midpoint per fine edge in edge order.
* ``voronoi_mesh``: the Voronoi cells of seeded points in the unit square, bounded by
  reflecting the seeds across the four sides (as ``examples/polygon_meshes.py:61-98``
  does for its hexagon family), boundary coordinates snapped to 0 and 1.
"""

from __future__ import annotations

import numpy as np

EPS = np.finfo(float).eps


def _cross(a, b):
    return a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]


class TriangleMesh:
    """Conforming planar triangles with signed edge incidence (see the module docstring)."""

    def __init__(self, points, cells):
        pts = np.array(points, dtype=float)
        cells = np.array(cells, dtype=np.int64)
        if pts.ndim != 2 or pts.shape[1] != 2 or cells.ndim != 2 or cells.shape[1] != 3 or not len(cells):
            raise ValueError("points must have shape (n, 2) and cells (m, 3)")
        v = pts[cells]
        a, b = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
        det = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
        if np.any(np.abs(det) <= EPS * np.linalg.norm(a, axis=1) * np.linalg.norm(b, axis=1)):
            raise ValueError("degenerate triangle")
        rev = det < 0
        cells[rev] = cells[rev][:, [0, 2, 1]]
        self.points, self.cells = pts, cells
        lookup: dict = {}
        faces, neighbors = [], []
        self.cell_faces = np.empty_like(cells)
        self.signs = np.empty_like(cells)
        for c, nodes in enumerate(cells):
            for s in range(3):
                i, j = int(nodes[s]), int(nodes[(s + 1) % 3])
                key = (min(i, j), max(i, j))
                if key not in lookup:
                    lookup[key] = len(faces)
                    faces.append((i, j))
                    neighbors.append([c, -1])
                    sign = 1
                else:
                    f = lookup[key]
                    if neighbors[f][1] != -1 or faces[f] == (i, j):
                        raise ValueError("nonmanifold face or overlapping cell orientation")
                    neighbors[f][1] = c
                    sign = -1
                self.cell_faces[c, s] = lookup[key]
                self.signs[c, s] = sign
        self.faces = np.array(faces, dtype=np.int64)
        self.face_cells = np.array(neighbors, dtype=np.int64)

    @property
    def boundary_faces(self):
        return np.flatnonzero(self.face_cells[:, 1] == -1)

    @property
    def areas(self):
        v = self.points[self.cells]
        a, b = v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]
        return (a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]) / 2


def ear_triangulation(points: np.ndarray) -> np.ndarray:
    """``_triangulate`` (``polygonal.py:33-57``): ear clipping of one simple
    counterclockwise polygon, the first valid ear in the current vertex order each time."""
    remaining = list(range(len(points)))
    triangles = []
    scale = float(np.max(np.ptp(points, axis=0)))
    tol = 64 * EPS * scale * scale
    while len(remaining) > 3:
        for j, b in enumerate(remaining):
            a, c = remaining[j - 1], remaining[(j + 1) % len(remaining)]
            if _cross(points[b] - points[a], points[c] - points[a]) <= tol:
                continue
            other = [v for v in remaining if v not in (a, b, c)]
            verts = points[[a, b, c]]
            diff = points[other, None, :] - verts[None, :, :]
            signs = _cross(np.roll(verts, -1, axis=0) - verts, diff)
            if np.any(np.all(signs >= -tol, axis=1)):
                continue
            triangles.append((a, b, c))
            remaining.pop(j)
            break
        else:
            raise ValueError("polygon must be simple and have resolvable nondegenerate ears")
    triangles.append((remaining[0], remaining[1], remaining[2]))
    return np.asarray(triangles, dtype=np.int64)


class PolygonMesh:
    """Planar polygon macrocells with oriented edges (see the module docstring)."""

    def __init__(self, points, cells, local_triangulation: str = "ears"):
        if local_triangulation not in ("ears", "boundary"):
            raise ValueError("local_triangulation must be ears or boundary")
        pts = np.array(points, dtype=float)
        self.points = pts
        self.local_triangulation = local_triangulation
        lookup: dict = {}
        faces, neighbors = [], []
        self.cells, self.cell_faces, self.signs, self._triangles = [], [], [], []
        for c, raw in enumerate(cells):
            idx = np.asarray(raw, dtype=np.int64).copy()
            xy = pts[idx]
            area = float(np.sum(_cross(xy - xy[0], np.roll(xy, -1, axis=0) - xy[0])) / 2)
            if area < 0:
                idx = idx[::-1].copy()
                xy = pts[idx]
            self._triangles.append(ear_triangulation(xy))
            lf, ls = [], []
            for a, b in zip(idx, np.roll(idx, -1)):
                key = (min(int(a), int(b)), max(int(a), int(b)))
                if key not in lookup:
                    lookup[key] = len(faces)
                    faces.append((int(a), int(b)))
                    neighbors.append([c, -1])
                    sign = 1
                else:
                    f = lookup[key]
                    if neighbors[f][1] != -1 or faces[f] == (a, b):
                        raise ValueError("nonmanifold macroface or overlapping cell orientation")
                    neighbors[f][1] = c
                    sign = -1
                lf.append(lookup[key])
                ls.append(sign)
            self.cells.append(idx)
            self.cell_faces.append(np.asarray(lf, dtype=np.int64))
            self.signs.append(np.asarray(ls, dtype=np.int64))
        self.faces = np.asarray(faces, dtype=np.int64)
        self.face_cells = np.asarray(neighbors, dtype=np.int64)

    @property
    def lengths(self):
        return np.linalg.norm(self.points[self.faces[:, 1]] - self.points[self.faces[:, 0]], axis=1)

    @property
    def boundary_faces(self):
        return np.flatnonzero(self.face_cells[:, 1] < 0)

    def base_triangles(self, cell: int):
        """The cell's vertices (with a fan centre when the triangulation adds one) and
        its base triangles (``submesh``, ``polygonal.py:233-255``)."""
        vertices = self.points[self.cells[cell]]
        base = self._triangles[cell]
        if self.local_triangulation == "boundary":
            corners = vertices[base]
            areas = _cross(corners[:, 1] - corners[:, 0], corners[:, 2] - corners[:, 0]) / 2
            center = areas @ corners.mean(axis=1) / areas.sum()
            n = len(vertices)
            tol = 64 * EPS * np.max(np.ptp(vertices, axis=0)) ** 2
            if np.all(_cross(np.roll(vertices, -1, axis=0) - vertices, center - vertices) > tol):
                vertices = np.vstack((vertices, center))
                base = np.column_stack((np.arange(n), np.roll(np.arange(n), -1), np.full(n, n)))
            else:
                vertices = np.vstack((vertices, corners.mean(axis=1)))
                base = np.array([(int(a), int(b), n + k) for k, tri in enumerate(base)
                                 for a, b in zip(tri, np.roll(tri, -1))])
        return vertices, base

    def submesh(self, cell: int, subdivisions: int) -> TriangleMesh:
        """Conforming refinement of the cell's base triangles into r^2 triangles each."""
        r = int(subdivisions)
        vertices, base = self.base_triangles(cell)
        lookup: dict = {}
        points, triangles = [], []
        for tri in base:
            local = {}
            for i in range(r + 1):
                for j in range(r + 1 - i):
                    weights = (r - i - j, i, j)
                    key = tuple(sorted((int(v), w) for v, w in zip(tri, weights) if w))
                    if key not in lookup:
                        lookup[key] = len(points)
                        points.append(np.asarray(weights) @ vertices[tri] / r)
                    local[i, j] = lookup[key]
            for i in range(r):
                for j in range(r - i):
                    triangles.append((local[i, j], local[i + 1, j], local[i, j + 1]))
                    if i + j < r - 1:
                        triangles.append((local[i + 1, j], local[i + 1, j + 1], local[i, j + 1]))
        return TriangleMesh(np.asarray(points), np.asarray(triangles, dtype=np.int64))


def p2_nodal_space(mesh: TriangleMesh):
    """``nodal_space`` for degree 2 (``triangle.py:65-92``): DOFs per triangle in the
    order (vertices, midpoints of the edges (0,1), (1,2), (2,0)) and node coordinates."""
    dofs = np.empty((len(mesh.cells), 6), dtype=np.int64)
    dofs[:, :3] = mesh.cells
    mid = (mesh.points[mesh.faces[:, 0]] * 0.5 + mesh.points[mesh.faces[:, 1]] * 0.5)
    nv = len(mesh.points)
    dofs[:, 3:] = nv + mesh.cell_faces
    return dofs, np.concatenate((mesh.points, mid))


def voronoi_mesh(count: int, seed: int, local_triangulation: str = "boundary") -> PolygonMesh:
    """Voronoi cells of ``count`` PCG64-uniform seeds in the unit square, bounded by the
    seeds' reflections across the four sides."""
    from scipy.spatial import Voronoi

    rng = np.random.Generator(np.random.PCG64(seed))
    seeds = rng.uniform(0.0, 1.0, size=(count, 2))
    copies = [seeds]
    for x in (-1, 0, 1):
        for y in (-1, 0, 1):
            if x == y == 0:
                continue
            shifted = seeds.copy()
            if x:
                shifted[:, 0] = -seeds[:, 0] + (2 if x == 1 else 0)
            if y:
                shifted[:, 1] = -seeds[:, 1] + (2 if y == 1 else 0)
            copies.append(shifted)
    vor = Voronoi(np.vstack(copies))
    regions = [np.asarray(vor.regions[r]) for r in vor.point_region[:count]]
    used = np.unique(np.concatenate(regions))
    if np.any(used < 0):
        raise RuntimeError("reflected Voronoi seeds must give bounded cells")
    remap = np.full(len(vor.vertices), -1)
    remap[used] = np.arange(len(used))
    coords = np.clip(vor.vertices[used], 0, 1)
    for b in (0.0, 1.0):
        coords[np.abs(coords - b) <= 64 * EPS] = b
    return PolygonMesh(coords, [remap[c] for c in regions], local_triangulation=local_triangulation)


class EdgeSkeleton:
    """One ``FaceSpace`` (``fem/traces/interval.py:13-116``) on every polygon edge,
    DOFs numbered edge by edge (``SkeletonSpace``, ``:119-161``); a cell's trace DOFs
    are its edges' blocks in side order."""

    def __init__(self, mesh: PolygonMesh, space=None):
        from .topology import FaceSpace

        self.mesh = mesh
        self.space = FaceSpace.uniform(1) if space is None else FaceSpace.of(space)
        self.modes = self.space.size
        self.offsets = np.arange(len(mesh.faces) + 1, dtype=np.int64) * self.modes
        self.size = int(self.offsets[-1])

    def dofs(self, face: int) -> np.ndarray:
        return np.arange(self.offsets[face], self.offsets[face + 1])

    def cell_dofs(self, cell: int) -> np.ndarray:
        return np.concatenate([self.dofs(int(f)) for f in self.mesh.cell_faces[cell]])

    def geometric_constraint(self, cell: int) -> np.ndarray:
        """G0 = B^T 1 of the cell: sign * length * the integral of each mode over [0, 1]."""
        moments = self.space.moments()
        m = self.mesh
        lengths = m.lengths[m.cell_faces[cell]]
        return (m.signs[cell][:, None] * lengths[:, None] * moments[None, :]).ravel()


def p2_trace_coupling(coarse: PolygonMesh, cell: int, fine: TriangleMesh, skeleton: EdgeSkeleton) -> np.ndarray:
    """``trace_coupling`` (``fem/scalar/triangle.py:160-205``) for P2 nodes: on every
    fine boundary edge lying on a macro edge, sign * length * Gauss sum of the P2
    interval basis (nodes 0, 1, 1/2) times the face space's modes, split at its breaks."""
    from numpy.polynomial.legendre import leggauss

    degree = 2
    space = skeleton.space
    nv = len(fine.points)
    width = skeleton.modes * len(coarse.cell_faces[cell])
    matrix = np.zeros((nv + len(fine.faces), width))
    gauss, gw = leggauss(max(space.degrees) + degree + 1)
    nodes_1d = np.r_[0.0, 1.0, 0.5]
    for side, face in enumerate(coarse.cell_faces[cell]):
        start, end = coarse.points[coarse.faces[face]]
        tangent = end - start
        length = np.linalg.norm(tangent)
        sign = coarse.signs[cell][side]
        for ff in fine.boundary_faces:
            nodes = fine.faces[ff]
            coords = fine.points[nodes]
            t = (coords - start) @ tangent / length ** 2
            if (not np.allclose(coords, start + t[:, None] * tangent, atol=1e-12, rtol=1e-12)
                    or min(t) < -1e-12 or max(t) > 1 + 1e-12):
                continue
            lo, hi = np.clip(np.sort(t), 0, 1)
            cuts = sorted({lo, hi, *(b for b in space.breaks if lo < b < hi)})
            ids = np.r_[nodes, nv + ff]
            for left, right in zip(cuts[:-1], cuts[1:]):
                param = left + (gauss + 1) * (right - left) / 2
                w = gw * (right - left) / 2 * length * sign
                s = (param - t[0]) / (t[1] - t[0])
                # interval P2 Lagrange basis on the nodes 0, 1, 1/2
                basis = np.stack([np.prod([(s - nodes_1d[m]) / (nodes_1d[k] - nodes_1d[m])
                                           for m in range(3) if m != k], axis=0) for k in range(3)], axis=1)
                matrix[ids, side * skeleton.modes:(side + 1) * skeleton.modes] += basis.T @ (
                    w[:, None] * space.evaluate(param))
    return matrix


def rt0_space(fine: TriangleMesh):
    """Unknowns of the mixed RT0 / P0 local problem (``normal_flux_blocks``,
    ``fem/hdiv/mixed.py:77-112``: the fine faces' fluxes, the fine cells' pressures, the
    boundary faces' multipliers in ``fine.boundary_faces`` order) and every fine
    triangle's six element slots (its three faces, its pressure, two multipliers).

    Returns ``(slots, valid, info, kernel)``: slots (triangles, 6) local unknowns;
    valid marks the slots that hold the triangle's own unknowns (a triangle's boundary
    faces select their multipliers; the other multiplier slots name distinct
    multipliers with zero entries); info (triangles, 5) the faces' signs and the local
    faces the two multiplier slots select (-1 for none); kernel the declared kernel Z
    (zero fluxes, unit pressures and multipliers)."""
    nq, npres = len(fine.faces), len(fine.cells)
    bfaces = fine.boundary_faces
    nb = len(bfaces)
    where = np.full(nq, -1, dtype=np.int64)
    where[bfaces] = np.arange(nb)
    slots = np.empty((npres, 6), dtype=np.int64)
    valid = np.ones((npres, 6), dtype=bool)
    info = np.full((npres, 5), -1, dtype=np.int32)
    slots[:, :3] = fine.cell_faces
    slots[:, 3] = nq + np.arange(npres)
    info[:, :3] = fine.signs
    for t in range(npres):
        own = [(s, int(where[f])) for s, f in enumerate(fine.cell_faces[t]) if where[f] >= 0]
        if len(own) > 2:
            raise NotImplementedError("a fine triangle with three boundary faces (a one-triangle local mesh)")
        taken = {k for _, k in own}
        spare = (k for k in range(nb) if k not in taken)
        for m in range(2):
            if m < len(own):
                info[t, 3 + m] = own[m][0]
                slots[t, 4 + m] = nq + npres + own[m][1]
            else:
                valid[t, 4 + m] = False
                slots[t, 4 + m] = nq + npres + next(spare)
    kernel = np.r_[np.zeros(nq), np.ones(npres + nb)]
    return slots, valid, info, kernel


def rt0_flux_map(coarse: PolygonMesh, cell: int, fine: TriangleMesh, skeleton: EdgeSkeleton) -> np.ndarray:
    """The RT0 half of ``face_integration`` (``fem/scalar/operators.py:200-244``): per fine
    boundary face (rows in ``fine.boundary_faces`` order) lying on a macro edge, the
    integrated outward flux of each trace mode, sign * length * Gauss sum of the modes
    on the face's parameter interval split at the space's breaks."""
    from numpy.polynomial.legendre import leggauss

    space = skeleton.space
    bfaces = fine.boundary_faces
    rt = np.zeros((len(bfaces), skeleton.modes * len(coarse.cell_faces[cell])))
    gauss, gw = leggauss(max(space.degrees) + 2)
    for side, face in enumerate(coarse.cell_faces[cell]):
        start, end = coarse.points[coarse.faces[face]]
        tangent = end - start
        length2 = tangent @ tangent
        sign = coarse.signs[cell][side]
        cols = slice(side * skeleton.modes, (side + 1) * skeleton.modes)
        for row, ff in enumerate(bfaces):
            coords = fine.points[fine.faces[ff]]
            t = (coords - start) @ tangent / length2
            if (not np.allclose(coords, start + t[:, None] * tangent, atol=1e-12, rtol=1e-12)
                    or min(t) < -1e-12 or max(t) > 1 + 1e-12):
                continue
            lo, hi = np.clip(np.sort(t), 0, 1)
            cuts = sorted({lo, hi, *(b for b in space.breaks if lo < b < hi)})
            for left, right in zip(cuts[:-1], cuts[1:]):
                param = left + (gauss + 1) * (right - left) / 2
                w = gw * (right - left) / 2 * np.sqrt(length2) * sign
                rt[row, cols] += w @ space.evaluate(param)
    return rt


def rt0_coupling(coarse: PolygonMesh, cell: int, fine: TriangleMesh, skeleton: EdgeSkeleton) -> np.ndarray:
    """The mixed coupling of ``normal_flux_blocks``: minus the flux map on the boundary
    multipliers' rows, zero on the fluxes and pressures."""
    rt = rt0_flux_map(coarse, cell, fine, skeleton)
    out = np.zeros((len(fine.faces) + len(fine.cells) + rt.shape[0], rt.shape[1]))
    out[len(fine.faces) + len(fine.cells):] = -rt
    return out


def check_rt0_skeleton(skeleton: EdgeSkeleton, refinements) -> None:
    """``_DarcyLocalFactory``'s RT0 condition (``primal.py:81-90``): degree-zero trace
    segments whose breaks fall on the fine edges of every cell's refinement."""
    space = skeleton.space
    if any(space.degrees):
        raise ValueError("RT0 needs degree-zero trace segments aligned with fine edges")
    for r in np.unique(np.asarray(refinements, dtype=np.int64)):
        b = np.array(space.breaks) * r
        if not np.allclose(b, np.round(b), atol=1e-12, rtol=0):
            raise ValueError("RT0 needs degree-zero trace segments aligned with fine edges")


def _cell_local_data(args):
    """Worker of ``local_data``: (fine mesh, local space, trace coupling) per cell."""
    coarse, skeleton, cells, refinements, formulation = args
    out = []
    for c, r in zip(cells, refinements):
        fine = coarse.submesh(int(c), int(r))
        if formulation == "mixed":
            out.append((fine, rt0_space(fine), rt0_coupling(coarse, int(c), fine, skeleton)))
        else:
            out.append((fine, p2_nodal_space(fine), p2_trace_coupling(coarse, int(c), fine, skeleton)))
    return out


def local_data(coarse: PolygonMesh, skeleton: EdgeSkeleton, refinements, workers: int = 1,
               formulation: str = "primal"):
    """Every cell's refined local mesh, local space (P2 nodes, or the RT0 / P0 slots of
    ``rt0_space`` for ``formulation="mixed"``) and trace coupling (host work of a
    polygon plan, independent per cell).  With ``workers`` > 1, batches of a few hundred
    cells and more are split over that many spawned processes (the same functions, so
    the same results); spawned children import the calling program's main module, so a
    script that asks for workers keeps its top-level work under
    ``if __name__ == "__main__":``."""
    M = len(coarse.cells)
    rs = np.broadcast_to(np.asarray(refinements, dtype=np.int64), (M,))
    if M < 256 or workers < 2:
        return _cell_local_data((coarse, skeleton, range(M), rs, formulation))
    import multiprocessing
    from concurrent.futures import ProcessPoolExecutor

    parts = [p for p in np.array_split(np.arange(M), 4 * workers) if len(p)]
    with ProcessPoolExecutor(workers, mp_context=multiprocessing.get_context("spawn")) as pool:
        done = pool.map(_cell_local_data, [(coarse, skeleton, p, rs[p], formulation) for p in parts])
        return [item for part in done for item in part]
