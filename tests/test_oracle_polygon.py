"""Polygon macro meshes, P2 local spaces and the config-3 oracle against fixtures
written by the reference itself (``tests/golden/make_polygon_golden.py``)."""

import numpy as np
import pytest

from oracle import polygon_mhm as op
from pymhm_b200.polygon import EdgeSkeleton, p2_nodal_space, p2_trace_coupling, voronoi_mesh
from pymhm_b200.workloads import DiscInclusions, disc_inclusions
from tests._cases import load, rel

POLYGON_CASES = ("polygon_voronoi12_p2_discs", "polygon_voronoi40_p2_discs")


def polygon_case(name):
    g = load(name)
    count, seed = int(g["count"]), int(g["seed"])
    mesh = voronoi_mesh(count, seed)
    sk = EdgeSkeleton(mesh)
    fines = [mesh.submesh(c, int(g["refinements"][c])) for c in range(count)]
    centres, radii = disc_inclusions(int(g["discs"][0]), rmin=0.04, rmax=0.09, seed=seed + 2)
    return g, mesh, sk, fines, DiscInclusions(centres, radii)


@pytest.mark.parametrize("name", POLYGON_CASES)
def test_polygon_topology_is_the_reference(name):
    g, mesh, sk, fines, _ = polygon_case(name)
    assert np.array_equal(mesh.points, g["points"])
    assert np.array_equal(mesh.faces, g["faces"]) and np.array_equal(mesh.face_cells, g["face_cells"])
    assert np.array_equal(np.concatenate(mesh.cells), g["cells"])
    assert np.array_equal(np.concatenate(mesh.cell_faces), g["cell_faces"])
    assert np.array_equal(np.concatenate(mesh.signs), g["signs"])
    assert np.array_equal(sk.offsets, g["offsets"])
    sizes = [len(p2_nodal_space(f)[1]) for f in fines]
    assert np.array_equal(np.r_[0, np.cumsum(sizes)], g["field_ptr"])


@pytest.mark.parametrize("name", POLYGON_CASES)
def test_polygon_oracle_matches_reference(name):
    g, mesh, sk, fines, field = polygon_case(name)
    sol = op.solve_darcy_p2(mesh, sk, fines, field, 1.0, keep_responses=True)
    from scipy import sparse

    from tests._full_size import pattern_differences

    m = sol["matrix"]
    N = len(g["rhs"])
    ref = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    scale = np.max(np.abs(ref.data))
    # The coarse-coarse entries -(A^T 1)^T E are rounding residues of the assembled
    # operator's column sums, magnified by the 1e4 contrast: they (and whether one of
    # them is exactly 0.0) depend on the last bits of A.  Everything else agrees closely.
    assert np.max(np.abs((m - ref).toarray())) <= 1e-8 * scale
    r, c, mine, theirs = pattern_differences(m, ref)
    assert np.all(mine <= 1e-8 * scale) and np.all(theirs <= 1e-8 * scale)
    # the residues above move the solution by ~1e-11: the FP64 parity bar applies
    for key in ("trace", "coarse"):
        assert rel(sol[key], g[key]) <= 1e-10, key
    assert rel(np.concatenate(sol["fields"]), g["fields"]) <= 1e-10
    assert np.array_equal(sol["corrected"], g["corrected"])
    for c in g["keep_cells"]:
        p = sol["responses"][c].problem
        assert np.max(np.abs(p.matrix.toarray() - g[f"cell{c}_A"])) <= 1e-15 * np.max(np.abs(g[f"cell{c}_A"]))
        assert np.max(np.abs(p.coupling - g[f"cell{c}_B"])) <= 1e-15 * np.max(np.abs(g[f"cell{c}_B"]))
        assert rel(p.load, g[f"cell{c}_f"]) <= 1e-14
        assert rel(p.constraints[:, 0], g[f"cell{c}_C"]) <= 1e-14


def test_p2_coupling_columns_sum_to_the_geometric_constraint():
    g, mesh, sk, fines, _ = polygon_case(POLYGON_CASES[0])
    for c, fine in enumerate(fines):
        B = p2_trace_coupling(mesh, c, fine, sk)
        g0 = sk.geometric_constraint(c)
        assert np.allclose(B.sum(axis=0), g0, rtol=1e-13, atol=1e-14 * np.max(np.abs(g0)))
