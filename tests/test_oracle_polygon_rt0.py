"""The mixed RT0 / P0 polygon provider: host topology (``rt0_space``, the flux map)
and the oracle against fixtures written by the reference itself
(``tests/golden/make_polygon_rt0_golden.py``)."""

import numpy as np
import pytest

from oracle import polygon_mhm as op
from pymhm_b200.polygon import EdgeSkeleton, check_rt0_skeleton, rt0_space, voronoi_mesh
from pymhm_b200.topology import FaceSpace
from pymhm_b200.workloads import DiscInclusions, disc_inclusions
from tests._cases import load, rel

RT0_CASES = ("polygon_voronoi12_rt0_discs", "polygon_voronoi20_rt0s2_discs")


def rt0_case(name):
    g = load(name)
    count, seed = int(g["count"]), int(g["seed"])
    mesh = voronoi_mesh(count, seed)
    sk = EdgeSkeleton(mesh, FaceSpace.uniform(0, int(g["segments"][0])))
    fines = [mesh.submesh(c, int(g["refinements"][c])) for c in range(count)]
    centres, radii = disc_inclusions(int(g["discs"][0]), rmin=0.04, rmax=0.09, seed=seed + 2)
    return g, mesh, sk, fines, DiscInclusions(centres, radii)


@pytest.mark.parametrize("name", RT0_CASES)
def test_rt0_local_problems_are_the_reference(name):
    g, mesh, sk, fines, field = rt0_case(name)
    for c in g["keep_cells"]:
        p = op.mixed_local_problem(mesh, sk, int(c), fines[c], field, 1.0)
        A = g[f"cell{c}_A"]
        assert p.matrix.shape == A.shape
        assert np.max(np.abs(p.matrix.toarray() - A)) <= 1e-13 * np.max(np.abs(A))
        assert np.array_equal(p.coupling, g[f"cell{c}_B"])
        assert np.array_equal(p.load, g[f"cell{c}_f"])
        assert np.array_equal(p.constraints[:, 0], g[f"cell{c}_C"])
        assert np.array_equal(p.kernel[:, 0], g[f"cell{c}_Z"])


@pytest.mark.parametrize("name", RT0_CASES)
def test_rt0_oracle_matches_reference(name):
    from scipy import sparse

    g, mesh, sk, fines, field = rt0_case(name)
    sol = op.solve_darcy_p2(mesh, sk, fines, field, 1.0, keep_responses=True, formulation="mixed")
    N = len(g["rhs"])
    ref = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    assert np.max(np.abs((sol["matrix"] - ref).toarray())) <= 1e-10 * np.max(np.abs(ref.data))
    for key in ("trace", "coarse"):
        assert rel(sol[key], g[key]) <= 1e-10, key
    assert rel(np.concatenate(sol["fields"]), g["fields"]) <= 1e-10
    assert np.array_equal(sol["corrected"], g["corrected"])
    for c in g["keep_cells"]:
        resp = sol["responses"][c]
        assert rel(resp.lifts, g[f"cell{c}_lifts"]) <= 1e-10


def test_rt0_space_slots():
    """Every element's valid slots name its own unknowns; the padding multiplier slots
    name distinct multipliers; every unknown is some element's valid slot; the declared
    kernel is an exact kernel of the assembled saddle."""
    mesh = voronoi_mesh(12, 3)
    sk = EdgeSkeleton(mesh, FaceSpace.uniform(0))
    for c, r in ((0, 1), (5, 2), (7, 3)):
        fine = mesh.submesh(c, r)
        slots, valid, info, kernel = rt0_space(fine)
        n = len(fine.faces) + len(fine.cells) + len(fine.boundary_faces)
        assert len(kernel) == n
        assert all(len(set(row)) == 6 for row in slots)
        assert np.array_equal(np.unique(slots[valid]), np.arange(n))
        assert np.array_equal(info[:, :3], fine.signs)
        p = op.mixed_local_problem(mesh, sk, c, fine, 1.0, 1.0)
        assert not np.any(p.matrix @ kernel)


def test_rt0_skeleton_alignment():
    mesh = voronoi_mesh(12, 3)
    check_rt0_skeleton(EdgeSkeleton(mesh, FaceSpace.uniform(0, 2)), [2, 4])
    with pytest.raises(ValueError, match="aligned"):
        check_rt0_skeleton(EdgeSkeleton(mesh, FaceSpace.uniform(0, 2)), [2, 3])
    with pytest.raises(ValueError, match="aligned"):
        check_rt0_skeleton(EdgeSkeleton(mesh, FaceSpace.uniform(1)), [2])


def test_rt0_solve_darcy_arguments():
    """The reference's argument errors (``primal.py:149-152, 245-249``), raised before
    any device work."""
    from pymhm_b200.polygon_darcy import solve_darcy

    mesh = voronoi_mesh(12, 3)
    with pytest.raises(ValueError, match="degree=1"):
        solve_darcy(mesh, formulation="mixed", degree=2)
    with pytest.raises(ValueError, match="formulation"):
        solve_darcy(mesh, formulation="dual")
