"""The mixed RT0 / P0 polygon path on the GPU (``PolygonP2Plan(formulation="mixed")``,
``solve_darcy(formulation="mixed")``) against fixtures written by the reference
(``tests/golden/make_polygon_rt0_golden.py``) and against the oracle."""

import numpy as np
import pytest

from oracle import polygon_mhm as op
from pymhm_b200.polygon import EdgeSkeleton, voronoi_mesh
from pymhm_b200.topology import FaceSpace
from pymhm_b200.workloads import DiscInclusions, disc_inclusions
from tests._cases import rel
from tests.test_oracle_polygon_rt0 import RT0_CASES, rt0_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ragged", [True, False])
@pytest.mark.parametrize("name", RT0_CASES)
def test_gpu_rt0_matches_reference(name, ragged):
    from pymhm_b200.polygon_darcy import PolygonP2Plan

    g, mesh, sk, fines, field = rt0_case(name)
    plan = PolygonP2Plan(mesh, sk, g["refinements"], formulation="mixed", ragged=ragged)
    sol = plan.solve(field, 1.0)
    for key in ("trace", "coarse"):
        assert rel(getattr(sol, key), g[key]) <= 1e-9, key
    assert rel(np.concatenate(sol.fields), g["fields"]) <= 1e-9
    assert np.array_equal(sol.corrected, g["corrected"])
    # the plan keeps the negated blocks (the same solution, a positive semi-definite
    # trace block for the global PCG)
    for c in g["keep_cells"]:
        ref = g[f"cell{c}_block"]
        assert np.max(np.abs(plan.cell_block(int(c)) + ref)) <= 1e-11 * np.max(np.abs(ref))


def test_gpu_rt0_solve_darcy_against_oracle():
    """Uneven refinements 1-5 over 60 Voronoi cells (local orders 12 to 490),
    constant permeability, through ``solve_darcy``."""
    from pymhm_b200.polygon_darcy import solve_darcy

    mesh = voronoi_mesh(60, 17)
    rs = np.random.Generator(np.random.PCG64(5)).integers(1, 6, size=60)
    sol = solve_darcy(mesh, formulation="mixed", degree=1, permeability=3.0, source=-2.0, local_refinement=rs)
    sk = EdgeSkeleton(mesh, FaceSpace.uniform(0))
    fines = [mesh.submesh(c, int(rs[c])) for c in range(60)]
    ref = op.solve_darcy_p2(mesh, sk, fines, 3.0, -2.0, formulation="mixed")
    assert rel(sol.trace, ref["trace"]) <= 1e-9
    assert rel(sol.coarse, ref["coarse"]) <= 1e-9
    assert rel(np.concatenate(sol.fields), np.concatenate(ref["fields"])) <= 1e-9


def test_gpu_rt0_discs_two_segments_against_oracle():
    """Two flux segments per edge, even refinements, 1e4-contrast discs."""
    from pymhm_b200.polygon_darcy import PolygonP2Plan

    mesh = voronoi_mesh(40, 29)
    rs = np.random.Generator(np.random.PCG64(6)).choice(np.array([2, 4]), size=40)
    sk = EdgeSkeleton(mesh, FaceSpace.uniform(0, 2))
    centres, radii = disc_inclusions(50, rmin=0.04, rmax=0.09, seed=31)
    field = DiscInclusions(centres, radii)
    sol = PolygonP2Plan(mesh, sk, rs, formulation="mixed").solve(field, 1.0)
    fines = [mesh.submesh(c, int(rs[c])) for c in range(40)]
    ref = op.solve_darcy_p2(mesh, sk, fines, field, 1.0, formulation="mixed")
    assert rel(sol.trace, ref["trace"]) <= 1e-9
    assert rel(np.concatenate(sol.fields), np.concatenate(ref["fields"])) <= 1e-9


def test_gpu_rt0_rejects_unaligned_and_large():
    from pymhm_b200.polygon_darcy import PolygonP2Plan, solve_darcy

    mesh = voronoi_mesh(12, 3)
    with pytest.raises(ValueError, match="aligned"):
        PolygonP2Plan(mesh, EdgeSkeleton(mesh, FaceSpace.uniform(0, 2)), 3, formulation="mixed")
    with pytest.raises(ValueError, match="degree=1"):
        solve_darcy(mesh, formulation="mixed", degree=2)
    with pytest.raises(NotImplementedError, match="mixed local problems"):
        PolygonP2Plan(mesh, EdgeSkeleton(mesh, FaceSpace.uniform(0)), 12, formulation="mixed")
