"""Neumann faces on whole bottom/top sides: the oracle and the host-side boundary data
against fixtures written by the reference (tests/golden/make_neumann_golden.py)."""

import numpy as np
import pytest

from oracle import q1_mhm as o
from tests._cases import load, rel
from pymhm_b200.workloads import sine_source

NEUMANN_CASES = {
    # name -> (face degree, refinement, permeability(g), source, dirichlet, neumann value)
    "darcy_4x4_r8_p2_noflow_tb": (2, (8, 8), lambda g: o.PixelField(g["kappa"], (1 / 32, 1 / 32)), 1.0,
                                  lambda x: 1.0 - x[:, 0], 0.0),
    "poisson_4x4_r4_p1_flux_bottom": (1, (4, 4), lambda g: 1.0, sine_source, 0.0, lambda x: 0.5 + x[:, 0]),
}


def neumann_map(g, value):
    return {int(f): value for f in g["neumann_faces"]}


@pytest.mark.parametrize("name", list(NEUMANN_CASES))
def test_oracle_matches_reference(name):
    g = load(name)
    deg, ref, perm, src, dr, val = NEUMANN_CASES[name]
    mesh = o.cartesian_mesh(4)
    sk = o.Skeleton(mesh, (o.FaceSpace.uniform(deg),) * len(mesh.faces))
    _, fixed = o.boundary_data(sk, dr, neumann_map(g, val))
    assert np.array_equal(np.array(sorted(fixed)), g["fixed_dofs"])
    assert np.allclose([fixed[k] for k in sorted(fixed)], g["fixed_values"], rtol=0, atol=1e-15)
    sol = o.solve_darcy_q1(mesh, sk, ref, perm(g), src, dr, neumann=neumann_map(g, val))
    for key, val_ in (("trace", sol.trace), ("coarse", sol.coarse), ("fields", sol.fields), ("flux", sol.flux)):
        assert rel(val_, g[key]) <= 1e-12, key
    assert np.array_equal(sol.trace[g["fixed_dofs"]], g["trace"][g["fixed_dofs"]])


@pytest.mark.parametrize("name", list(NEUMANN_CASES))
def test_host_boundary_data_matches_reference(name):
    from pymhm_b200.topology import (CartesianMacroMesh, FaceSpace, SkeletonSpace, boundary_data, neumann_fixed,
                                     neumann_sides)

    g = load(name)
    deg, ref, perm, src, dr, val = NEUMANN_CASES[name]
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(deg),) * len(mesh.faces))
    neu = neumann_map(g, val)
    assert np.array_equal(boundary_data(sk, dr, 4, neu), g["boundary"])
    dofs, values = neumann_fixed(sk, neu, 4)
    order = np.argsort(dofs)
    assert np.array_equal(dofs[order], g["fixed_dofs"])
    assert np.allclose(values[order], g["fixed_values"], rtol=0, atol=1e-15)
    assert neumann_sides(mesh, neu) == (3 if name.startswith("darcy") else 1)


def test_neumann_side_rules():
    from pymhm_b200.topology import CartesianMacroMesh, neumann_sides

    mesh = CartesianMacroMesh(4)
    pts = mesh.points[mesh.faces[mesh.boundary_faces]]
    bottom = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 1] == 0.0)]
    top = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 1] == 1.0)]
    left = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 0] == 0.0)]
    assert neumann_sides(mesh, None) == 0
    assert neumann_sides(mesh, {f: 0.0 for f in top}) == 2
    with pytest.raises(NotImplementedError, match="whole bottom and top sides"):
        neumann_sides(mesh, {f: 0.0 for f in bottom[:2]})
    with pytest.raises(NotImplementedError, match="whole bottom and top sides"):
        neumann_sides(mesh, {f: 0.0 for f in left})
    with pytest.raises(NotImplementedError):
        neumann_sides(mesh, {int(f): 0.0 for f in mesh.boundary_faces})
