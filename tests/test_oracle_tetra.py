"""The 3D P1 tetrahedral oracle and host topology against fixtures written by the
reference itself (``tests/golden/make_tetra_golden.py``)."""

import numpy as np
import pytest

from oracle import tetra_mhm as ot
from pymhm_b200.tetra import TetraMesh, TriangularSkeleton, duffy_tetrahedron, trace_coupling
from pymhm_b200.workloads import LayeredField, digest, layered_lognormal_permeability
from tests._cases import load, rel

# name -> (cube subdivisions, local refinement, face degree)
TETRA_CASES = {
    "tetra_cube2_r4_p1_layered": (2, 4, 1),
    "tetra_cube1_r8_p1_layered": (1, 8, 1),
    "tetra_cube2_r2_p0_layered": (2, 2, 0),
}


def tetra_case(name):
    g = load(name)
    cube, r, deg = TETRA_CASES[name]
    layers, pixels, seed = (int(v) for v in g["kappa_args"])
    values = layered_lognormal_permeability(layers, pixels, sigma=3.0, ell=0.1, contrast=1e6, seed=seed)
    assert digest(values) == str(g["kappa_sha256"])
    mesh = TetraMesh.unit_cube(cube)
    return g, mesh, TriangularSkeleton(mesh, deg), r, LayeredField(values)


@pytest.mark.parametrize("name", list(TETRA_CASES))
def test_topology_is_the_reference(name):
    g, mesh, sk, r, _ = tetra_case(name)
    for key in ("points", "cells", "faces", "cell_faces", "face_cells", "signs"):
        assert np.array_equal(getattr(mesh, key), g[key]), key
    assert np.array_equal(mesh.areas, g["areas"])
    assert np.array_equal(sk.offsets, g["offsets"])
    assert np.array_equal(sk.cell_dof_array, g["cell_dofs"])


@pytest.mark.parametrize("name", list(TETRA_CASES))
def test_oracle_matches_reference(name):
    g, mesh, sk, r, field = tetra_case(name)
    sol = ot.solve_darcy_p1(mesh, sk, r, field, 1.0, keep_responses=True)
    m = sol["matrix"]
    assert np.array_equal(m.indptr, g["indptr"]) and np.array_equal(m.indices, g["indices"])
    assert np.max(np.abs(m.data - g["data"])) <= 1e-15 * np.max(np.abs(g["data"]))
    assert rel(sol["rhs"], g["rhs"]) <= 1e-14
    for key in ("trace", "coarse", "fields"):
        assert rel(sol[key], g[key]) <= 1e-12, key
    assert np.array_equal(sol["corrected"], g["corrected"])
    for c in g["keep_cells"]:
        p = sol["responses"][c].problem
        assert np.array_equal(p.matrix.toarray(), g[f"cell{c}_A"])
        assert np.array_equal(p.load, g[f"cell{c}_f"])
        assert np.max(np.abs(p.coupling - g[f"cell{c}_B"])) <= 1e-15 * np.max(np.abs(g[f"cell{c}_B"]))


@pytest.mark.parametrize("name", list(TETRA_CASES))
def test_closed_form_coupling_equals_quadrature(name):
    """The host's closed-form trace coupling equals the reference's quadrature (fixture)."""
    g, mesh, sk, r, _ = tetra_case(name)
    B = trace_coupling(mesh, sk, r)
    for c in g["keep_cells"]:
        ref = g[f"cell{c}_B"]
        assert np.max(np.abs(B[c] - ref)) <= 1e-15 * np.max(np.abs(ref))
    g0 = sk.geometric_constraint()
    for c in range(len(mesh.cells)):
        assert np.allclose(B[c].sum(axis=0), g0[c], rtol=1e-14, atol=1e-17)


def test_duffy_rule():
    bary, w = duffy_tetrahedron(5)
    assert bary.shape == (125, 4) and np.isclose(w.sum(), 1.0, rtol=1e-15)
    # exact for a degree-5 monomial: int_T x^2 y z^2 dV / |T| = 6 * 2! 1! 2! / 8! = 24 / 40320 * 6
    x, y, z = bary[:, 1], bary[:, 2], bary[:, 3]
    assert np.isclose(w @ (x ** 2 * y * z ** 2), 6 * 2 * 1 * 2 / 40320, rtol=1e-13)
