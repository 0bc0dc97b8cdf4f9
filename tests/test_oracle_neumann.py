"""Neumann faces on whole bottom/top sides: the oracle and the host-side boundary data
against fixtures written by the reference (tests/golden/make_neumann_golden.py)."""

import numpy as np
import pytest

from oracle import q1_mhm as o
from tests._cases import load, rel
from pymhm_b200.workloads import sine_source

def _bottom_flux(x):
    return 0.5 + x[:, 0]


def _left_flux(x):
    return 0.3 - 0.2 * x[:, 1]


def _side(mesh, axis, value):
    return [int(f) for f in mesh.boundary_faces if np.all(mesh.points[mesh.faces[f]][:, axis] == value)]


def _partial_sides(mesh):
    out = {f: -1.0 for f in _side(mesh, 0, 0.0)[1:3]}
    out.update({f: 0.0 for f in _side(mesh, 1, 0.0)[:2] + _side(mesh, 1, 1.0)})
    return out


def _kappa(g):
    return o.PixelField(g["kappa"], (1 / 32, 1 / 32))


NEUMANN_CASES = {
    # name -> (face degree, refinement, permeability(g), source, dirichlet,
    #          Neumann sides: (axis, coordinate) -> outward flux)
    "darcy_4x4_r8_p2_noflow_tb": (2, (8, 8), _kappa, 1.0, lambda x: 1.0 - x[:, 0], {(1, 0.0): 0.0, (1, 1.0): 0.0}),
    "poisson_4x4_r4_p1_flux_bottom": (1, (4, 4), lambda g: 1.0, sine_source, 0.0, {(1, 0.0): _bottom_flux}),
    "darcy_4x4_r8_p2_noflow_lr": (2, (8, 8), _kappa, 1.0, lambda x: 1.0 - x[:, 1], {(0, 0.0): 0.0, (0, 1.0): 0.0}),
    "poisson_4x4_r4_p1_flux_left_bottom": (1, (4, 4), lambda g: 1.0, sine_source, 0.0,
                                           {(0, 0.0): _left_flux, (1, 0.0): _bottom_flux}),
    # part of two sides (the middle of the left side, the first half of the bottom) and the
    # whole top: the coarse operator's Woodbury correction
    "darcy_4x4_r8_p2_partial_sides": (2, (8, 8), _kappa, 0.0, 0.0, lambda mesh: _partial_sides(mesh)),
    # every side Neumann (outward flux 0.25, balancing the unit source): the mean-pressure gauge
    "darcy_4x4_r8_p1_pure_neumann": (1, (8, 8), _kappa, 1.0, 0.0,
                                     {(1, 0.0): 0.25, (1, 1.0): 0.25, (0, 0.0): 0.25, (0, 1.0): 0.25}),
}

MEAN_PRESSURE = {"darcy_4x4_r8_p1_pure_neumann": 0.3}

SIDE_BITS = {"darcy_4x4_r8_p2_noflow_tb": 3, "poisson_4x4_r4_p1_flux_bottom": 1, "darcy_4x4_r8_p2_noflow_lr": 12,
             "poisson_4x4_r4_p1_flux_left_bottom": 5, "darcy_4x4_r8_p1_pure_neumann": 15,
             "darcy_4x4_r8_p2_partial_sides": 2}


def neumann_map(g, sides, mesh=None):
    """The case's Neumann data per face; the faces are the fixture's."""
    if mesh is None:
        mesh = o.cartesian_mesh(4)
    if callable(sides):
        out = sides(mesh)
        assert sorted(out) == [int(f) for f in g["neumann_faces"]]
        return out
    out = {}
    for f in mesh.boundary_faces:
        pts = mesh.points[mesh.faces[f]]
        for (axis, value), data in sides.items():
            if np.all(pts[:, axis] == value):
                out[int(f)] = data
    assert sorted(out) == [int(f) for f in g["neumann_faces"]]
    return out


@pytest.mark.parametrize("name", list(NEUMANN_CASES))
def test_oracle_matches_reference(name):
    g = load(name)
    deg, ref, perm, src, dr, val = NEUMANN_CASES[name]
    mesh = o.cartesian_mesh(4)
    sk = o.Skeleton(mesh, (o.FaceSpace.uniform(deg),) * len(mesh.faces))
    _, fixed = o.boundary_data(sk, dr, neumann_map(g, val))
    assert np.array_equal(np.array(sorted(fixed)), g["fixed_dofs"])
    assert np.allclose([fixed[k] for k in sorted(fixed)], g["fixed_values"], rtol=0, atol=1e-15)
    sol = o.solve_darcy_q1(mesh, sk, ref, perm(g), src, dr, neumann=neumann_map(g, val),
                           mean_pressure=MEAN_PRESSURE.get(name, 0.0))
    for key, val_ in (("trace", sol.trace), ("coarse", sol.coarse), ("fields", sol.fields), ("flux", sol.flux)):
        assert rel(val_, g[key]) <= 1e-12, key
    assert np.array_equal(sol.trace[g["fixed_dofs"]], g["trace"][g["fixed_dofs"]])


@pytest.mark.parametrize("name", list(NEUMANN_CASES))
def test_host_boundary_data_matches_reference(name):
    from pymhm_b200.topology import (CartesianMacroMesh, FaceSpace, SkeletonSpace, boundary_data, neumann_fixed,
                                     neumann_layout)

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
    assert neumann_layout(mesh, neu)[0] == SIDE_BITS[name]


def test_neumann_side_rules():
    from pymhm_b200.topology import CartesianMacroMesh, neumann_layout

    mesh = CartesianMacroMesh(4)
    pts = mesh.points[mesh.faces[mesh.boundary_faces]]
    bottom = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 1] == 0.0)]
    top = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 1] == 1.0)]
    left = [int(f) for f, p in zip(mesh.boundary_faces, pts) if np.all(p[:, 0] == 0.0)]
    assert neumann_layout(mesh, None) == (0, [])
    assert neumann_layout(mesh, {f: 0.0 for f in top}) == (2, [])
    assert neumann_layout(mesh, {f: 0.0 for f in left}) == (4, [])
    assert neumann_layout(mesh, {f: 0.0 for f in bottom[:2]}) == (0, sorted(bottom[:2]))
    assert neumann_layout(mesh, {f: 0.0 for f in left + bottom[1:]}) == (4, sorted(bottom[1:]))
    assert neumann_layout(mesh, {int(f): 0.0 for f in mesh.boundary_faces}) == (15, [])


@pytest.mark.parametrize("bits", [4, 8, 12])
def test_coarse_x_basis_diagonalises_the_neumann_factor(bits):
    """The host eigenbasis of the coarse x factor; with both ends Neumann its first
    mode is exactly the constant."""
    from pymhm_b200.topology import coarse_x_basis

    nx = 7
    q, lam = coarse_x_basis(nx, bits)
    t = 2.0 * np.eye(nx) - np.eye(nx, k=1) - np.eye(nx, k=-1)
    t[0, 0] -= 1.0 if bits & 4 else 0.0
    t[-1, -1] -= 1.0 if bits & 8 else 0.0
    assert np.allclose(q.T @ q, np.eye(nx), atol=1e-14)
    assert np.allclose(q @ np.diag(lam) @ q.T, t, atol=1e-13)
    # a zero mode only when both x ends are Neumann (the y ends then carry the solve)
    assert (lam.min() <= 1e-14) == (bits == 12)


def test_mode0_pseudo_inverse():
    from pymhm_b200.topology import coarse_mode0_pinv

    ny, ay = 6, 0.7
    t = ay * (2.0 * np.eye(ny) - np.eye(ny, k=1) - np.eye(ny, k=-1))
    t[0, 0] -= ay
    t[-1, -1] -= ay
    p = coarse_mode0_pinv(ny, ay)
    assert np.allclose(p, np.linalg.pinv(t), atol=1e-13)
    assert np.allclose(p @ np.ones(ny), 0.0, atol=1e-13)


def test_partial_side_correction_inverts_the_masked_coarse_operator():
    """The Woodbury factor reproduces the inverse of G0^T G0 restricted to the free
    DOFs (the coarse operator the skeleton solve projects with) for Neumann faces on
    parts of sides."""
    from pymhm_b200 import topology as tp

    mesh = tp.CartesianMacroMesh(5, 4)
    sk = tp.SkeletonSpace(mesh, (tp.FaceSpace.uniform(2),) * len(mesh.faces))
    sh, sv = sk.uniform_by_orientation()
    g0 = tp.geometric_constraint(mesh, sh, sv)
    ax, ay = tp.coarse_coefficients(mesh, sh, sv)
    cells = len(mesh.cells)
    G = np.zeros((sk.size, cells))
    for c in range(cells):
        np.add.at(G[:, c], sk.cell_dof_array[c], g0[c])
    neu = {f: 0.0 for f in _side(mesh, 1, 0.0)[:2] + _side(mesh, 0, 0.0)[1:3] + _side(mesh, 1, 1.0)}
    bits, partial = tp.neumann_layout(mesh, neu)
    assert bits == 2 and len(partial) == 4
    fixed = np.concatenate([sk.dofs(f) for f in neu])
    G[fixed] = 0.0
    wb_cells, factor = tp.coarse_partial_correction(mesh, bits, partial, ax, ay)

    def tri(n, lo, hi):
        t = 2.0 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
        t[0, 0] -= 1.0 if lo else 0.0
        t[-1, -1] -= 1.0 if hi else 0.0
        return t

    a_sep = ay * np.kron(tri(4, bits & 1, bits & 2), np.eye(5)) + ax * np.kron(np.eye(4), tri(5, bits & 4, bits & 8))
    r = np.random.default_rng(3).normal(size=cells)
    y = np.linalg.solve(a_sep, r)
    exact = np.linalg.solve(G.T @ G, r)
    assert np.max(np.abs(y + factor @ y[wb_cells] - exact)) <= 1e-13 * np.max(np.abs(exact))
