"""SkeletonFactorization (LinearFactorization contract) on the oracle's assembled system."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_skeleton_factorization_solves_reference_matrix():
    from scipy import sparse

    from pymhm_b200.skeleton import SkeletonFactorization
    from pymhm_b200.topology import CartesianMacroMesh, FaceSpace, SkeletonSpace
    from tests._cases import load, rel

    g = load("darcy_4x4_r16_p2_lognormal")
    mesh = CartesianMacroMesh(4)
    sk = SkeletonSpace(mesh, (FaceSpace.uniform(2),) * len(mesh.faces))
    N = sk.size + len(mesh.cells)
    A = sparse.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=(N, N))
    with SkeletonFactorization(A, mesh, sk) as f:
        assert f.matches(A)
        B = A.copy()
        B.data[0] += 1.0
        assert not f.matches(B)
        x = f.solve(g["rhs"])
        assert rel(x[: sk.size], g["trace"]) <= 1e-10
        assert rel(x[sk.size:], g["coarse"]) <= 1e-10
        two = f.solve(np.column_stack((g["rhs"], 2 * g["rhs"])))
        assert rel(two[:, 1], 2 * x) <= 1e-12
    with pytest.raises(RuntimeError, match="closed"):
        f.solve(g["rhs"])
