"""BatchedFactorization / condense_batched / GpuLocalSolver contracts (cf. the reference's
tests/test_gpu_batch.py) and parity with the oracle's condensation."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batched_lu_reuses_factors_and_preserves_matrix():
    from pymhm_b200.batched import BatchedFactorization

    matrices = np.array([[[2.0, 1.0], [1.0, 3.0]], [[0.0, 1.0], [1.0, 0.0]]])
    original = matrices.copy()
    exact = np.arange(1.0, 13.0).reshape(2, 2, 3)
    with BatchedFactorization(matrices) as prepared:
        matrices[:] = 0
        for factor in (1.0, -3.0):
            result = prepared.solve(original @ (factor * exact), host=bool(factor == 1))
            result = result if isinstance(result, np.ndarray) else result.cpu().numpy()
            np.testing.assert_allclose(result, factor * exact, atol=1e-12)
        np.testing.assert_allclose(prepared.solve(np.zeros((2, 2, 1)), host=True), 0)
    with pytest.raises(RuntimeError, match="closed"):
        prepared.solve(np.zeros((2, 2, 1)))
    with pytest.raises(RuntimeError, match="closed"):
        prepared.__enter__()


@pytest.mark.parametrize("matrix,message", [
    ([[[0.0, 0.0], [1.0, 2.0]]], "zero row"),
    ([[[0.0, 1.0], [0.0, 2.0]]], "zero column"),
    ([[[1.0, 1.0], [1.0, 1.0]]], "singular pivot|rank deficient"),
    ([[[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 9.0]]], "rank deficient|singular pivot"),
])
def test_singularity_messages(matrix, message):
    from pymhm_b200.batched import BatchedFactorization
    from pymhm_b200.errors import LinearSolveError

    with pytest.raises(LinearSolveError, match=message):
        BatchedFactorization(matrix)


def test_argument_validation():
    from pymhm_b200.batched import BatchedFactorization

    with pytest.raises(ValueError, match="matrices"):
        BatchedFactorization(np.ones((2, 3)))
    with pytest.raises(ValueError, match="matrices"):
        BatchedFactorization([[[np.nan]]])
    with BatchedFactorization([[[2.0]]]) as f:
        with pytest.raises(ValueError, match="rhs"):
            f.solve(np.ones((1, 2, 1)))
        with pytest.raises(ValueError, match="rhs"):
            f.solve([[[np.inf]]])


def test_random_batches_with_refinement():
    from pymhm_b200.batched import BatchedFactorization

    rng = np.random.default_rng(271)
    for n in (12, 91, 200):
        a = rng.normal(size=(16, n, n)) + n * np.eye(n)
        a[:, :, 0] *= 1e6  # badly scaled column: equilibration matters
        x = rng.normal(size=(16, n, 5))
        b = a @ x
        with BatchedFactorization(a) as f:
            got = f.solve(b, host=True)
        r = np.linalg.norm(a @ got - b, axis=1) / np.linalg.norm(b, axis=1)
        assert np.all(r <= 1e-12)


@pytest.mark.parametrize("n,nrhs", [(33, 4), (45, 1), (160, 1), (161, 4), (326, 4), (326, 17), (640, 16), (641, 3),
                                    (1000, 1)])
def test_factor_and_solve_paths(n, nrhs):
    """Every factor path (shared memory n <= 160, blocked 161..640, unblocked on the
    factors array above) and solve path (chunked with the right-hand sides in shared
    memory for nrhs <= 16, one warp per column otherwise) on matrices that need row
    pivoting."""
    from pymhm_b200.batched import BatchedFactorization

    rng = np.random.default_rng(n + nrhs)
    a = rng.normal(size=(4, n, n))
    a[:, :, 1] *= 1e5
    x = rng.normal(size=(4, n, nrhs))
    b = a @ x
    with BatchedFactorization(a) as f:
        got = f.solve(b, host=True)
        piv = f.pivots.cpu().numpy()
    assert np.any(piv != np.arange(n))  # pivoting happened
    r = np.linalg.norm(a @ got - b, axis=1) / np.linalg.norm(b, axis=1)
    assert np.all(r <= 1e-12)
    assert np.max(np.abs(got - x)) <= 1e-8 * np.max(np.abs(x))


def test_blocked_factor_reports_rank_deficiency():
    from pymhm_b200.batched import BatchedFactorization
    from pymhm_b200.errors import LinearSolveError

    rng = np.random.default_rng(5)
    a = rng.normal(size=(2, 300, 300))
    a[1, 150] = a[1, 20] * 3.0  # dependent rows in the second matrix only
    with pytest.raises(LinearSolveError, match="rank deficient|singular pivot"):
        BatchedFactorization(a)


def test_condense_batched_matches_oracle_condensation():
    """Augmented Q1 systems from the fixture, through the generic batched path."""
    from types import SimpleNamespace

    from pymhm_b200.batched import condense_batched
    from tests._cases import load

    g = load("darcy_4x4_r16_p2_lognormal")
    probs = []
    for c in g["keep_cells"]:
        aug, rhs = g[f"cell{c}_aug"], g[f"cell{c}_rhs"]
        probs.append(SimpleNamespace(condensation_system=lambda aug=aug, rhs=rhs: (aug, rhs),
                                     response_from_solution=lambda s: s))
    out = condense_batched(probs)
    for c, sol in zip(g["keep_cells"], out):
        n = len(g[f"cell{c}_source"])
        t = g[f"cell{c}_lifts"].shape[1]
        ref = g[f"cell{c}_lifts"]
        assert np.linalg.norm(sol[:n, 1:1 + t] - ref) <= 1e-10 * np.linalg.norm(ref)


def test_gpu_local_solver_protocol():
    from scipy import sparse

    from pymhm_b200.batched import GpuLocalSolver
    from tests._cases import load

    g = load("poisson_8x8_r4_p1")
    aug, rhs = sparse.csc_matrix(g["cell9_aug"]), g["cell9_rhs"]
    out = GpuLocalSolver()(aug.copy(), rhs.copy())
    assert out.shape == rhs.shape
    assert np.all(np.linalg.norm(aug @ out - rhs, axis=0) <= 1e-10 * np.linalg.norm(rhs, axis=0) + 1e-300)


def test_condense_batched_uneven_sizes_keep_order():
    """A mixed batch (three local sizes and right-hand-side widths, interleaved) is
    grouped by (augmented size, rhs width) as ``cuda.py:300-305`` does and returned in
    input order, each cell matching the reference's own lifts and source response."""
    from types import SimpleNamespace

    from pymhm_b200.batched import condense_batched
    from tests._cases import load

    cells = []
    for name in ("poisson_8x8_r4_p1", "darcy_4x4_r16_p2_lognormal", "affine_3x2_rect_r4x5_p1s2"):
        g = load(name)
        for c in g["keep_cells"]:
            cells.append((g[f"cell{c}_aug"], g[f"cell{c}_rhs"], g[f"cell{c}_source"], g[f"cell{c}_lifts"]))
    order = np.random.default_rng(5).permutation(len(cells))
    cells = [cells[i] for i in order]
    assert len({(c[0].shape[0], c[1].shape[1]) for c in cells}) >= 3
    probs = [SimpleNamespace(condensation_system=lambda aug=aug, rhs=rhs: (aug, rhs),
                             response_from_solution=lambda s: s) for aug, rhs, _, _ in cells]
    out = condense_batched(probs)
    assert len(out) == len(cells)
    for (aug, rhs, source, lifts), sol in zip(cells, out):
        n, t = len(source), lifts.shape[1]
        assert sol.shape == rhs.shape
        assert np.linalg.norm(sol[:n, 1:1 + t] - lifts) <= 1e-10 * np.linalg.norm(lifts)
        # some cells carry a numerically zero source response: bound it absolutely too
        assert np.linalg.norm(sol[:n, 0] - source) <= 1e-10 * np.linalg.norm(source) + 1e-14
