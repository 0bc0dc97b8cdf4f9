"""Large local systems (augmented orders 641 to 4096): the windowed-pivot LU in HBM and
its checked solve through the C ABI, and polygon batches whose local P2 spaces reach
config 3's upper sizes, against dense LAPACK solves and against the oracle."""

import ctypes as C

import numpy as np
import pytest

from tests._cases import rel

pytestmark = pytest.mark.gpu

RAGGED = [("mat_off", "<i8"), ("vec_off", "<i8"), ("rhs_off", "<i8"), ("n", "<i4"), ("nrhs", "<i4"),
          ("slot", "<i4"), ("reserved", "<i4")]


def bordered_system(rng, m, nb, contrast=1.0):
    """A connected weighted-graph Laplacian of order m (the constants its kernel), bordered
    by a positive mean constraint scaled as the reference scales it and padded with an
    identity block to order nb: the structure of a Neumann local problem's augmented
    matrix."""
    W = np.abs(rng.standard_normal((m, m))) * (rng.random((m, m)) < 8.0 / m)
    W = np.triu(W, 1)
    W[np.arange(m - 1), np.arange(1, m)] += 1.0
    W *= np.where(rng.random((m, m)) < 0.2, contrast, 1.0)
    W = W + W.T
    A = np.diag(W.sum(1)) - W
    c = rng.random(m) + 0.5
    c /= c.sum()
    c *= min(1.0, np.abs(A).max() / np.abs(c).max())
    K = np.eye(nb)
    K[:m, :m] = A
    K[:m, m] = c
    K[m, :m] = c
    K[m, m] = 0.0
    return K


def run_large(mats, rhss, max_n=None):
    """Factor and solve ragged systems through mhm_batched_factor_large /
    mhm_batched_solve_large (largest first); returns solutions and status words."""
    import torch

    from pymhm_b200 import _lib

    lib = _lib.lib()
    P = _lib.ptr
    dev = torch.device("cuda")
    order = sorted(range(len(mats)), key=lambda k: -mats[k].shape[0])
    moff, voff, roff = np.cumsum([0] + [m.shape[0] ** 2 for m in mats]), np.cumsum([0] + [m.shape[0] for m in mats]), \
        np.cumsum([0] + [r.size for r in rhss])
    desc = np.array([(moff[k], voff[k], roff[k], mats[k].shape[0], rhss[k].shape[1], k, 0) for k in order],
                    dtype=RAGGED)
    d_desc = torch.as_tensor(desc.view(np.uint8).copy()).to(dev)
    A = torch.as_tensor(np.concatenate([m.ravel() for m in mats])).to(dev)
    B = torch.as_tensor(np.concatenate([r.ravel() for r in rhss])).to(dev)
    F = torch.empty_like(A)
    X = torch.zeros_like(B)
    nv = int(voff[-1])
    piv = torch.empty(nv, dtype=torch.int32, device=dev)
    rs, cs = torch.empty(nv, dtype=torch.float64, device=dev), torch.empty(nv, dtype=torch.float64, device=dev)
    work = torch.empty(66 * nv, dtype=torch.float64, device=dev)
    status = torch.full((len(mats),), -1, dtype=torch.int32, device=dev)
    mx = max(m.shape[0] for m in mats) if max_n is None else max_n
    mw = max(r.shape[1] for r in rhss)
    sh = _lib.stream_handle(None)
    _lib.check(lib.mhm_batched_factor_large(len(mats), P(d_desc), mx, P(A), P(F), P(piv), P(rs), P(cs), P(status),
                                            sh), "factor")
    _lib.check(lib.mhm_batched_solve_large(len(mats), P(d_desc), mx, mw, P(A), P(F), P(piv), P(rs), P(cs), P(B),
                                           P(X), P(work), 1e-10, 0.0, 2, P(status), sh), "solve")
    torch.cuda.synchronize()
    x = X.cpu().numpy()
    return [x[roff[k]: roff[k + 1]].reshape(rhss[k].shape) for k in range(len(mats))], status.cpu().numpy()


def test_large_orders_match_dense_solves():
    """Orders 672 .. 2592 with identity padding, the bordering row on both sides of a
    32-column panel boundary (m = 704, 736: the last node row closes a panel and the
    bordering row opens the next), 1 to 30 right-hand sides: every column meets the
    reference's 1e-10 residual acceptance and matches LAPACK to 1e-10."""
    rng = np.random.default_rng(4101)
    shapes = [(700, 704, 5), (704, 736, 17), (736, 768, 30), (1000, 1024, 1), (1500, 1536, 22), (2590, 2592, 12),
              (650, 672, 3)]
    mats = [bordered_system(rng, m, nb, contrast=[1.0, 30.0][i % 2]) for i, (m, nb, _) in enumerate(shapes)]
    rhss = []
    for (m, nb, w) in shapes:
        b = rng.standard_normal((nb, w))
        b[m + 1:] = 0.0
        rhss.append(b)
    xs, status = run_large(mats, rhss)
    assert np.all(status == 0), status
    for K, b, x in zip(mats, rhss, xs):
        ref = np.linalg.solve(K, b)
        assert rel(x, ref) <= 1e-10
        r = np.linalg.norm(K @ x - b, axis=0) / np.linalg.norm(b, axis=0)
        assert np.all(r <= 1e-10)


def test_large_orders_report_contract_failures():
    """A zero row and an order above the launch maximum give the small-tier codes (zero
    row, size) without touching the other systems of the launch."""
    from pymhm_b200 import _lib

    rng = np.random.default_rng(4102)
    good = bordered_system(rng, 800, 832)
    zero = good.copy()
    zero[5, :] = 0.0
    big = bordered_system(rng, 900, 928)
    rhss = [rng.standard_normal((832, 4)), rng.standard_normal((832, 4)), rng.standard_normal((928, 4))]
    xs, status = run_large([good, zero, big], rhss, max_n=900)
    assert status[0] == _lib.CELL_OK
    assert status[1] == _lib.CELL_ZERO_ROW
    assert status[2] == _lib.CELL_SIZE
    assert rel(xs[0], np.linalg.solve(good, rhss[0])) <= 1e-10


def test_large_orders_odd_and_contract_codes():
    """Odd orders (701, 999: rows not 16-byte aligned, so the trailing update loads C
    and L21 directly instead of by bulk copies) match LAPACK; a bordering row orthogonal
    to the constants makes the system singular (rank test or zero pivot), and a
    non-finite entry gives the non-finite code."""
    from pymhm_b200 import _lib

    rng = np.random.default_rng(4103)
    odd = [bordered_system(rng, 700, 701), bordered_system(rng, 990, 999, contrast=30.0)]
    sing = bordered_system(rng, 800, 801)
    c = rng.standard_normal(800)
    c -= c.mean()  # orthogonal to the constants: [[A, c], [c^T, 0]] is singular
    sing[:800, 800] = c
    sing[800, :800] = c
    nanm = bordered_system(rng, 700, 704)
    nanm[3, 5] = np.nan
    mats = odd + [sing, nanm]
    rhss = [rng.standard_normal((m.shape[0], 6)) for m in mats]
    xs, status = run_large(mats, rhss)
    assert status[0] == _lib.CELL_OK and status[1] == _lib.CELL_OK
    for K, b, x in zip(odd, rhss, xs):
        assert rel(x, np.linalg.solve(K, b)) <= 1e-10
    assert status[2] in (_lib.CELL_RANK_DEFICIENT, _lib.CELL_SINGULAR_PIVOT, _lib.CELL_RESIDUAL)
    assert status[3] == _lib.CELL_NONFINITE


def large_polygon_case():
    from pymhm_b200.polygon import EdgeSkeleton, voronoi_mesh
    from pymhm_b200.workloads import DiscInclusions, disc_inclusions

    mesh = voronoi_mesh(12, 41)
    sk = EdgeSkeleton(mesh)
    rs = np.array([2, 4, 8, 10, 12, 14, 3, 9, 11, 6, 20, 7])
    field = DiscInclusions(*disc_inclusions(40, rmin=0.01, rmax=0.03, seed=42), inside=30.0)
    return mesh, sk, rs, field


def test_polygon_large_cells_match_oracle():
    """Twelve Voronoi cells whose P2 spaces span 51 to 3281 unknowns (both tiers in one
    solve), 40 discs of permeability 30: trace, coarse unknowns and fields against the
    oracle's solve at 1e-10, with the large tier in one chunk and, with the smallest
    workspace (one largest matrix per half), in two."""
    from oracle import polygon_mhm as op
    from pymhm_b200.polygon_darcy import PolygonP2Plan

    mesh, sk, rs, field = large_polygon_case()
    ref = op.solve_darcy_p2(mesh, sk, [mesh.submesh(c, int(rs[c])) for c in range(len(rs))], field, 1.0)
    dense = np.linalg.solve(ref["matrix"].toarray(), ref["rhs"])
    spread = rel(dense[: len(ref["trace"])], ref["trace"])
    sols = []
    for ws in (None, 1):
        plan = PolygonP2Plan(mesh, sk, rs, workspace_bytes=ws)
        assert plan.n_cells.max() + 1 > 3000 and plan.n_cells.min() + 1 < 640
        assert len(plan.chunks) == (1 if ws is None else 2)
        sol = plan.solve(field, 1.0)
        assert rel(sol.trace, ref["trace"]) <= max(1e-10, 2.0 * spread)
        assert rel(sol.coarse, ref["coarse"]) <= 1e-10
        assert rel(np.concatenate(sol.fields), np.concatenate(ref["fields"])) <= 1e-10
        assert np.array_equal(sol.corrected, ref["corrected"])
        sols.append(sol)
    assert rel(sols[0].trace, sols[1].trace) <= 1e-13


def test_polygon_large_cells_without_ragged_launches():
    """The per-bin path of the small tier combined with the large tier gives the ragged
    path's solution."""
    from pymhm_b200.polygon_darcy import PolygonP2Plan

    mesh, sk, rs, field = large_polygon_case()
    a = PolygonP2Plan(mesh, sk, rs, ragged=True).solve(field, 1.0)
    b = PolygonP2Plan(mesh, sk, rs, ragged=False).solve(field, 1.0)
    assert rel(a.trace, b.trace) <= 1e-11
    assert rel(np.concatenate(a.fields), np.concatenate(b.fields)) <= 1e-11
