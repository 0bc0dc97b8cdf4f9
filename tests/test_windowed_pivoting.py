"""The large-order LU's pivoting rule, restated in NumPy and checked on the CPU: for
bordered semi-definite systems [[A, c], [c^T, 0]] (A with the constants as its
kernel) padded with identity rows, a blocked LU whose row search is restricted to each
32-column panel's diagonal window and the one row below it factors exactly, including
when the last node row closes a panel and the bordering row opens the next."""

import numpy as np
import pytest
import scipy.linalg as sl

KP = 32


def windowed_lu(K):
    """Row/column max-equilibration, then the blocked right-looking LU of the large-order
    kernel: per panel, partial pivoting over the (w + 1) x w window, the window's row
    exchanges applied to the other columns, U12 = L11^-1 A12, L21 = A21 U11^-1 and the
    trailing update.  Returns the packed factors, the LAPACK pivot sequence and the
    scales."""
    n = K.shape[0]
    rs = 1.0 / np.abs(K).max(axis=1)
    F = K * rs[:, None]
    cs = 1.0 / np.abs(F).max(axis=0)
    F = F * cs[None, :]
    piv = np.arange(n)
    for kb in range(0, n, KP):
        w = min(KP, n - kb)
        h = min(w + 1, n - kb)
        win = F[kb:kb + h, kb:kb + w].copy()
        perm = []
        for c in range(w):
            p = c + int(np.argmax(np.abs(win[c:h, c])))
            perm.append(p)
            win[[c, p], :] = win[[p, c], :]
            assert win[c, c] != 0.0
            win[c + 1:h, c + 1:w] -= np.outer(win[c + 1:h, c] / win[c, c], win[c, c + 1:w])
            win[c + 1:h, c] /= win[c, c]
        F[kb:kb + h, kb:kb + w] = win
        src = list(range(h))
        for c, p in enumerate(perm):
            piv[kb + c] = kb + p
            src[c], src[p] = src[p], src[c]
        other = np.r_[0:kb, kb + w:n]
        rows = F[kb:kb + h][:, other].copy()
        F[np.ix_(kb + np.arange(h), other)] = rows[src]
        L11 = np.tril(win[:w, :w], -1) + np.eye(w)
        U11 = np.triu(win[:w, :w])
        F[kb:kb + w, kb + w:] = sl.solve_triangular(L11, F[kb:kb + w, kb + w:], lower=True, unit_diagonal=True)
        F[kb + h:, kb:kb + w] = sl.solve_triangular(U11, F[kb + h:, kb:kb + w].T, trans=1).T
        F[kb + w:, kb + w:] -= F[kb + w:, kb:kb + w] @ F[kb:kb + w, kb + w:]
    return F, piv, rs, cs


def lu_solve(F, piv, rs, cs, b):
    x = b * rs[:, None]
    for k, p in enumerate(piv):
        if p != k:
            x[[k, p]] = x[[p, k]]
    x = sl.solve_triangular(F, x, lower=True, unit_diagonal=True)
    x = sl.solve_triangular(F, x)
    return x * cs[:, None]


def bordered(rng, m, nb, contrast=1.0):
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


@pytest.mark.parametrize("m,nb,contrast", [(100, 128, 1.0), (127, 128, 30.0), (128, 160, 1.0), (159, 160, 1e3),
                                           (95, 96, 30.0), (250, 256, 1.0)])
def test_windowed_pivoting_factors_bordered_systems(m, nb, contrast):
    """Orders with the bordering row inside a panel, on a panel's first row (m = 128:
    the last node row closes the panel before it) and on the padding boundary; the
    solution of the equilibrated factors has a LAPACK-level residual."""
    rng = np.random.default_rng(m + nb)
    K = bordered(rng, m, nb, contrast)
    F, piv, rs, cs = windowed_lu(K)
    b = rng.standard_normal((nb, 4))
    b[m + 1:] = 0.0
    x = lu_solve(F, piv, rs, cs, b)
    ref = np.linalg.solve(K, b)
    assert np.linalg.norm(K @ x - b) <= 1e-12 * np.linalg.norm(b)
    assert np.linalg.norm(x - ref) <= 1e-9 * np.linalg.norm(ref)
    # the node rows' leading pivots need no exchange below the window: every exchange
    # stays inside its panel's window
    for k, p in enumerate(piv):
        assert k <= p <= (k // KP) * KP + KP


def test_last_node_panel_takes_the_bordering_row():
    """When the last node row closes a panel, that panel's node rows alone are singular
    (the constants are in A's kernel): the window's extra row, the bordering row, is
    exchanged into the panel, and without it the panel factorization breaks down."""
    rng = np.random.default_rng(7)
    m, nb = 128, 160
    K = bordered(rng, m, nb)
    _, piv, _, _ = windowed_lu(K)
    assert m in piv[m - KP:m]
    # the same panel restricted to its own rows: a pivot at rounding level
    A = K[:m, :m] * (1.0 / np.abs(K[:m, :m]).max())
    lu = sl.lu_factor(A)
    assert np.abs(np.diag(lu[0])).min() <= 1e-10
