"""Cumulant analysis of the simulator's outputs.

Restates, in numpy, the formulas the reference applies to its outputs in
MATLAB (analysis/readRMS.m, analysis/readRMS_pgse.m): normalisation of the
moment tensors by sig0 with the tensor multiplicities, directional D(t) and
K(t), the PGSE b-value, and the shell-wise and linear least-squares DKI fits
of the signal.
"""
from __future__ import annotations

import numpy as np

# readRMS.m:13-18
D_CNT = np.array([1, 2, 2, 1, 2, 1], dtype=np.float64)
W_CNT = np.array([1, 4, 4, 6, 12, 6, 4, 12, 12, 4, 1, 4, 6, 4, 1], dtype=np.float64)
D_IND = np.array([[1, 1], [1, 2], [1, 3], [2, 2], [2, 3], [3, 3]]) - 1
W_IND = np.array([[1, 1, 1, 1], [1, 1, 1, 2], [1, 1, 1, 3], [1, 1, 2, 2], [1, 1, 2, 3],
                  [1, 1, 3, 3], [1, 2, 2, 2], [1, 2, 2, 3], [1, 2, 3, 3], [1, 3, 3, 3],
                  [2, 2, 2, 2], [2, 2, 2, 3], [2, 2, 3, 3], [2, 3, 3, 3], [3, 3, 3, 3]]) - 1


def normalized_moments(sig0, dx2, dx4):
    """dx2t = dx2 .* D_cnt ./ sig0, dx4t = dx4 .* W_cnt ./ sig0 (readRMS.m:44-45)."""
    s = np.asarray(sig0, dtype=np.float64).reshape(-1, 1)
    return np.asarray(dx2) * D_CNT / s, np.asarray(dx4) * W_CNT / s


def ndir2(n):
    """readRMS.m:123-125: products n_i n_j over D_ind."""
    n = np.atleast_2d(np.asarray(n, dtype=np.float64))
    return np.prod(n[:, D_IND], axis=2)


def ndir4(n):
    """readRMS.m:119-121: products n_i n_j n_k n_l over W_ind."""
    n = np.atleast_2d(np.asarray(n, dtype=np.float64))
    return np.prod(n[:, W_IND], axis=2)


def akc_mom(dx2t, dx4t, td, n):
    """Directional kurtosis and diffusivity from the moments (readRMS.m:96-103):
    D = <x^2>/(2t), K = <x^4>/<x^2>^2 - 3.  Returns (K, D), [T, ndir]."""
    x2 = np.asarray(dx2t) @ ndir2(n).T
    x4 = np.asarray(dx4t) @ ndir4(n).T
    D = x2 / 2.0 / np.asarray(td, dtype=np.float64).reshape(-1, 1)
    K = x4 / x2 ** 2 - 3.0
    return K, D


def axis_dk(sig0, dx2, dx4, td):
    """D(t), K(t) along x, y, z: [T, 3] each."""
    dx2t, dx4t = normalized_moments(sig0, dx2, dx4)
    K, D = akc_mom(dx2t, dx4t, td, np.eye(3))
    return D, K


def pgse_bval(grad):
    """b = |g|^2 delta^2 (Delta - delta/3) (readRMS_pgse.m:53); grad rows are
    (Delta, delta, |g|, gx, gy, gz)."""
    g = np.asarray(grad, dtype=np.float64).reshape(-1, 6)
    return g[:, 2] ** 2 * g[:, 1] ** 2 * (g[:, 0] - g[:, 1] / 3.0)


def pgse_gradient_for_b(b, Delta, delta):
    """|g| giving b-value b for a rectangular PGSE pair."""
    return np.sqrt(np.asarray(b, dtype=np.float64) / (delta ** 2 * (Delta - delta / 3.0)))


# ---- DKI fits of the signal (readRMS.m:47-48, 51-94, 105-117) ----
# MATLAB's eps, added inside the logarithm as the readers do
EPS = np.finfo(np.float64).eps


def narrow_signal(sig0, sigre):
    """sig = |sigRe| ./ sig0, [T, nbvec] (readRMS.m:47-48)."""
    return np.abs(np.asarray(sigre, dtype=np.float64)) / np.asarray(sig0, dtype=np.float64).reshape(-1, 1)


def mldivide(a, y):
    """MATLAB's a \\ y for a rectangular a: QR with column pivoting (LAPACK
    dgeqp3 through scipy), rank from |R_kk| > max(m, n) eps |R_11|, and the
    basic solution (zeros on the columns past the rank)."""
    from scipy.linalg import qr, solve_triangular
    a = np.asarray(a, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    m, n = a.shape
    q, r, piv = qr(a, mode="economic", pivoting=True)
    d = np.abs(np.diag(r))
    tol = max(m, n) * EPS * (d[0] if d.size else 0.0)
    k = 0
    while k < d.size and d[k] > tol:
        k += 1
    x = np.zeros((n,) + y.shape[1:])
    if k:
        x[piv[:k]] = solve_triangular(r[:k, :k], (q.T @ y)[:k])
    return x


def dki_shell(sig, bvec, bval, td, intercept=False):
    """Shell-wise fit (readRMS.m:51-78; intercept=True: readRMS_pgse.m:60-89):
    per unique direction, log(S + eps) ~ [1] -b, b^2/6 .. b^nb/6; then the
    directional <x^2>, <x^4> fitted by the 2nd/4th order tensor elements.
    Returns dt [T, 21]."""
    sig = np.atleast_2d(np.asarray(sig, dtype=np.float64))
    bvec = np.asarray(bvec, dtype=np.float64).reshape(-1, 3)
    bval = np.asarray(bval, dtype=np.float64).reshape(-1)
    td = np.asarray(td, dtype=np.float64).reshape(-1)
    bvecu, inv = np.unique(bvec, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    nbval = np.unique(bval).size
    n2, n4 = ndir2(bvecu), ndir4(bvecu)
    off = 1 if intercept else 0
    dt = np.zeros((sig.shape[0], 21))
    for i in range(sig.shape[0]):
        Di = np.zeros(len(bvecu))
        Ki = np.zeros(len(bvecu))
        for j in range(len(bvecu)):
            Ij = inv == j
            b = bval[Ij]
            cols = ([np.ones_like(b)] if intercept else []) + [-b] + [b ** p / 6.0 for p in range(2, nbval + 1)]
            X = mldivide(np.stack(cols, axis=1), np.log(sig[i, Ij] + EPS))
            Di[j] = X[off]
            Ki[j] = X[off + 1] / X[off] ** 2
        dx2g = Di * 2.0 * td[i]
        dx4g = (Ki + 3.0) * dx2g ** 2
        dt[i, :6] = mldivide(n2, dx2g)
        dt[i, 6:] = mldivide(n4, dx4g)
    return dt


def dki_lls(sig, bvec, bval):
    """Linear least-squares DKI fit (readRMS.m:80-91): log(S + eps) against
    -b D_cnt g_i g_j and b^2/6 W_cnt g_i g_j g_k g_l.  Returns dt [T, 21]."""
    sig = np.atleast_2d(np.asarray(sig, dtype=np.float64))
    g = np.asarray(bvec, dtype=np.float64).reshape(-1, 3)
    b = np.asarray(bval, dtype=np.float64).reshape(-1, 1)
    norm = np.sqrt((g ** 2).sum(axis=1, keepdims=True))
    norm[norm == 0] = 1.0
    g = g / norm
    a = np.concatenate([-(b * ndir2(g)) * D_CNT, (b ** 2 / 6.0 * ndir4(g)) * W_CNT], axis=1)
    return mldivide(a, np.log(sig + EPS).T).T


def akc_shell(dt, n, td):
    """(K, D) along n from a shell fit (readRMS.m:105-112)."""
    dt = np.atleast_2d(np.asarray(dt, dtype=np.float64))
    x2 = dt[:, :6] @ ndir2(n).T
    x4 = dt[:, 6:] @ ndir4(n).T
    D = x2 / 2.0 / np.asarray(td, dtype=np.float64).reshape(-1, 1)
    return x4 / x2 ** 2 - 3.0, D


def akc_lls(dt, n):
    """(K, D) along n from an LLS fit, read off the DKI signal model
    ln S = -b D(n) + b^2 D(n)^2 K(n) / 6 (Jensen et al., Magn. Reson. Med.
    53:1432, 2005); readRMS.m:114-117 calls the external DKI.akc for this."""
    dt = np.atleast_2d(np.asarray(dt, dtype=np.float64))
    n = np.atleast_2d(np.asarray(n, dtype=np.float64))
    n = n / np.linalg.norm(n, axis=1, keepdims=True)
    D = dt[:, :6] @ (ndir2(n) * D_CNT).T
    W = dt[:, 6:] @ (ndir4(n) * W_CNT).T
    return W / D ** 2, D
