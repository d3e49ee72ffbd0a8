"""Cumulant analysis of the simulator's outputs.

Restates, in numpy, the formulas the reference applies to its outputs in
MATLAB (analysis/readRMS.m, analysis/readRMS_pgse.m): normalisation of the
moment tensors by sig0 with the tensor multiplicities, directional D(t) and
K(t), and the PGSE b-value.
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
