"""General gradient waveforms: piecewise-constant vector waveforms on time bins.

The engine's waveform mode (RMS_MODE_WAVEFORM in include/rms.h) generalises the
reference's rectangular PGSE pair (hpc_code/lib/main_PGSE.cu:336-346): a
waveform j is a [nbins, 3] array w_j (phase per um per ms: gamma g for the
reference's units) held constant over each bin of ``tn / nbins`` steps, and

    phase_j = dt * sum_b w_j[b] . X_b,   X_b = sum over bin b's steps of the
                                          displacement (um) after each step.

The reference's PGSE phase is the special case of one step per bin and
w_j[i] = +|g| g_hat in the first lobe, -|g| g_hat in the second.
"""
from __future__ import annotations

import numpy as np


def pgse_waveform(grad, dt: float, tn: int) -> np.ndarray:
    """The reference's PGSE gradients (rows Delta, delta, |g|, gx, gy, gz, as in
    gradient_time.txt) as waveforms with one step per bin: [ngrad, tn, 3].

    Lobe rule of main_PGSE.cu:340-346 with t_i = (i + 1) dt: + while t_i < delta,
    - while Delta <= t_i < Delta + delta."""
    g = np.asarray(grad, dtype=np.float64).reshape(-1, 6)
    t = (np.arange(tn) + 1) * dt
    out = np.zeros((g.shape[0], tn, 3))
    for j, (Delta, delta, mag, gx, gy, gz) in enumerate(g):
        sign = np.where(t < delta, 1.0, np.where((t >= Delta) & (t < Delta + delta), -1.0, 0.0))
        out[j] = sign[:, None] * mag * np.array([gx, gy, gz])[None, :]
    return out


def bvalue(wave, bin_time: float) -> np.ndarray:
    """b = integral of |q(t)|^2 dt, q(t) = integral_0^t w, for piecewise-constant
    waveforms [n, nbins, 3] on bins of length ``bin_time`` (exact for that
    shape: q is piecewise linear)."""
    w = np.asarray(wave, dtype=np.float64)
    q0 = np.concatenate([np.zeros_like(w[:, :1]), np.cumsum(w, axis=1)[:, :-1]], axis=1) * bin_time
    # over one bin q = q0 + w s, s in [0, T]: integral |q|^2 = T|q0|^2 + T^2 q0.w + T^3|w|^2/3
    T = bin_time
    per = (T * (q0 * q0).sum(-1) + T * T * (q0 * w).sum(-1) + T ** 3 * (w * w).sum(-1) / 3.0)
    return per.sum(axis=1)


def random_smooth(n: int, nbins: int, gmax: float, seed: int = 0, nmodes: int = 6) -> np.ndarray:
    """Seeded random smooth waveforms [n, nbins, 3]: per axis a sum of the sine
    modes sin(pi m t / T), m = 1..nmodes, with random amplitudes falling as 1/m,
    minus its mean (zero net area per axis: a refocused echo), scaled so that
    the largest component of each waveform is gmax."""
    rng = np.random.default_rng(seed)
    s = (np.arange(nbins) + 0.5) / nbins
    modes = np.stack([np.sin(np.pi * m * s) for m in range(1, nmodes + 1)])     # [nmodes, nbins]
    coef = rng.normal(size=(n, 3, nmodes)) / np.arange(1, nmodes + 1)
    w = np.einsum("nam,mb->nba", coef, modes)
    w -= w.mean(axis=1, keepdims=True)     # zero net area per axis
    peak = np.abs(w).max(axis=(1, 2), keepdims=True)
    return w * (gmax / np.maximum(peak, 1e-300))


def scale_to_b(wave, bin_time: float, b) -> np.ndarray:
    """Waveforms rescaled so that each has b-value b (scalar or [n])."""
    w = np.asarray(wave, dtype=np.float64)
    b0 = bvalue(w, bin_time)
    f = np.sqrt(np.asarray(b, dtype=np.float64) / np.maximum(b0, 1e-300))
    return w * f.reshape(-1, 1, 1)
