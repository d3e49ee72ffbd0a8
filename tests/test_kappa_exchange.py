"""Permeability κ, end to end on the CPU: the library turns κ into a
permeation probability (rms_sim_create with RMS_PERM_KAPPA, the 3-D rule of
analysis/interaction.m:437-439), the oracle walks the reference's algorithm
with it (hpc_code/lib/main.cu:274-289), and the T2-weighted signal sig0(t) of
two slabs exchanging water through one membrane must follow the exact
continuum solution.

Geometry: slabs [0, a) (label 1, T2 = 50 ms) and [a, 2a) (label 2, T2 = 500
ms), a = 2 um, reflecting walls at 0 and 2a, one permeable plane at a;
walkers start uniformly.  Continuum model: dm/dt = D m'' - m / T2(x), zero
flux at the walls, flux D m' = κ (m_left - m_right) across the membrane;
sig0(t) / N = the mean of m(t) with m(0) = 1.  Solved by finite volumes
(400 cells, the membrane a conductance in series with the half cells) and
a matrix exponential.  Exchange moves magnetisation from the slow- to the
fast-relaxing slab, so sig0 at 100 ms is 13 % below the impermeable value
for κ = 0.02 um/ms.

The oracle equals the engine's COMPAT walk bit for bit (tests/test_gpu_parity),
so this pins the κ mode of the product as well.
"""
import math
import os

import numpy as np
import pytest
from scipy.linalg import expm

import pyoracle
from rms_b200 import engine

A, D0, RES, DT = 2.0, 2.0, 0.5, 0.01
T2L, T2R = 50.0, 500.0
TN, TP = 10000, 100


def continuum_sig0(kappa, times, n=200):
    h = A / n
    N = 2 * n
    L = np.zeros((N, N))
    for i in range(N):
        if i > 0 and i != n:
            L[i, i - 1] += D0 / h ** 2
            L[i, i] -= D0 / h ** 2
        if i < N - 1 and i != n - 1:
            L[i, i + 1] += D0 / h ** 2
            L[i, i] -= D0 / h ** 2
    if kappa > 0:
        G = 1.0 / (h / D0 + 1.0 / kappa)     # half cell, membrane, half cell in series
        L[n - 1, n - 1] -= G / h
        L[n - 1, n] += G / h
        L[n, n] -= G / h
        L[n, n - 1] += G / h
    L -= np.diag(np.r_[np.full(n, 1.0 / T2L), np.full(n, 1.0 / T2R)])
    return np.array([(expm(L * t) @ np.ones(N)).mean() for t in times])


def walk(kappa, npar, seed):
    nvox = int(round(A / RES))
    lab = np.zeros((2 * nvox, 4, 4), dtype=np.uint8)
    lab[:nvox] = 1
    lab[nvox:] = 2
    # the permeation table from the library's κ mode
    sim = engine.Sim(lab, dt=DT, tn=TN, npar=npar, res=RES, diffusivity=[0.0, D0, D0],
                     t2=[1e9, T2L, T2R], bval=[], bvec=np.zeros((0, 3)), timepoints=TP,
                     permeation="kappa", kappa=kappa)
    pij = sim.get("pij")
    step, t2s, _, td = pyoracle.reference_tables(DT, RES, [0.0, D0, D0], [1e9, T2L, T2R], timepoints=TP, tn=TN)
    job = pyoracle.Job(lab, dt=DT, tn=TN, npar=npar, res=RES, step=step, t2_steps=t2s, pij=pij,
                       seed=seed, timepoints=TP, td=td)
    o = pyoracle.run_oracle(job, nthreads=max(1, min(16, os.cpu_count() or 1)))
    return o["sig0"] / npar, td


@pytest.mark.parametrize("kappa", [0.02, 0.05])
def test_exchange_follows_the_continuum_solution(kappa):
    npar = 20000
    s, td = walk(kappa, npar, seed=11)
    sel = np.array([9, 24, 49, 74, 99])
    want = continuum_sig0(kappa, td[sel])
    # per-walker weights lie in [exp(-t/50), 1]: sd <= 0.5, so the mean's
    # standard error is <= 0.5 / sqrt(N) = 0.0035; allow 2 of it
    np.testing.assert_allclose(s[sel], want, atol=0.007)
    # the impermeable curve is far outside that band at late times
    none = continuum_sig0(0.0, td[sel[-1:]])
    assert none[0] - want[-1] > 0.05
    # κ read back from the last record: the κ whose continuum curve passes there
    lo, hi = 0.0, 4.0 * kappa
    for _ in range(30):
        mid = 0.5 * (lo + hi)
        if continuum_sig0(mid, td[sel[-1:]], n=50)[0] > s[sel[-1]]:
            lo = mid
        else:
            hi = mid
    assert abs(0.5 * (lo + hi) - kappa) < 0.15 * kappa, (0.5 * (lo + hi), kappa)
