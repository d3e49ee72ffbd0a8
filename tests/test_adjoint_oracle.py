"""The oracle's adjoint (or_adjoint_split, pyoracle.adjoint_split): the FP64
restatement of the GPU adjoint kernel (csrc/rms_adjoint.cu) on the replay of
the split walk, checked on the CPU against central finite differences of the
oracle's own forward walk with common random numbers (the same seed: the same
walkers and draws).

Bars, as for the GPU adjoint: the waveform gradient is exact pathwise (the
phase is linear in the waveform) and the T2 gradient analytic, so both meet
the finite difference to its truncation error; the D gradient (pathwise, the
event sequence frozen) is exact where the walk is continuous in the step
length -- periodic walls and impermeable flat membranes -- and within 1 %
there.  The GPU kernel walks the same walkers in FP32, so these sums are the
checker for its output walker set by walker set.
"""
import os

import numpy as np
import pytest

import pyoracle
from rms_b200 import engine, waveforms

DT, TN, NB, RES, N = 5e-4, 2000, 100, 0.1, 4096
W = np.random.default_rng(11).normal(size=(4, 2))
THREADS = max(1, min(16, os.cpu_count() or 1))


def planes():
    lab = np.full((24, 12, 12), 2, dtype=np.uint8)
    lab[(np.arange(24) // 6) % 2 == 0] = 1
    return lab


def base_waves(nw=4, seed=2):
    w = waveforms.random_smooth(nw, NB, 1.0, seed=seed)
    return waveforms.scale_to_b(w, DT * TN / NB, np.linspace(0.3, 1.2, nw))


def job(lab, wave, D=2.0, kappa=0.0, t2=(1e6, 70.0, 70.0), seed=5, npar=N):
    # the permeation table from the library's kappa mode (host code, no GPU)
    sim = engine.Sim(lab, dt=DT, tn=TN, npar=npar, res=RES, diffusivity=[0.0, D, D], t2=list(t2),
                     wave=wave, timepoints=100, permeation="kappa", kappa=kappa, boundary="periodic")
    pij = sim.get("pij")
    sim.close()
    step, t2s, _, td = pyoracle.reference_tables(DT, RES, [0.0, D, D], list(t2), 100, TN)
    return pyoracle.Job(lab, dt=DT, tn=TN, npar=npar, res=RES, step=step, t2_steps=t2s, pij=pij, seed=seed,
                        timepoints=100, td=td, wave=wave, boundary=pyoracle.BOUNDARY_PERIODIC)


def loss(j):
    o = pyoracle.run_oracle(j, nthreads=THREADS, split=True)
    return float((o["sigw"] * W).sum() / j.npar)


def grads(j, D=2.0, t2=(1e6, 70.0, 70.0), kappa=None):
    sums = pyoracle.adjoint_split(j, W.reshape(-1) / j.npar)
    return sums, pyoracle.adjoint_gradients(j, sums, D, t2, kappa)


def test_adjoint_walks_the_forward_walk():
    wave = base_waves()
    j = job(planes(), wave)
    sums, g = grads(j)
    o = pyoracle.run_oracle(j, nthreads=THREADS, split=True)
    np.testing.assert_allclose(sums["sigw"], o["sigw"], rtol=1e-12, atol=1e-9)
    assert g["loss"] == pytest.approx(loss(j), rel=1e-12)


def test_waveform_gradient_is_exact():
    wave = base_waves()
    lab = planes()
    _, g = grads(job(lab, wave))
    d = np.random.default_rng(3).normal(size=wave.shape) * np.abs(wave).max()
    h = 1e-4
    want = (loss(job(lab, wave + h * d)) - loss(job(lab, wave - h * d))) / (2 * h)
    got = float((g["d_wave"] * d).sum())
    assert got == pytest.approx(want, rel=1e-6)


@pytest.mark.parametrize("c", [1, 2])
def test_t2_gradient_is_exact(c):
    wave = base_waves()
    lab = planes()
    t2 = np.array([1e6, 70.0, 60.0])
    _, g = grads(job(lab, wave, t2=tuple(t2)), t2=t2)

    def f(x):
        tt = t2.copy()
        tt[c] = x
        return loss(job(lab, wave, t2=tuple(tt)))

    h = 1e-4 * t2[c]
    want = (f(t2[c] + h) - f(t2[c] - h)) / (2 * h)
    assert g["d_t2"][c] == pytest.approx(want, rel=1e-6)


def test_diffusivity_gradient_on_flat_membranes():
    # impermeable flat membranes and periodic walls: reflections are
    # continuous in the step length, so the frozen-event derivative is exact
    # almost surely
    wave = base_waves()
    lab = planes()
    _, g = grads(job(lab, wave))
    h = 1e-3
    want = (loss(job(lab, wave, D=2.0 * (1 + h))) - loss(job(lab, wave, D=2.0 * (1 - h)))) / (2 * 2.0 * h)
    assert g["d_diffusivity"] == pytest.approx(want, rel=0.01)
