"""The oracle's adjoint (or_adjoint_split, pyoracle.adjoint_split): the FP64
restatement of the GPU adjoint kernel (csrc/rms_adjoint.cu) on the replay of
the split walk, checked on the CPU against central finite differences of the
oracle's own forward walk with common random numbers (the same seed: the same
walkers and draws).

Bars, as for the GPU adjoint: the waveform gradient is exact pathwise (the
phase is linear in the waveform) and the T2 gradient analytic, so both meet
the finite difference to its truncation error; the pathwise D gradient (the
event sequence frozen) is exact where the walk is continuous in the step
length -- periodic walls and impermeable flat membranes -- and within 1 %
there; on a voxelised axon it misses the jumps at the membrane's corners,
which the time-rescaling D gradient sees (checked against the least-squares
slope of the loss over +-5 % of D).  The GPU kernel walks the same walkers in
FP32, so these sums are the checker for its output walker set by walker set.
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
    assert g["d_diffusivity_pathwise"] == pytest.approx(want, rel=0.01)


def test_time_rescaling_sees_the_corner_jumps_of_a_voxelised_axon():
    """On a voxelised axon (kappa = 0) the walk's output jumps in the step
    length where a trajectory strikes a membrane face or passes its corner;
    the pathwise D gradient misses those jumps (measured: -60 %), the
    time-rescaling one does not.  Reference: the least-squares slope of the
    loss over D +- 5 % (seven points, common random numbers), two seeds of
    16384 walkers; the time-rescaling estimate's spread is about 8 % per run
    here, so the bar is 15 % on the two-seed mean."""
    from rms_b200 import geometry
    wave = base_waves()
    lab = geometry.axon_lattice(24, 24, 48, RES, seed=4, exterior=2, r0=0.6)
    n, seeds = 16384, (5, 6)
    tr, path, ref = [], [], []
    for seed in seeds:
        _, g = grads(job(lab, wave, npar=n, seed=seed))
        tr.append(g["d_diffusivity"])
        path.append(g["d_diffusivity_pathwise"])
        xs = 2.0 * (1 + 0.05 * np.linspace(-1, 1, 7))
        ref.append(np.polyfit(xs, [loss(job(lab, wave, D=x, npar=n, seed=seed)) for x in xs], 1)[0])
    want = float(np.mean(ref))
    assert float(np.mean(tr)) == pytest.approx(want, rel=0.15), (tr, ref)
    assert float(np.mean(path)) / want < 0.6, (path, ref)


def test_forced_draws_and_score_function_agree_on_kappa():
    """Two unbiased estimates of dL/dkappa on a permeable voxelised axon
    (kappa = 0.05, T2 80 / 20 ms so that a crossing changes the loss): the
    forced draws (one permeation draw per walker walked the other way, the
    rest of the walk on the same streams) and the score function.  Over 8
    walker shards of 2048 their means agree within 3 standard errors of the
    difference, and the forced draws' spread is under half the score's
    (measured: 0.012 vs 0.053 for this seed)."""
    from rms_b200 import geometry
    wave = base_waves()
    lab = geometry.axon_lattice(24, 24, 48, RES, seed=4, exterior=2, r0=0.6)
    t2, n, kap = (1e6, 80.0, 20.0), 16384, 0.05
    j = job(lab, wave, kappa=kap, t2=t2, npar=n, seed=7)
    forced, score = [], []
    for k in range(8):
        sk = pyoracle.adjoint_split(j, W.reshape(-1) / n, n * k // 8, n * (k + 1) // 8)
        assert sk["F"] != 0.0
        gk = pyoracle.adjoint_gradients(j, sk, 2.0, t2, kap, nwalk=n // 8)
        forced.append(8 * gk["d_kappa"])
        score.append(8 * gk["d_kappa_score"])
    se_f = np.std(forced, ddof=1) / np.sqrt(8)
    se_s = np.std(score, ddof=1) / np.sqrt(8)
    assert abs(np.mean(forced) - np.mean(score)) < 3 * np.hypot(se_f, se_s), (forced, score)
    assert se_f < 0.5 * se_s, (se_f, se_s)


def test_forced_draws_vanish_without_permeation():
    """kappa = 0: no permeation draw is made, so the forced-draw sum is 0."""
    wave = base_waves()
    sums, g = grads(job(planes(), wave))
    assert sums["F"] == 0.0 and sums["E"] == 0.0
