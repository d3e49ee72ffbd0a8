"""The general-waveform mode's oracle and host helpers, on CPU.

The waveform mode is an engine extension (the reference's only gradient form
is the PGSE pair of hpc_code/lib/main_PGSE.cu:336-346).  Its FP64 replay in
the oracle is pinned to the PGSE replay: the reference's PGSE gradients
written as one-step-per-bin waveforms give the same phases, so the cosine
sums equal the PGSE signal up to summation order.
"""
import numpy as np

import pyoracle
from rms_b200 import geometry, waveforms


def _job(lab, *, tn, npar, seed, grad=None, wave=None, boundary=0):
    D, T2 = [0, 2.0, 1.5], [80, 80, 40]
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, 100, tn)
    return pyoracle.Job(lab, dt=2e-4, tn=tn, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij,
                        seed=seed, td=td, timepoints=100, boundary=boundary, grad=grad, wave=wave)


def test_pgse_as_waveform_matches_pgse_replay():
    lab = geometry.axon_lattice(12, 12, 20, 0.1, seed=2, exterior=2, r0=0.35)
    tn = 400
    rng = np.random.default_rng(0)
    ng = 6
    g = np.column_stack([rng.choice([0.03, 0.05], ng), rng.choice([0.01, 0.02], ng),
                         rng.uniform(1, 6, ng), rng.normal(size=(ng, 3))])
    g[:, 3:] /= np.linalg.norm(g[:, 3:], axis=1, keepdims=True)
    pg = pyoracle.run_oracle(_job(lab, tn=tn, npar=200, seed=5, grad=g), split=True)
    wave = waveforms.pgse_waveform(g, 2e-4, tn)
    wv = pyoracle.run_oracle(_job(lab, tn=tn, npar=200, seed=5, wave=wave), split=True)
    np.testing.assert_allclose(wv["sigw"][:, 0], pg["sig"], rtol=1e-10, atol=1e-10)
    # the walk itself is the same
    np.testing.assert_array_equal(wv["dx2"], pg["dx2"])
    np.testing.assert_array_equal(wv["npar_count"], pg["npar_count"])


def test_waveform_bin_means_sum_to_phase():
    lab = np.ones((10, 10, 10), dtype=np.uint8)
    tn, nb = 300, 30
    wave = waveforms.random_smooth(4, nb, 1.0, seed=3)
    job = _job(lab, tn=tn, npar=3, seed=9, wave=wave, boundary=1)
    o = pyoracle.run_oracle(job, trace_walkers=3, split=True)
    xb = o["trace"]["binmean"]                       # [walkers, bins, 3], um
    phase = 2e-4 * (tn // nb) * np.einsum("wba,jba->wj", xb, wave)
    T2s = job.t2[1]
    s0 = np.exp(-tn / T2s)
    np.testing.assert_allclose(o["sigw"][:, 0], (s0 * np.cos(phase)).sum(0), rtol=1e-9)
    np.testing.assert_allclose(o["sigw"][:, 1], (s0 * np.sin(phase)).sum(0), rtol=1e-9, atol=1e-12)
    # periodic walls: bin means are differences of the traced positions up
    # to the (unknown) start, so consecutive bins' means differ by the mean
    # of the traced positions' differences
    pos = o["trace"]["pos"] * 0.1                    # um, folded into the 1 um box
    step = np.diff(pos, axis=1)
    step -= np.round(step / 1.0)                     # undo the wraps
    pos = np.concatenate([pos[:, :1], pos[:, :1] + np.cumsum(step, axis=1)], axis=1)
    mb = pos.reshape(3, nb, tn // nb, 3).mean(axis=2)
    np.testing.assert_allclose(np.diff(xb, axis=1), np.diff(mb, axis=1), atol=1e-9)


def test_bvalue_of_pgse_waveform():
    dt, tn = 1e-3, 20000
    Delta, delta, g = 10.0, 4.0, 0.05
    wave = waveforms.pgse_waveform([[Delta, delta, g, 1, 0, 0]], dt, tn)
    b = waveforms.bvalue(wave, dt)[0]
    want = g * g * delta * delta * (Delta - delta / 3)       # readRMS_pgse.m:53
    assert abs(b / want - 1) < 2e-3


def test_random_smooth_and_scale():
    w = waveforms.random_smooth(8, 64, 0.02, seed=1)
    assert w.shape == (8, 64, 3)
    assert np.allclose(np.abs(w).max(axis=(1, 2)), 0.02)
    assert np.abs(w.sum(axis=1)).max() < 1e-12
    ws = waveforms.scale_to_b(w, 0.1, np.linspace(1, 8, 8))
    np.testing.assert_allclose(waveforms.bvalue(ws, 0.1), np.linspace(1, 8, 8), rtol=1e-12)
