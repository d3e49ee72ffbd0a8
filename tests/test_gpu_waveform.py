"""General gradient waveforms (RMS_MODE_WAVEFORM) in the split walk, on the GPU.

Three checks:
  - the reference's PGSE gradients written as one-step-per-bin waveforms give
    the PGSE signal of the same walk (same kernel, same random streams);
  - random smooth waveforms against the oracle's FP64 replay of the split walk
    (signal within 2e-3 of S0, per-walker bin means for the walkers that did
    not decorrelate within 1e-4 um);
  - free diffusion: S = exp(-b_walk D0), b_walk the b-value of the discrete
    walk's phase (dt^3 sum_k Q_k^2, Q_k the waveform's area after step k).
"""
import numpy as np
import pytest

import pyoracle
from rms_b200 import engine, geometry, waveforms

pytestmark = pytest.mark.gpu


def lattice(seed=3):
    lab = geometry.axon_lattice(16, 16, 24, 0.1, seed=seed, exterior=2, r0=0.45)
    lab[:2] = 0
    return lab


def test_pgse_as_waveform_matches_pgse_mode():
    rng = np.random.default_rng(8)
    ng, tn = 12, 2000
    g = np.column_stack([rng.choice([0.2, 0.25], ng), rng.choice([0.05, 0.1], ng),
                         rng.uniform(1, 5, ng), rng.normal(size=(ng, 3))])
    g[:, 3:] /= np.linalg.norm(g[:, 3:], axis=1, keepdims=True)
    kw = dict(dt=2e-4, tn=tn, npar=8192, res=0.1, diffusivity=[0, 2.0, 1.0], t2=[80, 80, 40])
    pg = engine.Sim(lattice(), grad=g, **kw).run(seed=4, precision="split").outputs()
    wv = engine.Sim(lattice(), wave=waveforms.pgse_waveform(g, 2e-4, tn), **kw).run(seed=4, precision="split").outputs()
    # same walk: moments and counts agree to summation order
    np.testing.assert_array_equal(wv["npar_count"], pg["npar_count"])
    np.testing.assert_allclose(wv["dx2"], pg["dx2"], rtol=1e-12, atol=1e-18)
    # phases summed per step (waveform) or per lobe (PGSE) in FP32-then-FP64:
    # the cosine sums agree to FP32 rounding of the phase
    s0 = pg["sig0"][-1]
    assert np.abs(wv["sigw"][:, 0] - pg["sig"]).max() < 1e-4 * kw["npar"]
    assert np.abs(wv["sigw"][:, 0]).max() <= kw["npar"] * 1.000001
    assert s0 > 0


def test_waveform_vs_fp64_replay_and_trajectories():
    import torch
    tn, nb, nw, n = 2000, 100, 16, 16384
    wave = waveforms.random_smooth(nw, nb, 1.0, seed=5)
    wave = waveforms.scale_to_b(wave, 2e-4 * tn / nb, np.linspace(0.2, 3.0, nw))
    D, T2 = [0, 2.0, 1.0], [80, 80, 40]
    lab = lattice(6)
    sim = engine.Sim(lab, dt=2e-4, tn=tn, npar=n, res=0.1, diffusivity=D, t2=T2, wave=wave)
    traj = torch.full((n, nb, 3), float("nan"), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    got = sim.run(seed=21, precision="split", traj_out=traj.data_ptr()).outputs()
    xb = traj.cpu().numpy()
    assert np.isfinite(xb).all()
    step, t2s, _, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, 1000, tn)
    job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=n, res=0.1, step=step, t2_steps=t2s, pij=sim.get("pij"),
                       seed=21, td=td, wave=wave)
    want = pyoracle.run_oracle(job, nthreads=8, split=True)
    S, Sw = got["sigw"] / got["sig0"][0], want["sigw"] / want["sig0"][0]
    assert np.abs(S - Sw).max() < 2e-3, np.abs(S - Sw).max()
    # per-walker bin means of the first 256 walkers against the replay's
    tr = pyoracle.run_oracle(job, w_end=256, trace_walkers=256, split=True)["trace"]["binmean"]
    err = np.abs(xb[:256] - tr).max(axis=(1, 2))
    assert (err < 1e-4).mean() >= 0.95, np.sort(err)[-20:]


def test_free_waveform_signal_matches_gaussian_limit():
    tn, nb, nw = 4000, 200, 8
    D0, dt = 2.0, 2e-4
    wave = waveforms.random_smooth(nw, nb, 1.0, seed=11)
    wave = waveforms.scale_to_b(wave, dt * tn / nb, np.linspace(0.25, 2.0, nw))
    # the discrete walk's b-value: phase = dt sum_i w_i . x_i, x_i after step i
    per_step = np.repeat(wave, tn // nb, axis=1)                       # [nw, tn, 3]
    Q = np.cumsum(per_step[:, ::-1], axis=1)[:, ::-1]                   # sum_{i >= k} w_i
    b_walk = dt ** 3 * (Q * Q).sum(axis=(1, 2))
    lab = np.ones((16, 16, 16), dtype=np.uint8)
    n = 65536
    sim = engine.Sim(lab, dt=dt, tn=tn, npar=n, res=0.1, diffusivity=[0, D0], t2=[1e12, 1e12],
                     wave=wave, boundary="periodic")
    o = sim.run(seed=2, precision="split").outputs()
    S = o["sigw"][:, 0] / n
    want = np.exp(-b_walk * D0)
    assert np.abs(S - want).max() < 4.0 / np.sqrt(n) + 2e-3, (S, want)
    assert np.abs(o["sigw"][:, 1] / n).max() < 4.0 / np.sqrt(n)


def test_waveform_mode_errors():
    lab = lattice()
    wave = waveforms.random_smooth(2, 10, 1.0)
    kw = dict(dt=2e-4, npar=64, res=0.1, diffusivity=[0, 2, 1], t2=[80, 80, 40], timepoints=10, wave=wave)
    sim = engine.Sim(lab, tn=100, **kw)
    with pytest.raises(engine.RmsError):
        sim.run(precision="compat")      # the FP64 reference-order walk has no waveform mode
    sim.run(precision="split")
    assert sim.get("sigw").shape == (4,)
    with pytest.raises(engine.RmsError):
        engine.Sim(lab, tn=105, **kw)    # TN not a multiple of the bins
