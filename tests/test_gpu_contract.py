"""The multi-waveform phase contraction (rms_contract_phases) on the GPU.

Inputs as in the contraction workload: positions from a seeded Gaussian random
walk sampled on time bins (um), smooth random waveforms scaled to b-values up
to 10 ms/um^2 (phase per um per bin).  Both methods are checked against the
FP64 restatement (pyoracle.contract_phases_fp64) on the same FP32 inputs.

Tolerances (on the signal, i.e. sums divided by the walker count):
  - FP32 CUDA cores: 2e-5 (FP32 phases, |phi| up to ~20 rad: ~1e-6 relative);
  - BF16 hi/lo on the tensor cores: 1e-4 (each operand kept to 16 bits of
    mantissa; the lo x lo product is dropped).
"""
import numpy as np
import pytest

import pyoracle
from rms_b200 import engine, waveforms

pytestmark = pytest.mark.gpu


def make_inputs(nwalk, nbins, nwave, seed=0, D=2.0, T=10.0, bmax=10.0):
    rng = np.random.default_rng(seed)
    dtb = T / nbins
    steps = rng.normal(scale=np.sqrt(2 * D * dtb), size=(nwalk, nbins, 3)).astype(np.float32)
    pos = np.cumsum(steps, axis=1, dtype=np.float32)
    w = waveforms.random_smooth(nwave, nbins, 1.0, seed=seed + 1)
    b = np.linspace(0.0, bmax, nwave)
    w = waveforms.scale_to_b(w, dtb, np.maximum(b, 1e-6))
    wave = (w * dtb).astype(np.float32)     # phase per um of the bin's position
    return np.ascontiguousarray(pos), np.ascontiguousarray(wave), b


def run(pos, wave, method):
    import torch
    d_pos = torch.from_numpy(pos).cuda()
    d_wave = torch.from_numpy(wave).cuda()
    out = torch.full((wave.shape[0], 2), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ms = engine.contract_phases(d_pos.data_ptr(), pos.shape[0], pos.shape[1], d_wave.data_ptr(), wave.shape[0],
                                out.data_ptr(), method=method)
    assert ms > 0
    return out.cpu().numpy()


@pytest.mark.parametrize("method,tol", [("fp32", 2e-5), ("bf16x3", 1e-4)])
def test_contraction_ragged_sizes(method, tol):
    # walkers not a multiple of the tile, waveforms not a multiple of 128,
    # K = 48 not a multiple of the 32-wide chunk
    pos, wave, _ = make_inputs(4000, 16, 200, seed=3)
    got = run(pos, wave, method)
    want = pyoracle.contract_phases_fp64(pos, wave)
    err = np.abs(got - want).max() / pos.shape[0]
    assert err < tol, err


@pytest.mark.parametrize("method,tol", [("fp32", 2e-5), ("bf16x3", 1e-4)])
def test_contraction_full_shape_sample(method, tol):
    # the contraction workload's shape (256 bins x 3, 1024 waveforms) on 65536 walkers
    pos, wave, b = make_inputs(65536, 256, 1024, seed=7)
    got = run(pos, wave, method)
    want = pyoracle.contract_phases_fp64(pos, wave)
    err = np.abs(got - want).max(axis=1) / pos.shape[0]
    assert err.max() < tol, (err.max(), b[np.argmax(err)])
    # the signal itself decays with b (Gaussian phase): S ~ exp(-b D) for small b
    S = got[:, 0] / pos.shape[0]
    assert abs(S[0] - 1.0) < 1e-3


def test_contraction_methods_agree_and_errors():
    pos, wave, _ = make_inputs(1000, 8, 64, seed=1)
    a = run(pos, wave, "fp32")
    c = run(pos, wave, "bf16x3")
    assert np.abs(a - c).max() / 1000 < 1e-4
    pos5, wave5, _ = make_inputs(300, 5, 16, seed=2)
    got = run(pos5, wave5, "fp32")        # any nbins on the CUDA cores
    np.testing.assert_allclose(got / 300, pyoracle.contract_phases_fp64(pos5, wave5) / 300, atol=2e-5)
    with pytest.raises(engine.RmsError):
        run(pos5, wave5, "bf16x3")        # tensor path: nbins % 4 == 0


def test_presplit_positions_from_the_walk():
    """The walk writes the bin means as BF16 pairs (traj_split); the contraction
    reading them through TMA equals the one converting the FP32 means of the
    same walk, bit for bit (the same BF16 operands), and FP64 within 1e-4."""
    import torch
    from rms_b200 import geometry
    nb, nw, n = 64, 200, 5000
    dt, tn = 5e-4, 1280
    lab = geometry.axon_lattice(20, 20, 40, 0.1, seed=3, exterior=2, r0=0.5)
    dtb = dt * tn / nb
    w = waveforms.scale_to_b(waveforms.random_smooth(nw, nb, 1.0, seed=2), dtb, np.linspace(0.1, 8.0, nw))
    wave = np.ascontiguousarray((w * dtb).astype(np.float32))
    kw = dict(dt=dt, tn=tn, npar=n, res=0.1, diffusivity=[0, 2.0, 2.0], t2=[1e6, 80, 60], wave=np.zeros((1, nb, 3)),
              timepoints=nb, boundary="periodic")
    f32 = torch.empty((n, nb, 3), dtype=torch.float32, device="cuda")
    split = torch.empty((n, nb, 3), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    engine.Sim(lab, **kw).run(seed=4, precision="split", traj_out=f32.data_ptr())
    engine.Sim(lab, **kw).run(seed=4, precision="split", traj_out=split.data_ptr(), traj_split=True)
    d_wave = torch.from_numpy(wave).cuda()
    outs = {}
    for name, buf, method in (("f32", f32, "bf16x3"), ("split", split, "bf16x3_presplit")):
        out = torch.full((nw, 2), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        engine.contract_phases(buf.data_ptr(), n, nb, d_wave.data_ptr(), nw, out.data_ptr(), method=method)
        outs[name] = out.cpu().numpy()
    np.testing.assert_array_equal(outs["split"], outs["f32"])
    want = pyoracle.contract_phases_fp64(f32.cpu().numpy(), wave)
    assert np.abs(outs["split"] - want).max() / n < 1e-4
    # the pairs sum to the FP32 means to BF16 hi/lo precision
    raw = split.view(torch.int16).cpu().numpy().reshape(-1)
    m = n * nb * 3
    hi = (raw[:m].astype(np.uint32) << 16).view(np.float32)
    lo = (raw[m:2 * m].astype(np.uint32) << 16).view(np.float32)
    x = f32.cpu().numpy().reshape(-1)
    assert np.abs(hi + lo - x).max() <= 2 ** -16 * np.abs(x).max()
