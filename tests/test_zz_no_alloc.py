"""rms_sim_run_noalloc, the walk for callers that cannot allocate device
memory (their memory belongs to their own allocator, or they must not hit
cudaMalloc's device-wide synchronisation).  The caller owns the lattice and
output buffers -- here torch tensors -- and the library keeps all its scratch
in one fixed device array.

Checked through the C ABI against the ordinary entry point (rms_sim_run, split
walk) on the same job: the same walkers are walked, so compartment counts are
equal and the FP64 sums agree to 1e-9 of each row's scale (only the summation
order differs).  Two calls in a row: the second shows the shared scratch is
cleared between calls.  This file runs last (pytest collects it last) so a
failure here never hides the other tests' results.
"""
import numpy as np
import pytest

from conftest import assert_fp64_close
from rms_b200 import engine, geometry

pytestmark = pytest.mark.gpu


def unpack(rows: np.ndarray, T: int, nbvec: int, nc: int, mode: str) -> dict:
    """Row layout of include/rms.h: sig0 | dx2 x6 | dx4 x15 | counts | (sigRe)."""
    W = 32 if mode == "pgse" else 32 + 32 * ((nbvec + 31) // 32)
    r = rows.reshape(T, W)
    o = dict(sig0=r[:, 0], dx2=r[:, 1:7], dx4=r[:, 7:22], npar_count=r[:, 22:22 + nc])
    if mode == "narrow":
        o["sigre"] = r[:, 32:32 + nbvec]
    return o


@pytest.mark.parametrize("mode", ["narrow", "pgse"])
def test_noalloc_walk_matches_rms_sim_run(mode):
    import torch
    lab = geometry.axon_lattice(20, 20, 32, 0.1, seed=7, exterior=2, r0=0.6)
    lab[:2] = 0
    kw = dict(dt=2e-4, tn=1000, npar=20000, res=0.1, diffusivity=[0, 2.0, 1.0], t2=[80, 80, 40])
    nbvec = 0
    if mode == "pgse":
        g = np.array([[0.1, 0.05, 2.0, 1, 0, 0], [0.15, 0.05, 3.0, 0, 0.6, 0.8], [0.05, 0.02, 4.0, 0, 1, 0]])
        kw["grad"] = g
    else:
        nbvec = 5
        kw["bval"] = [0.5, 1, 1.5, 2, 3.0]
        kw["bvec"] = np.tile([[0.6, 0.8, 0.0]], (5, 1))
    sim = engine.Sim(lab, **kw)
    want = sim.run(seed=11, precision="split").outputs()

    T, nc = 1000, 3
    W = 32 if mode == "pgse" else 32 + 32 * ((nbvec + 31) // 32)
    d_lab = torch.from_numpy(np.ascontiguousarray(lab)).cuda()
    rows = torch.empty(T * W, dtype=torch.float64, device="cuda")
    sig = torch.empty(32, dtype=torch.float64, device="cuda")
    for call in range(2):
        rows.fill_(float("nan"))   # every value must be written by the call
        sig.fill_(float("nan"))
        torch.cuda.synchronize()
        sim.run_noalloc(d_lab.data_ptr(), rows.data_ptr(), sig.data_ptr() if mode == "pgse" else 0, seed=11)
        got = unpack(rows.cpu().numpy(), T, nbvec, nc, mode)
        assert np.array_equal(got["npar_count"], want["npar_count"]), f"call {call}: counts differ"
        for k in ("sig0", "dx2", "dx4") + (("sigre",) if mode == "narrow" else ()):
            assert_fp64_close(got[k], want[k], 1e-9, f"call {call}: {k}")
        if mode == "pgse":
            assert_fp64_close(sig.cpu().numpy()[:3], want["sig"], 1e-9, f"call {call}: sig")


def _many_compartments(nc: int) -> np.ndarray:
    """Axon (label 1) in label-2 exterior, the exterior cut into z slabs that
    carry labels 3 .. nc-1."""
    lab = geometry.axon_lattice(16, 16, 40, 0.1, seed=5, exterior=2, r0=0.5)
    slab = 40 // nc
    for c in range(3, nc):
        part = lab[:, :, (c - 2) * slab:(c - 1) * slab]
        part[part == 2] = c
    lab[:1] = 0
    return lab


@pytest.mark.parametrize("nc", [5, 7])
def test_noalloc_many_compartments_match_rms_sim_run(nc):
    """Nc up to the no-allocation walk's limit of 7: the compartment tables
    it builds on the host stack hold 2 Nc + Nc^2 entries."""
    import torch
    lab = _many_compartments(nc)
    D = [0.0] + [1.0 + 0.15 * c for c in range(1, nc)]
    T2 = [80.0] + [30.0 + 10.0 * c for c in range(1, nc)]
    kw = dict(dt=2e-4, tn=1000, npar=8192, res=0.1, diffusivity=D, t2=T2, bval=[1.0, 2.0],
              bvec=[[1.0, 0, 0], [0, 0.6, 0.8]])
    sim = engine.Sim(lab, **kw)
    want = sim.run(seed=3, precision="split").outputs()
    assert (want["npar_count"][0, 3:] > 0).all(), "every extra compartment holds walkers"
    T, W = 1000, 64
    d_lab = torch.from_numpy(np.ascontiguousarray(lab)).cuda()
    rows = torch.empty(T * W, dtype=torch.float64, device="cuda")
    for call in range(2):
        rows.fill_(float("nan"))
        torch.cuda.synchronize()
        sim.run_noalloc(d_lab.data_ptr(), rows.data_ptr(), 0, seed=3)
        got = unpack(rows.cpu().numpy(), T, 2, nc, "narrow")
        assert np.array_equal(got["npar_count"], want["npar_count"]), f"call {call}: counts differ"
        for k in ("sig0", "dx2", "dx4", "sigre"):
            assert_fp64_close(got[k], want[k], 1e-9, f"call {call}: {k}")


def test_noalloc_checks_the_device_lattice():
    """The caller's device lattice is checked before the walk: a label >= Nc
    and a lattice without labelled voxels are refused (RMS_ERR_RANGE), and a
    good lattice still runs afterwards."""
    import torch
    lab = geometry.axon_lattice(12, 12, 16, 0.1, seed=2, exterior=2, r0=0.4)
    sim = engine.Sim(lab, dt=2e-4, tn=1000, npar=256, res=0.1, diffusivity=[0, 2.0, 1.0], t2=[80, 80, 40],
                     bval=[1.0], bvec=[[1.0, 0, 0]])
    rows = torch.empty(1000 * 64, dtype=torch.float64, device="cuda")
    for bad_label in (3, 7, 9):
        bad = lab.copy()
        bad[5, 6, 7] = bad_label
        d_bad = torch.from_numpy(bad).cuda()
        with pytest.raises(engine.RmsError) as e:
            sim.run_noalloc(d_bad.data_ptr(), rows.data_ptr(), 0, seed=1)
        assert e.value.code == -4 and "not below Nc" in str(e.value)
    d_zero = torch.zeros(lab.shape, dtype=torch.uint8, device="cuda")
    with pytest.raises(engine.RmsError) as e:
        sim.run_noalloc(d_zero.data_ptr(), rows.data_ptr(), 0, seed=1)
    assert e.value.code == -4
    # an odd start address exercises the check's unaligned head and tail
    buf = torch.zeros(lab.size + 1, dtype=torch.uint8, device="cuda")
    buf[1:] = torch.from_numpy(lab.reshape(-1))
    sim.run_noalloc(buf.data_ptr() + 1, rows.data_ptr(), 0, seed=1)
    want = sim.run(seed=1, precision="split").outputs()
    got = unpack(rows.cpu().numpy(), 1000, 1, 3, "narrow")
    assert np.array_equal(got["npar_count"], want["npar_count"])


def test_noalloc_refuses_oversized_job():
    import torch
    lab = np.ones((8, 8, 8), dtype=np.uint8)
    # 2000 timepoints x (32 + 4064) doubles per warp row block exceeds the scratch
    sim = engine.Sim(lab, dt=2e-4, tn=2000, npar=64, res=0.1, diffusivity=[0, 2.0], t2=[80, 80],
                     timepoints=2000, bval=np.ones(4064), bvec=np.tile([[1.0, 0, 0]], (4064, 1)))
    d_lab = torch.from_numpy(lab).cuda()
    rows = torch.empty(8, dtype=torch.float64, device="cuda")
    with pytest.raises(engine.RmsError) as e:
        sim.run_noalloc(d_lab.data_ptr(), rows.data_ptr(), 0, seed=1)
    assert e.value.code == -4
