"""Edge cases on the GPU: one walker, walker counts around a warp tile, a
one-voxel periodic lattice, one step per record, a one-member batch, and a
contraction of one walker against one waveform."""
import numpy as np
import pytest

import pyoracle
from conftest import assert_fp64_close
from rms_b200 import engine, geometry, waveforms

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("npar", [1, 31, 33])
def test_walker_counts_around_a_tile_match_the_oracle(npar):
    lab = geometry.axon_lattice(12, 12, 16, 0.1, seed=1, exterior=2, r0=0.4)
    D, T2 = [0.0, 2.0, 1.0], [80.0, 80.0, 40.0]
    sim = engine.Sim(lab, dt=2e-4, tn=200, npar=npar, res=0.1, diffusivity=D, t2=T2, bval=[1.0], bvec=[[1, 0, 0]],
                     timepoints=200)
    got = sim.run(seed=3, precision="compat").outputs()
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, 200, 200)
    job = pyoracle.Job(lab, dt=2e-4, tn=200, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=3, td=td,
                       timepoints=200, bval=[1.0], bvec=[[1, 0, 0]])
    want = pyoracle.run_oracle(job)
    assert np.array_equal(got["npar_count"], want["npar_count"])
    assert_fp64_close(got["dx2"], want["dx2"], 1e-9, "dx2")
    split = sim.run(seed=3, precision="split").outputs()
    assert np.array_equal(split["npar_count"].sum(axis=1), np.full(200, float(npar)))


def test_one_voxel_periodic_lattice_is_free_diffusion():
    sim = engine.Sim(np.ones((1, 1, 1), dtype=np.uint8), dt=2e-4, tn=4000, npar=8192, res=0.1,
                     diffusivity=[0.0, 2.0], t2=[1e6, 1e6], bval=[], bvec=np.zeros((0, 3)), timepoints=100,
                     boundary="periodic")
    for prec in ("compat", "split"):
        o = sim.run(seed=5, precision=prec).outputs()
        D, _ = sim.cumulants()
        assert np.abs(D[-1] / 2.0 - 1).max() < 0.05, (prec, D[-1])
        assert np.array_equal(o["npar_count"][:, 1], np.full(100, 8192.0))


def test_one_member_batch_equals_a_single_run():
    lab = geometry.axon_lattice(16, 16, 24, 0.1, seed=2, exterior=2)
    kw = dict(dt=2e-4, tn=500, npar=3000, res=0.1, diffusivity=[0, 2.0, 2.0], t2=[80, 80, 60], bval=[],
              bvec=np.zeros((0, 3)), timepoints=100, permeation="kappa", kappa=0.02)
    a = engine.Sim(lab, **kw)
    engine.batch_run([a], seed=9, precision="split")
    b = engine.Sim(lab, **kw).run(seed=9, precision="split")
    np.testing.assert_array_equal(a.get("npar_count"), b.get("npar_count"))
    assert_fp64_close(a.get("dx2").reshape(100, 6), b.get("dx2").reshape(100, 6), 1e-12, "dx2")


def test_contraction_of_one_walker_and_one_waveform():
    import torch
    pos = np.random.default_rng(0).normal(size=(1, 8, 3)).astype(np.float32)
    wave = np.random.default_rng(1).normal(size=(1, 8, 3)).astype(np.float32)
    want = pyoracle.contract_phases_fp64(pos, wave)
    for method, tol in (("fp32", 1e-6), ("bf16x3", 5e-5)):
        d_pos, d_wave = torch.from_numpy(pos).cuda(), torch.from_numpy(wave).cuda()
        out = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        engine.contract_phases(d_pos.data_ptr(), 1, 8, d_wave.data_ptr(), 1, out.data_ptr(), method=method)
        assert np.abs(out.cpu().numpy() - want).max() < tol, method


def test_trace_and_metrics_lines(tmp_path):
    """RMS_TRACE prints one phase line per launch on stderr, and
    rms_main --metrics one JSON line of throughput; stdout keeps the
    reference's lines and the outputs are the reference program's."""
    import json
    import os
    import subprocess
    from conftest import golden_seed, unpack_golden
    from rms_b200 import runio
    d = unpack_golden("narrow_3comp", str(tmp_path / "run"), inputs_only=True)
    want = runio.read_outputs(unpack_golden("narrow_3comp", str(tmp_path / "want")))
    env = dict(os.environ, RMS_TRACE="1")
    r = subprocess.run([engine.CLI_PATH, "--seed", str(golden_seed("narrow_3comp")), "--metrics"], cwd=d, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Done! Elpased time" in r.stdout and "rms trace" not in r.stdout
    trace = [ln for ln in r.stderr.splitlines() if ln.startswith("rms trace: compat 1 sim(s)")]
    assert len(trace) == 1 and "kernels: walk" in trace[0], r.stderr
    m = json.loads([ln for ln in r.stderr.splitlines() if ln.startswith("{")][-1])
    assert m["walker_steps"] == 64 * 1000 and m["precision"] == "compat"
    assert m["walk_ms"] > 0 and m["walker_steps_per_s_walk"] > 0 and m["wall_ms"] >= m["run_ms"] > 0
    got = runio.read_outputs(d)
    assert np.array_equal(got.npar_count, want.npar_count)


@pytest.mark.parametrize("precision", ["split", "compat"])
def test_new_lattice_after_a_run_walks_the_new_lattice(precision):
    """rms_sim_set_lattice on a simulation that has run uploads the lattice
    straight from the caller's buffer; the next run equals a fresh
    simulation's run on that lattice (and the caller may reuse its buffer as
    soon as the call returns)."""
    import torch
    kw = dict(dt=2e-4, tn=500, npar=2000, res=0.1, diffusivity=[0.0, 2.0, 1.0], t2=[80.0, 80.0, 40.0],
              bval=[1.0], bvec=[[1, 0, 0]], timepoints=500)
    a = geometry.axon_lattice(16, 16, 24, 0.1, seed=1, exterior=2, r0=0.5)
    b = geometry.axon_lattice(16, 16, 24, 0.1, seed=2, exterior=2, r0=0.7)
    sim = engine.Sim(a, **kw)
    sim.run(seed=4, precision=precision)
    buf = torch.from_numpy(np.ascontiguousarray(b)).pin_memory()
    sim.set_lattice(buf.numpy())
    buf.zero_()                                # the caller's buffer is free again
    got = sim.run(seed=4, precision=precision).outputs()
    want = engine.Sim(b, **kw).run(seed=4, precision=precision).outputs()
    assert np.array_equal(got["npar_count"], want["npar_count"])
    assert_fp64_close(got["dx2"], want["dx2"], 1e-9, "dx2")
    assert_fp64_close(got["sigre"], want["sigre"], 1e-9, "sigre")


def test_refused_lattice_after_a_run_keeps_the_previous_one():
    """After a run, rms_sim_set_lattice checks the new lattice on the GPU: a
    label >= Nc or a lattice with no labelled voxel is refused with
    RMS_ERR_RANGE (the message names the first bad voxel, as the host check
    does), and the simulation keeps walking the lattice it had."""
    kw = dict(dt=2e-4, tn=500, npar=2000, res=0.1, diffusivity=[0.0, 2.0, 1.0], t2=[80.0, 80.0, 40.0],
              bval=[1.0], bvec=[[1, 0, 0]], timepoints=500)
    a = geometry.axon_lattice(16, 16, 24, 0.1, seed=1, exterior=2, r0=0.5)
    b = geometry.axon_lattice(16, 16, 24, 0.1, seed=2, exterior=2, r0=0.7)
    sim = engine.Sim(a, **kw)
    sim.run(seed=4, precision="split")
    sim.set_lattice(b)                      # accepted on the device
    bad = b.copy()
    bad[3, 4, 5] = 3
    with pytest.raises(engine.RmsError) as e:
        sim.set_lattice(bad)
    assert e.value.code == -4 and "at voxel" in str(e.value) and str(3 * 16 * 24 + 4 * 24 + 5) in str(e.value)
    with pytest.raises(engine.RmsError) as e:
        sim.set_lattice(np.zeros_like(b))
    assert e.value.code == -4
    got = sim.run(seed=4, precision="compat").outputs()
    want = engine.Sim(b, **kw).run(seed=4, precision="compat").outputs()
    assert np.array_equal(got["npar_count"], want["npar_count"])
    assert_fp64_close(got["dx2"], want["dx2"], 1e-9, "dx2")
