"""GPU parity of the FP64 reference-compatible walk (RMS_PREC_COMPAT),
through the C ABI, against the oracle and the reference's own outputs.

Bar: per-walker voxel and face-event sequences and the compartment counts
are equal bit for bit; FP64 sums agree to 1e-9 of each row's scale (the only
differences are last-bit results of sin/cos/exp and the summation order).
"""
import os
import subprocess

import numpy as np
import pytest

import pyoracle
from conftest import assert_fp64_close, golden_seed, unpack_golden
from rms_b200 import engine, geometry, runio

pytestmark = pytest.mark.gpu
RTOL = 1e-9


def sim_for(job: pyoracle.Job, **over) -> engine.Sim:
    """The product's simulation of an oracle job (tables rederived from D, T2)."""
    kw = dict(dt=job.dt, tn=job.tn, npar=job.npar, res=job.res, diffusivity=job._D, t2=job._T2,
              timepoints=job.timepoints, nite=job.nite,
              boundary="periodic" if job.boundary else "mirror")
    if job.mode == pyoracle.MODE_PGSE:
        kw["grad"] = job.grad.reshape(-1, 6)
    else:
        kw["bval"], kw["bvec"] = job.bval, job.bvec.reshape(-1, 3)
    kw.update(over)
    return engine.Sim(job.labels, **kw)


def make_job(lab, *, D, T2, dt=2e-4, tn=1000, npar=64, res=0.1, seed=1, timepoints=1000,
             nite=4, boundary=0, bval=None, bvec=None, grad=None, pij=None, kappa=None):
    step, t2s, pij_ref, _ = pyoracle.reference_tables(dt, res, D, T2, timepoints, tn)
    job = pyoracle.Job(lab, dt=dt, tn=tn, npar=npar, res=res, step=step, t2_steps=t2s,
                       pij=pij if pij is not None else pij_ref, seed=seed, timepoints=timepoints,
                       nite=nite, boundary=boundary, bval=bval, bvec=bvec, grad=grad)
    job._D, job._T2 = list(D), list(T2)
    return job


def compare(job, sim_over=None, trace=True):
    sim = sim_for(job, **(sim_over or {}))
    sim.run(seed=job.seed, precision="compat", trace_walkers=job.npar if trace else 0)
    got = sim.outputs()
    want = pyoracle.run_oracle(job, trace_walkers=job.npar if trace else 0)
    if trace:
        tg, tw = sim.trace(job.npar), want["trace"]
        assert np.array_equal(tg["init_voxel"], tw["init_voxel"]), "initial voxels differ"
        bad = np.argwhere(tg["voxel"] != tw["voxel"])
        assert bad.size == 0, f"voxel sequences differ first at walker/step {bad[:3].tolist()}"
        assert np.array_equal(tg["events"], tw["events"]), "face-event sequences differ"
        # positions agree to the last bits of sin/cos (CUDA's vs glibc's)
        assert np.abs(tg["pos"] - tw["pos"]).max() < 1e-9, "positions drift apart"
    assert np.array_equal(got["npar_count"], want["npar_count"]), "compartment counts differ"
    assert_fp64_close(got["sig0"], want["sig0"], RTOL, "sig0")
    assert_fp64_close(got["dx2"], want["dx2"], RTOL, "dx2")
    assert_fp64_close(got["dx4"], want["dx4"], RTOL, "dx4")
    if job.mode == pyoracle.MODE_PGSE:
        assert_fp64_close(got["sig"], want["sig"], RTOL, "sig")
    elif job.nbvec:
        assert_fp64_close(got["sigre"], want["sigre"], RTOL, "sigRe")
    return sim, got, want


def lattice3(seed=1, shape=(16, 16, 24), r0=0.45):
    lab = geometry.axon_lattice(*shape, 0.1, seed=seed, exterior=2, r0=r0)
    lab[:2, :, :] = 0
    return lab


def test_narrow_three_compartments_traces():
    rng = np.random.default_rng(0)
    bv = rng.normal(size=(40, 3)); bv /= np.linalg.norm(bv, axis=1, keepdims=True)
    job = make_job(lattice3(), D=[0, 2.0, 1.0], T2=[80, 80, 40], npar=96, seed=11,
                   bval=rng.uniform(0.1, 3, 40), bvec=bv)
    compare(job)


def test_pgse_three_compartments_traces():
    rng = np.random.default_rng(1)
    ng = 70
    g = np.column_stack([rng.choice([0.05, 0.1, 0.15], ng), rng.choice([0.02, 0.0503, 0.1], ng),
                         rng.uniform(0.5, 5, ng), rng.normal(size=(ng, 3))])
    g[:, 3:] /= np.linalg.norm(g[:, 3:], axis=1, keepdims=True)
    job = make_job(lattice3(2), D=[0, 2.0, 1.5], T2=[80, 70, 50], npar=80, tn=2000, seed=5, grad=g)
    compare(job)


def test_periodic_boundary():
    lab = geometry.axon_lattice(10, 10, 16, 0.1, seed=4, exterior=2, r0=0.3)
    job = make_job(lab, D=[0, 2.0, 2.0], T2=[80, 80, 80], npar=64, seed=3, boundary=1,
                   bval=[1.0], bvec=[[0, 0, 1]])
    compare(job)


def kappa_job(nite, tn, timepoints):
    lab = lattice3(3)
    D, T2, dt = [0, 2.0, 2.0], [80, 60, 60], 2e-4
    s_probe = engine.Sim(lab, dt=dt, tn=1000, npar=8, res=0.1, diffusivity=D, t2=T2,
                         bval=[1.0], bvec=[[1, 0, 0]], permeation="kappa", kappa=0.05)
    pij = s_probe.get("pij")
    return make_job(lab, D=D, T2=T2, npar=64, seed=8, tn=tn, timepoints=timepoints, nite=nite,
                    bval=[1.0, 2.0], bvec=[[1, 0, 0], [0, 1, 0]], pij=pij)


def test_kappa_permeation_and_timepoints():
    compare(kappa_job(4, 1500, 300), sim_over=dict(permeation="kappa", kappa=0.05))


def test_small_nite_bounded_horizon():
    """With nite < 4 walkers often end a step on a face; the next step's
    grazing first segment then scales a position difference by 1/|v_a|, so the
    last-bit sin/cos differences between CUDA and glibc grow geometrically and
    traces separate after a few hundred steps (measured: first voxel
    difference near step 1240 of 1500 with nite = 2; none with nite = 4).
    Checked: identical traces over the first 100 steps, positions within 1e-9."""
    job = kappa_job(2, 1000, 1000)
    sim = sim_for(job, permeation="kappa", kappa=0.05)
    sim.run(seed=job.seed, precision="compat", trace_walkers=job.npar)
    tg = sim.trace(job.npar)
    tw = pyoracle.run_oracle(job, trace_walkers=job.npar)["trace"]
    h = 100
    assert np.array_equal(tg["voxel"][:, :h], tw["voxel"][:, :h])
    assert np.array_equal(tg["events"][:, :h], tw["events"][:, :h])
    assert np.abs(tg["pos"][:, :h] - tw["pos"][:, :h]).max() < 1e-9
    dropped = ((tw["events"][:, :h] >> 31) & 1).sum()
    assert dropped > 0   # the cap is exercised


def test_max_nite_and_walls():
    # a lattice with lots of faces per step: the 7-segment cap and mirror walls
    lab = np.ones((3, 3, 3), dtype=np.uint8)
    lab[1, 1, 1] = 2
    job = make_job(lab, D=[0, 2.0, 0.5], T2=[80, 80, 80], npar=64, seed=2, nite=7, res=0.06,
                   bval=[1.0], bvec=[[1, 0, 0]])
    compare(job)


def test_multi_warp_shards_sum_to_whole():
    job = make_job(lattice3(4), D=[0, 2.0, 1.0], T2=[80, 80, 40], npar=200, seed=21,
                   bval=[1.0], bvec=[[1, 0, 0]])
    sim = sim_for(job)
    whole = sim.run(seed=job.seed).outputs()
    parts = [sim_for(job).run(seed=job.seed, walker_range=r).outputs() for r in ((0, 77), (77, 200))]
    assert np.array_equal(parts[0]["npar_count"] + parts[1]["npar_count"], whole["npar_count"])
    assert_fp64_close(parts[0]["dx2"] + parts[1]["dx2"], whole["dx2"], 1e-12, "dx2")


def test_rerun_is_bitwise_repeatable():
    job = make_job(lattice3(5), D=[0, 2.0, 1.0], T2=[80, 80, 40], npar=500, seed=9,
                   bval=[1.0, 2.0], bvec=[[1, 0, 0], [0, 0, 1]])
    sim = sim_for(job)
    a = sim.run(seed=9).outputs()
    b = sim.run(seed=9).outputs()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("case", ["narrow_3comp", "pgse_3comp", "realistic_mito_1", "realistic_undulation_pgse"])
def test_matches_reference_program_outputs(case, tmp_path):
    """The golden run directories hold the reference program's own output
    files (hpc_code/lib/main*.cu run on the host with the same seed).  The
    realistic cases walk the reference's own axons: realistic_mito_1 (its
    first mitochondria axon, 0.2 % of the voxels labelled -- rejection-sampled
    starts take ~480 tries, main.cu:117-125 -- and partial permeation into the
    mitochondria, P = 0.258, main.cu:274-289) and realistic_undulation_pgse
    (its first undulating axon under five PGSE gradients, main_PGSE.cu)."""
    d = unpack_golden(case, str(tmp_path / "run"), inputs_only=True)
    want_dir = unpack_golden(case, str(tmp_path / "want"))
    sim = engine.Sim.from_dir(d).run(seed=golden_seed(case))
    sim.write_dir(d)
    got, want = runio.read_outputs(d), runio.read_outputs(want_dir)
    assert np.array_equal(got.npar_count, want.npar_count)
    assert np.array_equal(got.sim_para, want.sim_para)
    assert np.array_equal(got.diff_time, want.diff_time)
    assert_fp64_close(got.sig0, want.sig0, 1e-12, "sig0")
    assert_fp64_close(got.dx2, want.dx2, RTOL, "dx2")
    assert_fp64_close(got.dx4, want.dx4, RTOL, "dx4")
    if want.sig is not None:
        assert_fp64_close(got.sig, want.sig, RTOL, "sig")
    else:
        assert_fp64_close(got.sigre, want.sigre, RTOL, "sigRe")
    # identical file layout: line count and columns per line
    for fn in os.listdir(want_dir):
        if fn in ("sig0.txt", "dx2.txt", "dx4.txt", "sigRe.txt", "sig.txt", "NPar_count.txt",
                  "sim_para.txt", "diff_time.txt"):
            a = open(os.path.join(d, fn)).read().split("\n")
            b = open(os.path.join(want_dir, fn)).read().split("\n")
            assert [len(x.split("\t")) for x in a] == [len(x.split("\t")) for x in b], fn


def test_cli_drop_in(tmp_path):
    d = unpack_golden("pgse_3comp", str(tmp_path / "run"), inputs_only=True)
    want = runio.read_outputs(unpack_golden("pgse_3comp", str(tmp_path / "want")))
    r = subprocess.run([engine.CLI_PATH, "--seed", str(golden_seed("pgse_3comp"))], cwd=d,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Done! Elpased time" in r.stdout
    assert r.stdout.count("permeation probability=") == 9
    got = runio.read_outputs(d)
    assert np.array_equal(got.npar_count, want.npar_count)
    assert_fp64_close(got.sig, want.sig, RTOL, "sig")


def test_cli_binary_lattice_gives_the_reference_outputs(tmp_path):
    """fiber.bin (raw bytes) in place of fiber.txt: the same walk, the same
    reference output files."""
    d = unpack_golden("narrow_3comp", str(tmp_path / "run"), inputs_only=True)
    want = runio.read_outputs(unpack_golden("narrow_3comp", str(tmp_path / "want")))
    vals = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8)
    os.remove(os.path.join(d, "fiber.txt"))
    runio.write_lattice_binary(os.path.join(d, "fiber.bin"), vals)
    r = subprocess.run([engine.CLI_PATH, "--seed", str(golden_seed("narrow_3comp"))], cwd=d,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = runio.read_outputs(d)
    assert np.array_equal(got.npar_count, want.npar_count)
    assert_fp64_close(got.sigre, want.sigre, RTOL, "sigRe")
    assert_fp64_close(got.dx4, want.dx4, RTOL, "dx4")
