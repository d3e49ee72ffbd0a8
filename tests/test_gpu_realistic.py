"""GPU parity at the benchmark's shapes and on the reference's own geometry,
through the C ABI.

* COMPAT (FP64, the reference's arithmetic) on the 64 x 64 x 512 single-axon
  lattice of the single-axon configuration (1e5 walkers, 5000 steps, moments
  every 10 steps, periodic walls): per-walker voxel and face-event sequences
  of a walker subset equal the oracle's bit for bit, and the whole job's
  counts and sums equal the oracle's (counts exactly, sums to 1e-9 of each
  row's scale).
* COMPAT traces on the reference's first mitochondria axon
  (hpc_code/input/I_realistic_axon_mitochondria/fiber.mat, golden case
  realistic_mito_1): sparse rejection sampling and partial permeation.
* SPLIT against the FP64 replay of the same walkers (oracle or_run_split) on
  the single-axon lattice and on the mitochondria axon, 16384 walkers: D(t)
  within 0.5 %, K(t) within 2 % (absolute 0.02 where |K| < 1), records 50 on.
"""
import os

import numpy as np
import pytest

import pyoracle
from conftest import assert_fp64_close, unpack_golden
from rms_b200 import analysis, engine, geometry

pytestmark = pytest.mark.gpu
THREADS = max(1, min(32, os.cpu_count() or 1))


def single_axon_job(npar, seed, tn=5000, timepoints=500):
    lab = geometry.config_axon("single", seed=0)
    D, T2, dt = [0.0, 2.0], [1e12, 1e12], 2e-4
    step, t2s, pij, td = pyoracle.reference_tables(dt, 0.1, D, T2, timepoints, tn)
    job = pyoracle.Job(lab, dt=dt, tn=tn, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=seed,
                       timepoints=timepoints, td=td, boundary=pyoracle.BOUNDARY_PERIODIC,
                       bval=[1.0, 2.0], bvec=[[1.0, 0, 0], [0, 0, 1.0]])
    sim = engine.Sim(lab, dt=dt, tn=tn, npar=npar, res=0.1, diffusivity=D, t2=T2, timepoints=timepoints,
                     boundary="periodic", bval=[1.0, 2.0], bvec=[[1.0, 0, 0], [0, 0, 1.0]])
    return sim, job


def mito_job(npar, seed, tn=2000, timepoints=1000, tmp=None):
    d = unpack_golden("realistic_mito_1", tmp, inputs_only=True)
    vals = open(os.path.join(d, "simParamInput.txt")).read().split()
    n1, n2, n3 = (int(x) for x in vals[-3:])
    lab = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8).reshape(n1, n2, n3)
    D = [float(x) for x in open(os.path.join(d, "diffusivity.txt")).read().split()]
    T2 = [float(x) for x in open(os.path.join(d, "T2.txt")).read().split()]
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, timepoints, tn)
    bval, bvec = [1.0, 2.5], [[0.6, 0.8, 0.0], [0.0, 0.0, 1.0]]
    job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=seed,
                       timepoints=timepoints, td=td, bval=bval, bvec=bvec)
    sim = engine.Sim(lab, dt=2e-4, tn=tn, npar=npar, res=0.1, diffusivity=D, t2=T2, timepoints=timepoints,
                     bval=bval, bvec=bvec)
    return sim, job


def check_traces_and_sums(sim, job, ntrace):
    sim.run(seed=job.seed, precision="compat", trace_walkers=ntrace)
    got = sim.outputs()
    tg = sim.trace(ntrace)
    tw = pyoracle.run_oracle(job, 0, ntrace, trace_walkers=ntrace)["trace"]
    assert np.array_equal(tg["init_voxel"], tw["init_voxel"]), "initial voxels differ"
    bad = np.argwhere(tg["voxel"] != tw["voxel"])
    assert bad.size == 0, f"voxel sequences differ first at walker/step {bad[:3].tolist()}"
    assert np.array_equal(tg["events"], tw["events"]), "face-event sequences differ"
    want = pyoracle.run_oracle(job, nthreads=THREADS)
    assert np.array_equal(got["npar_count"], want["npar_count"]), "compartment counts differ"
    for k in ("sig0", "dx2", "dx4", "sigre"):
        assert_fp64_close(got[k], want[k], 1e-9, k)
    return tg


def check_split(sim, job, td):
    got = sim.run(seed=job.seed, precision="split").outputs()
    want = pyoracle.run_oracle(job, nthreads=THREADS, split=True)
    Dg, Kg = analysis.axis_dk(got["sig0"], got["dx2"], got["dx4"], td)
    Dw, Kw = analysis.axis_dk(want["sig0"], want["dx2"], want["dx4"], td)
    sl = slice(50, None)
    dD = np.abs(Dg[sl] / Dw[sl] - 1).max()
    dK = (np.abs(Kg[sl] - Kw[sl]) / np.maximum(np.abs(Kw[sl]), 1.0)).max()
    assert dD < 0.005, f"D(t) differs from the FP64 replay by {dD:.2e}"
    assert dK < 0.02, f"K(t) differs from the FP64 replay by {dK:.2e}"
    assert np.array_equal(got["npar_count"].sum(axis=1), want["npar_count"].sum(axis=1))
    S, Sw = got["sigre"] / got["sig0"][:, None], want["sigre"] / want["sig0"][:, None]
    assert np.abs(S - Sw).max() < 2e-3
    return dD, dK


def test_compat_single_axon_lattice_traces_and_sums():
    sim, job = single_axon_job(100_000, seed=13)
    tg = check_traces_and_sums(sim, job, 256)
    # the traced walkers leave their start voxel and meet the membrane
    assert (tg["events"] != 0).any()


def test_compat_reference_mito_axon_traces(tmp_path):
    sim, job = mito_job(1024, seed=29, tmp=str(tmp_path))
    tg = check_traces_and_sums(sim, job, 1024)
    assert (tg["events"] != 0).any()


def test_split_vs_fp64_replay_single_axon_lattice():
    sim, job = single_axon_job(16384, seed=41)
    check_split(sim, job, job.td)


def test_split_vs_fp64_replay_reference_mito_axon(tmp_path):
    sim, job = mito_job(16384, seed=43, tmp=str(tmp_path))
    check_split(sim, job, job.td)
