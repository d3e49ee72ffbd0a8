"""Pins the oracle (oracle/rms_oracle.c, the C restatement of the reference
walk) to the reference itself.

1. Against the golden run directories: output files written by the reference
   program (hpc_code/lib/main.cu, main_PGSE.cu compiled for the host through
   oracle/ref_shim), regenerated by tests/golden/make_golden.py -- including
   one of the reference's own realistic lattices (an axon with mitochondria,
   0.2 % of the box labelled: ~480 rejection-sampling tries per walker).
2. Against the reference host build directly (oracle/_ref), bit for bit, on
   fresh random jobs -- skipped when that build is absent.
"""
import math
import os

import numpy as np
import pytest

import pyoracle
from conftest import golden_seed, unpack_golden
from rms_b200 import geometry, runio


def job_from_dir(d, seed):
    """The oracle job for a run directory, with the tables derived exactly as
    the reference's main() derives them (main.cu:414-487)."""
    vals = open(os.path.join(d, "simParamInput.txt")).read().split()
    pgse = os.path.exists(os.path.join(d, "gradient_time.txt"))
    dt, tn, npar = float(vals[0]), int(vals[1]), int(vals[2])
    rest = vals[3:] if pgse else vals[4:]
    nc, res = int(rest[0]), float(rest[1])
    n1, n2, n3 = (int(x) for x in rest[2:5])
    D = np.loadtxt(os.path.join(d, "diffusivity.txt"), ndmin=1)
    T2 = np.loadtxt(os.path.join(d, "T2.txt"), ndmin=1)
    lab = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8).reshape(n1, n2, n3)
    step, t2s, pij, td = pyoracle.reference_tables(dt, res, D, T2, 1000, tn)
    kw = dict(dt=dt, tn=tn, npar=npar, res=res, step=step, t2_steps=t2s, pij=pij, seed=seed, td=td)
    if pgse:
        g = np.loadtxt(os.path.join(d, "gradient_time.txt")).reshape(-1, 6)
        return pyoracle.Job(lab, grad=g, **kw)
    bval = np.loadtxt(os.path.join(d, "bval.txt"), ndmin=1)
    bvec = np.loadtxt(os.path.join(d, "bvec.txt")).reshape(-1, 3)
    return pyoracle.Job(lab, bval=bval, bvec=bvec, **kw)


def fmt15(a):
    """The reference's text form of a double (ostream precision 15)."""
    return np.array(["%.15g" % x for x in np.asarray(a).ravel()])


@pytest.mark.parametrize("case", ["narrow_3comp", "pgse_3comp", "realistic_mito_1", "realistic_undulation_pgse"])
def test_oracle_reproduces_reference_outputs(case, tmp_path):
    d = unpack_golden(case, str(tmp_path))
    job = job_from_dir(d, golden_seed(case))
    o = pyoracle.run_oracle(job)
    files = {"sig0": "sig0.txt", "dx2": "dx2.txt", "dx4": "dx4.txt", "npar_count": "NPar_count.txt"}
    files["sig" if job.mode == pyoracle.MODE_PGSE else "sigre"] = "sig.txt" if job.mode else "sigRe.txt"
    for key, fn in files.items():
        tokens = np.array(open(os.path.join(d, fn)).read().split())
        assert np.array_equal(fmt15(o[key]), tokens), f"{case}: {fn} differs"
    # the outputs exercise every kind of face event
    assert o["npar_count"][-1].sum() == job.npar


def random_job(seed, pgse, nc=3, boundary=0):
    rng = np.random.default_rng(seed)
    lab = geometry.axon_lattice(14, 12, 20, 0.1, seed=seed, exterior=2, r0=0.4)
    lab[: rng.integers(1, 3), :, :] = 0
    D = [0.0, float(rng.uniform(1.5, 2.5)), float(rng.uniform(0.5, 2.5))]
    T2 = [80.0, float(rng.uniform(30, 90)), float(rng.uniform(30, 90))]
    dt, tn = 2e-4, 1000 * int(rng.integers(1, 3))
    step, t2s, pij, td = pyoracle.reference_tables(dt, 0.1, D, T2, 1000, tn)
    kw = dict(dt=dt, tn=tn, npar=48, res=0.1, step=step, t2_steps=t2s, pij=pij,
              seed=int(rng.integers(0, 2**63)), td=td, boundary=boundary)
    if pgse:
        ng = 6
        g = np.column_stack([rng.uniform(0.02, 0.3, ng), rng.uniform(0.01, 0.2, ng),
                             rng.uniform(0.5, 4, ng), rng.normal(size=(ng, 3))])
        g[:, 3:] /= np.linalg.norm(g[:, 3:], axis=1, keepdims=True)
        return pyoracle.Job(lab, grad=g, **kw)
    nb = 5
    bv = rng.normal(size=(nb, 3))
    bv /= np.linalg.norm(bv, axis=1, keepdims=True)
    return pyoracle.Job(lab, bval=rng.uniform(0.2, 3.0, nb), bvec=bv, **kw)


needs_ref = pytest.mark.skipif(not pyoracle.ref_available(), reason="oracle/_ref not built (reference checkout absent)")


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("pgse", [False, True])
def test_oracle_bit_exact_vs_reference_build(seed, pgse):
    job = random_job(seed, pgse)
    ref = pyoracle.run_reference_walkers(job, job.npar, 1)
    ora = pyoracle.run_oracle(job)
    for k in ("sig0", "dx2", "dx4", "npar_count", "sig" if pgse else "sigre"):
        assert np.array_equal(ref[k], ora[k]), k


@needs_ref
def test_reference_threads_reduce_in_fixed_order():
    job = random_job(9, False)
    a = pyoracle.run_reference_walkers(job, job.npar, 3)
    b = pyoracle.run_reference_walkers(job, job.npar, 3)
    for k in ("sig0", "dx2", "dx4", "sigre"):
        assert np.array_equal(a[k], b[k])


def test_oracle_parallel_matches_serial():
    job = random_job(4, True)
    a = pyoracle.run_oracle(job)
    b = pyoracle.run_oracle(job, nthreads=4)
    for k in ("sig0", "dx2", "dx4", "sig"):
        np.testing.assert_allclose(b[k], a[k], rtol=1e-12, atol=1e-12 * np.abs(a[k]).max())
    assert np.array_equal(a["npar_count"], b["npar_count"])


def test_oracle_periodic_conserves_walkers_and_wraps():
    job = random_job(5, False, boundary=pyoracle.BOUNDARY_PERIODIC)
    o = pyoracle.run_oracle(job, trace_walkers=job.npar)
    ev = o["trace"]["events"]
    # wall events (type 1) happen and every record counts every walker
    types = [(ev >> (4 * k + 2)) & 3 for k in range(4)]
    nev = (ev >> 28) & 7
    wall = sum(((t == 1) & (k < nev)).sum() for k, t in enumerate(types))
    assert wall > 0
    assert np.all(o["npar_count"].sum(axis=1) == job.npar)
