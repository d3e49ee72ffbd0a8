"""The split-precision walk (RMS_PREC_SPLIT) on the GPU, through the C ABI.

Its error is stated against an FP64 single-walker replay (the oracle's
or_run_split): the same algorithm fed the same random streams, every quantity
after the start position in FP64.  Bar (the engine's stated tolerance):
D(t) within 0.5 % and K(t) within 2 % (absolute 0.02 where |K| < 1) of the
replay, compartment counts conserved, signals within 2e-3 of S0.

The FP32 and FP64 walks are the same walk until a face decision falls within
the FP32 position error of a tie; such a walker then takes another branch and
decorrelates (measured: 6 of 400 walkers within 2000 steps in the thin-axon
lattice below, walker by walker; with partial permeation a step that reaches a
membrane in one precision and not in the other also shifts that walker's
permeation draws).  The fourth moment feels those few walkers, and their share
of a difference of sums falls as 1/sqrt(N): the permeable narrow-pulse case
uses 65536 walkers (16384 put one record of one axis at 2.2 % in K), the
others 16384.
"""
import numpy as np
import pytest

import pyoracle
from rms_b200 import analysis, engine, geometry

pytestmark = pytest.mark.gpu


def lattice3(seed=1, shape=(16, 16, 24), r0=0.45):
    lab = geometry.axon_lattice(*shape, 0.1, seed=seed, exterior=2, r0=r0)
    lab[:2, :, :] = 0
    return lab


def jobs(lab, D, T2, *, npar, tn, seed, boundary="mirror", bval=None, bvec=None, grad=None,
         permeation="reference", kappa=0.0):
    kw = dict(dt=2e-4, tn=tn, npar=npar, res=0.1, diffusivity=D, t2=T2, boundary=boundary,
              permeation=permeation, kappa=kappa)
    if grad is not None:
        kw["grad"] = grad
    else:
        kw["bval"], kw["bvec"] = bval, bvec
    sim = engine.Sim(lab, **kw)
    step, t2s, _, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, 1000, tn)
    job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=npar, res=0.1, step=step, t2_steps=t2s,
                       pij=sim.get("pij"), seed=seed, td=td, boundary=1 if boundary == "periodic" else 0,
                       bval=bval, bvec=bvec, grad=grad)
    return sim, job


def check_dk(got, want, what):
    Dg, Kg = analysis.axis_dk(got["sig0"], got["dx2"], got["dx4"], got["td"])
    Dw, Kw = analysis.axis_dk(want["sig0"], want["dx2"], want["dx4"], got["td"])
    sl = slice(50, None)
    dD = np.abs(Dg[sl] / Dw[sl] - 1).max()
    assert dD < 0.005, f"{what}: D(t) differs by {dD:.2e}"
    dK = np.abs(Kg[sl] - Kw[sl]) / np.maximum(np.abs(Kw[sl]), 1.0)
    assert dK.max() < 0.02, f"{what}: K(t) differs by {dK.max():.2e}"
    return dD, dK.max()


def test_split_vs_fp64_replay_permeable_narrow():
    rng = np.random.default_rng(3)
    bv = rng.normal(size=(6, 3)); bv /= np.linalg.norm(bv, axis=1, keepdims=True)
    b = np.array([0.5, 1, 1.5, 2, 2.5, 3.0])
    n = 65536
    sim, job = jobs(lattice3(), [0, 2.0, 1.0], [80, 80, 40], npar=n, tn=2000, seed=17, bval=b, bvec=bv)
    got = sim.run(seed=17, precision="split").outputs()
    want = pyoracle.run_oracle(job, nthreads=8, split=True)
    check_dk(got, want, "narrow")
    assert np.array_equal(got["npar_count"].sum(axis=1), np.full(1000, float(n)))
    assert np.abs(got["npar_count"] - want["npar_count"]).max() <= 0.01 * n
    np.testing.assert_allclose(got["sig0"], want["sig0"], rtol=1e-5)
    S, Sw = got["sigre"] / got["sig0"][:, None], want["sigre"] / want["sig0"][:, None]
    assert np.abs(S - Sw).max() < 2e-3


def test_split_vs_fp64_replay_pgse_kappa_periodic():
    rng = np.random.default_rng(4)
    ng = 24
    g = np.column_stack([rng.choice([0.1, 0.2], ng), rng.choice([0.05, 0.1], ng),
                         rng.uniform(0.5, 4, ng), rng.normal(size=(ng, 3))])
    g[:, 3:] /= np.linalg.norm(g[:, 3:], axis=1, keepdims=True)
    sim, job = jobs(lattice3(5), [0, 2.0, 2.0], [80, 70, 50], npar=16384, tn=2000, seed=23, grad=g,
                    boundary="periodic", permeation="kappa", kappa=0.05)
    got = sim.run(seed=23, precision="split").outputs()
    want = pyoracle.run_oracle(job, nthreads=8, split=True)
    check_dk(got, want, "pgse")
    assert np.abs(got["sig"] / got["sig0"][-1] - want["sig"] / want["sig0"][-1]).max() < 2e-3


def test_launch_variants_walk_the_same_walkers():
    lab = lattice3(2)
    sim = engine.Sim(lab, dt=2e-4, tn=1000, npar=20000, res=0.1, diffusivity=[0, 2.0, 1.0],
                     t2=[80, 80, 40], bval=[1.0], bvec=[[1, 0, 0]])
    base = sim.run(seed=5, precision="split", variant=1).outputs()
    for k, block, minb in engine.split_variants()[1:]:
        o = sim.run(seed=5, precision="split", variant=k).outputs()
        assert np.array_equal(o["npar_count"], base["npar_count"]), (k, block, minb)
        np.testing.assert_allclose(o["dx2"], base["dx2"], rtol=1e-9, atol=1e-12)


def test_split_statistically_equals_compat():
    """Independent samples (different streams): late-time D and K agree
    within Monte Carlo error (1e5 walkers)."""
    lab = geometry.axon_lattice(32, 32, 64, 0.1, seed=9, exterior=2, r0=1.0)
    kw = dict(dt=2e-4, tn=4000, npar=100000, res=0.1, diffusivity=[0, 2.0, 1.0], t2=[80, 80, 40],
              bval=[], bvec=np.zeros((0, 3)))
    o_c = engine.Sim(lab, **kw).run(seed=1, precision="compat").outputs()
    o_s = engine.Sim(lab, **kw).run(seed=2, precision="split").outputs()
    Dc, Kc = analysis.axis_dk(o_c["sig0"], o_c["dx2"], o_c["dx4"], o_c["td"])
    Ds, Ks = analysis.axis_dk(o_s["sig0"], o_s["dx2"], o_s["dx4"], o_s["td"])
    late = slice(500, None)
    assert np.abs(Ds[late].mean(0) / Dc[late].mean(0) - 1).max() < 0.01
    assert np.abs(Ks[late].mean(0) - Kc[late].mean(0)).max() < 0.05
    np.testing.assert_allclose(o_s["sig0"], o_c["sig0"], rtol=0.01)
