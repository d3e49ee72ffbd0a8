"""Alternative membrane rules (reject, leap) in the split walk on the GPU
against the oracle's FP64 replay with the same rule and streams (D(t) within
0.5 %, K(t) within 2 %, counts within 1 % -- the split walk's bar), and the
reflecting rule unchanged by their presence."""
import numpy as np
import pytest

import pyoracle
from rms_b200 import analysis, engine, geometry

pytestmark = pytest.mark.gpu


def check(got, want):
    Dg, Kg = analysis.axis_dk(got["sig0"], got["dx2"], got["dx4"], got["td"])
    Dw, Kw = analysis.axis_dk(want["sig0"], want["dx2"], want["dx4"], got["td"])
    sl = slice(20, None)
    assert np.abs(Dg[sl] / Dw[sl] - 1).max() < 0.005
    assert (np.abs(Kg[sl] - Kw[sl]) / np.maximum(np.abs(Kw[sl]), 1.0)).max() < 0.02


@pytest.mark.parametrize("rule", ["reject", "leap"])
@pytest.mark.parametrize("geom", ["planes", "axon"])
def test_rule_matches_fp64_replay(rule, geom):
    if geom == "planes":
        lab = np.full((24, 8, 8), 2, dtype=np.uint8)
        lab[6:12] = 1
        lab[18:24] = 1
        kappa = 0.0
    else:
        lab = geometry.axon_lattice(16, 16, 24, 0.1, seed=2, exterior=2, r0=0.45)
        kappa = 0.05
    n, tn = 16384, 2000
    kw = dict(dt=2e-4, tn=tn, npar=n, res=0.1, diffusivity=[0, 2.0, 2.0], t2=[1e6, 80.0, 60.0],
              bval=[], bvec=np.zeros((0, 3)), timepoints=100, boundary="periodic", permeation="kappa", kappa=kappa)
    sim = engine.Sim(lab, rule=rule, **kw)
    got = sim.run(seed=3, precision="split").outputs()
    step, t2s, _, td = pyoracle.reference_tables(2e-4, 0.1, [0, 2.0, 2.0], [1e6, 80.0, 60.0], 100, tn)
    job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=n, res=0.1, step=step, t2_steps=t2s, pij=sim.get("pij"), seed=3,
                       td=td, timepoints=100, boundary=1, rule={"reject": 1, "leap": 2}[rule])
    want = pyoracle.run_oracle(job, nthreads=8, split=True)
    check(got, want)
    assert np.abs(got["npar_count"] - want["npar_count"]).max() <= 0.01 * n
    np.testing.assert_allclose(got["sig0"], want["sig0"], rtol=1e-5)
    # the reflecting walk of the same job differs (the rule is in effect)
    ref = engine.Sim(lab, **kw).run(seed=3, precision="split").outputs()
    assert not np.array_equal(ref["dx2"], got["dx2"])


def test_compat_refuses_other_rules():
    lab = np.ones((8, 8, 8), dtype=np.uint8)
    sim = engine.Sim(lab, dt=2e-4, tn=100, npar=64, res=0.1, diffusivity=[0, 2.0], t2=[80, 80],
                     bval=[], bvec=np.zeros((0, 3)), timepoints=10, rule="reject")
    with pytest.raises(engine.RmsError):
        sim.run(precision="compat")
