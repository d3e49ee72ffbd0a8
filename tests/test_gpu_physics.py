"""Analytic limits on the GPU (the third oracle).

 - free diffusion: D(t) = D0; K(t) = -1.2/n for n fixed-length isotropic
   steps (per axis <x^2> = s^2/3, <x^4> = s^4/5 per step);
 - one compartment: sig0 = N exp(-t/T2) exactly;
 - narrow pulse and PGSE in free space: S/S0 = exp(-b D0),
   b = |g|^2 delta^2 (Delta - delta/3) (analysis/readRMS_pgse.m:53);
 - impermeable parallel planes a apart: D_parallel = D0 and
   D_perp -> a^2 / (12 t) (part2_demo1_2_diffusivity.m fits a_eff this way).

The signal tests use periodic walls: under the reference's mirror walls the
displacement is taken against the mirrored origin (hpc_code/lib/main.cu:302-310),
so each wall hit flips the sign of that axis's displacement -- harmless for the
even moments, not for the phase once walkers reach the lattice edge.
"""
import numpy as np
import pytest

from rms_b200 import analysis, engine

pytestmark = pytest.mark.gpu
PRECISIONS = ["compat", "split"]


def free_sim(npar, tn, D0=2.0, T2=1e9, shape=(32, 32, 32), **kw):
    lab = np.ones(shape, dtype=np.uint8)
    return engine.Sim(lab, dt=2e-4, tn=tn, npar=npar, res=0.1, diffusivity=[0, D0],
                      t2=[80.0, T2], **kw)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_free_diffusion_moments(precision):
    N, tn = 40000, 2000
    sim = free_sim(N, tn, bval=[], bvec=np.zeros((0, 3)))
    o = sim.run(seed=123, precision=precision).outputs()
    D, K = analysis.axis_dk(o["sig0"], o["dx2"], o["dx4"], o["td"])
    n = np.arange(1000) * (tn // 1000) + 1
    sl = slice(200, None)
    assert np.abs(D[sl] / 2.0 - 1).max() < 0.04
    assert abs(D[sl].mean() / 2.0 - 1) < 0.01
    k_expect = -1.2 / n[sl, None]
    assert np.abs(K[sl] - k_expect).mean() < 0.05
    # first record: one step of exactly sqrt(6 D0 dt) length
    r2 = o["dx2"][0, 0] + o["dx2"][0, 3] + o["dx2"][0, 5]
    assert r2 / N == pytest.approx(6 * 2.0 * 2e-4, rel=1e-9 if precision == "compat" else 1e-6)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_sig0_is_t2_decay(precision):
    N, tn, T2 = 2000, 1000, 30.0
    sim = free_sim(N, tn, T2=T2, bval=[1.0], bvec=[[1, 0, 0]])
    o = sim.run(seed=5, precision=precision).outputs()
    want = N * np.exp(-o["td"] / T2)
    np.testing.assert_allclose(o["sig0"], want, rtol=1e-6 if precision == "split" else 1e-12)
    assert np.all(o["npar_count"][:, 1] == N)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_narrow_pulse_free_signal(precision):
    N, tn = 40000, 2000
    b = np.array([0.2, 0.5, 1.0, 1.5])
    sim = free_sim(N, tn, bval=b, bvec=np.tile([[0.0, 0.6, 0.8]], (4, 1)), boundary="periodic")
    o = sim.run(seed=77, precision=precision).outputs()
    S = o["sigre"] / o["sig0"][:, None]
    # standard error of a mean of cosines over 4e4 walkers is below 0.004
    assert np.abs(S[500:].mean(axis=0) - np.exp(-b * 2.0)).max() < 0.015


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pgse_free_signal(precision):
    N, tn, dt = 40000, 4000, 2e-4
    Delta, delta = 0.5, 0.2
    bv = np.array([0.2, 0.5, 1.0, 2.0])
    g = analysis.pgse_gradient_for_b(bv, Delta, delta)
    grad = np.column_stack([np.full(4, Delta), np.full(4, delta), g, np.tile([0.0, 0.0, 1.0], (4, 1))])
    sim = free_sim(N, tn, grad=grad, boundary="periodic")
    o = sim.run(seed=31, precision=precision).outputs()
    S = o["sig"] / N
    # discrete-time b: sum over the lobe steps, as the walk accumulates phase
    assert np.abs(S - np.exp(-bv * 2.0)).max() < 0.015


@pytest.mark.parametrize("precision", PRECISIONS)
def test_parallel_planes(precision):
    # label 1 slab, 8 voxels thick in x, between impermeable null layers
    a_vox, res = 8, 0.1
    lab = np.zeros((a_vox + 2, 24, 24), dtype=np.uint8)
    lab[1:1 + a_vox] = 1
    N, tn = 20000, 10000
    sim = engine.Sim(lab, dt=2e-4, tn=tn, npar=N, res=res, diffusivity=[0, 2.0], t2=[80, 1e9],
                     bval=[], bvec=np.zeros((0, 3)))
    o = sim.run(seed=4, precision=precision).outputs()
    D, _ = analysis.axis_dk(o["sig0"], o["dx2"], o["dx4"], o["td"])
    t = o["td"]
    a = a_vox * res
    assert abs(D[300:, 1:].mean() / 2.0 - 1) < 0.02          # parallel: free
    late = slice(800, None)
    np.testing.assert_allclose(D[late, 0], a * a / (12 * t[late]), rtol=0.08)


def test_library_cumulants_match_the_readrms_restatement():
    from rms_b200 import analysis
    lab = np.ones((20, 20, 20), dtype=np.uint8)
    sim = engine.Sim(lab, dt=2e-4, tn=2000, npar=20000, res=0.1, diffusivity=[0, 2.0], t2=[1e6, 1e6],
                     bval=[], bvec=np.zeros((0, 3)), boundary="periodic")
    o = sim.run(seed=3, precision="split").outputs()
    D, K = sim.cumulants()
    Dw, Kw = analysis.axis_dk(o["sig0"], o["dx2"], o["dx4"], o["td"])
    np.testing.assert_allclose(D[1:], Dw[1:], rtol=1e-12)
    np.testing.assert_allclose(K[5:], Kw[5:], rtol=1e-9, atol=1e-12)
    n = np.array([[0.6, 0.8, 0.0], [0.0, 0.6, 0.8]])
    Dn, Kn = sim.cumulants(n)
    dx2t, dx4t = analysis.normalized_moments(o["sig0"], o["dx2"], o["dx4"])
    Kr, Dr = analysis.akc_mom(dx2t, dx4t, o["td"], n)
    np.testing.assert_allclose(Dn[1:], Dr[1:], rtol=1e-12)
    np.testing.assert_allclose(abs(Dn[-1] / 2.0 - 1).max(), 0, atol=0.02)


def test_gpu_tube_lattice_equals_the_host_builder():
    import time
    from rms_b200 import geometry
    for shp, ext in (((64, 64, 512), 0), ((96, 80, 200), 2)):
        host = geometry.axon_lattice(*shp, 0.1, seed=5, exterior=ext)
        sim = engine.Sim(shape=shp, dt=2e-4, tn=1000, npar=2000, res=0.1, diffusivity=[0, 2.0, 2.0],
                         t2=[80, 80, 60], bval=[], bvec=np.zeros((0, 3)))
        r2, cx, cy = geometry.axon_slices(*shp, 0.1, seed=5)
        sim.set_tube_lattice(r2, cx, cy, inside=1, outside=ext)
        a = sim.run(seed=1, precision="split").outputs()
        ref = engine.Sim(host, dt=2e-4, tn=1000, npar=2000, res=0.1, diffusivity=[0, 2.0, 2.0],
                         t2=[80, 80, 60], bval=[], bvec=np.zeros((0, 3)))
        b = ref.run(seed=1, precision="split").outputs()
        # the same lattice: the same walk (FP64 totals up to their summation order)
        np.testing.assert_allclose(a["dx2"], b["dx2"], rtol=1e-12, atol=1e-300)
        np.testing.assert_array_equal(a["npar_count"], b["npar_count"])
