"""The adjoint of the waveform-mode signal (rms_adjoint_run, rms_b200.adjoint)
against central finite differences of the forward walk with common random
numbers (the same seed, so the same walkers and draws).

L = sum_j gC_j C_j + gS_j S_j over the normalised signal sums, with seeded
weights.  Bars:
  - waveforms (exact pathwise: the phase is linear in the waveform) and T2
    (analytic): within 1 % of the finite difference;
  - D with impermeable flat membranes (parallel planes: reflections are
    continuous in the step length): within 1 %;
  - kappa: a score-function (Monte Carlo) estimate, and the finite difference
    jumps wherever a crossing decision flips, so the reference is the
    least-squares slope of L over +-15 %, seven points, and the bar 20 %.
Walls are periodic.  Two places where the walk's output is not continuous in
the step length, so the frozen-event D term misses jumps: a mirror wall (the
reference mirrors the origin image, hpc_code/lib/main.cu:302-310, so a
displacement component jumps from -x0 to +x0) and the convex corners of a
voxelised membrane (a trajectory either strikes the face or passes the
corner).  With permeable membranes, a changed step length also changes which
steps reach a membrane and so which permeation draws are made.  The D test
therefore uses impermeable flat membranes.
"""
import numpy as np
import pytest

from rms_b200 import engine, geometry, waveforms

pytestmark = pytest.mark.gpu

DT, TN, NB, NPAR, RES = 5e-4, 2000, 100, 65536, 0.1


def lattice():
    return geometry.axon_lattice(24, 24, 48, RES, seed=4, exterior=2, r0=0.6)


def base_waves(nw=4, seed=2):
    w = waveforms.random_smooth(nw, NB, 1.0, seed=seed)
    return waveforms.scale_to_b(w, DT * TN / NB, np.linspace(0.3, 1.2, nw))


def planes():
    lab = np.full((24, 12, 12), 2, dtype=np.uint8)
    lab[(np.arange(24) // 6) % 2 == 0] = 1
    return lab


def make(wave, D=2.0, kappa=0.05, t2=(1e6, 80.0, 60.0), lab=None, npar=NPAR):
    return engine.Sim(lattice() if lab is None else lab, dt=DT, tn=TN, npar=npar, res=RES, diffusivity=[0.0, D, D],
                      t2=list(t2), wave=wave, timepoints=100, permeation="kappa", kappa=kappa, boundary="periodic")


WEIGHTS = np.random.default_rng(11).normal(size=(4, 2))


def loss(wave, npar=NPAR, **kw):
    sim = make(wave, npar=npar, **kw)
    sim.run(seed=5, precision="split")
    return float((sim.get("sigw").reshape(-1, 2) * WEIGHTS).sum() / npar)


def adj(wave, npar=NPAR, **kw):
    return make(wave, npar=npar, **kw).adjoint(WEIGHTS.reshape(-1) / npar, seed=5)


def fd(f, x, h):
    return (f(x + h) - f(x - h)) / (2 * h)


def slope(f, x, rel):
    xs = x * (1 + rel * np.linspace(-1, 1, 7))
    return np.polyfit(xs, [f(v) for v in xs], 1)[0]


def test_adjoint_forward_matches_the_walk():
    wave = base_waves()
    sim = make(wave)
    sim.run(seed=5, precision="split")
    r = sim.adjoint(WEIGHTS.reshape(-1) / NPAR, seed=5)
    np.testing.assert_allclose(r["sigw"] / NPAR, sim.get("sigw").reshape(-1, 2) / NPAR, atol=2e-4)
    assert abs(r["loss"] - loss(wave)) < 2e-4


def test_waveform_gradient_matches_finite_difference():
    wave = base_waves()
    r = adj(wave)
    d = np.random.default_rng(3).normal(size=wave.shape) * np.abs(wave).max()
    want = fd(lambda t: loss(wave + t * d), 0.0, 1e-3)
    got = float((r["d_wave"] * d).sum())
    assert abs(got / want - 1) < 0.01, (got, want)


@pytest.mark.parametrize("c", [1, 2])
def test_t2_gradient_matches_finite_difference(c):
    wave = base_waves()
    t2 = np.array([1e6, 80.0, 60.0])
    r = adj(wave, t2=tuple(t2))

    def f(x):
        tt = t2.copy()
        tt[c] = x
        return loss(wave, t2=tuple(tt))

    want = fd(f, t2[c], 1e-3 * t2[c])
    assert abs(r["d_t2"][c] / want - 1) < 0.01, (r["d_t2"][c], want)


def test_diffusivity_gradient_impermeable_planes():
    wave = base_waves()
    kw = dict(kappa=0.0, t2=(1e6, 70.0, 70.0), lab=planes())
    r = adj(wave, **kw)
    want = fd(lambda D: loss(wave, D=D, **kw), 2.0, 2e-3)
    assert abs(r["d_diffusivity"] / want - 1) < 0.01, (r["d_diffusivity"], want)


def test_kappa_gradient_permeable_axon():
    # score-function spread over seeds at 65536 walkers was ~6 % here; 4x the
    # walkers halves it
    wave = base_waves()
    kw = dict(kappa=0.05, t2=(1e6, 70.0, 70.0), npar=4 * NPAR)
    r = adj(wave, **kw)
    want = slope(lambda k: loss(wave, **dict(kw, kappa=k)), 0.05, 0.15)
    assert abs(r["d_kappa"] / want - 1) < 0.2, (r["d_kappa"], want)


def test_torch_autograd_through_rotations():
    import torch
    from rms_b200 import adjoint
    g0 = base_waves(1)[0]                                   # [nbins, 3]
    R = torch.from_numpy(np.stack([np.linalg.qr(np.random.default_rng(k).normal(size=(3, 3)))[0]
                                   for k in range(4)]))
    setup = adjoint.WalkSetup(lattice(), DT, TN, NPAR, RES, seed=5, timepoints=100, boundary="periodic")
    g = torch.tensor(g0, requires_grad=True)
    D = torch.tensor(2.0, dtype=torch.float64, requires_grad=True)
    kap = torch.tensor(0.05, dtype=torch.float64, requires_grad=True)
    t2 = torch.tensor([1e6, 80.0, 60.0], dtype=torch.float64, requires_grad=True)
    wave = torch.einsum("jab,nb->jna", R, g)
    S = adjoint.waveform_signal(wave, D, kap, t2, setup)
    L = (S * torch.from_numpy(WEIGHTS)).sum()
    L.backward()
    assert abs(L.item() - loss(wave.detach().numpy())) < 1e-9
    d = np.random.default_rng(8).normal(size=g0.shape) * np.abs(g0).max()
    Rn = R.numpy()
    want = fd(lambda t: loss(np.einsum("jab,nb->jna", Rn, g0 + t * d)), 0.0, 1e-3)
    got = float((g.grad.numpy() * d).sum())
    assert abs(got / want - 1) < 0.01, (got, want)
    assert t2.grad.shape == (3,) and np.isfinite(D.grad.item()) and np.isfinite(kap.grad.item())
