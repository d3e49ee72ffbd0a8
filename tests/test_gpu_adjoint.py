"""The adjoint of the waveform-mode signal (rms_adjoint_run, rms_b200.adjoint)
against central finite differences of the forward walk with common random
numbers (the same seed, so the same walkers and draws).

L = sum_j gC_j C_j + gS_j S_j over the normalised signal sums, with seeded
weights.  Bars:
  - waveforms (exact pathwise: the phase is linear in the waveform) and T2
    (analytic): within 1 % of the finite difference;
  - D, pathwise with the events frozen, on impermeable flat membranes
    (parallel planes: reflections are continuous in the step length): within
    1 %;
  - D by time rescaling (rms_adjoint_run's d_diffusivity) on the voxelised
    axon, where the pathwise term misses the jumps at the membrane's
    corners: against the least-squares slope of the loss over D +- 5 % at
    1e6 walkers, within 3 %;
  - the kernel's walker sums against the oracle's FP64 restatement
    (or_adjoint_split) of the same walkers, on flat planes where the FP32 and
    FP64 walks cannot part (reflections and crossings are continuous there);
  - kappa: a Monte Carlo estimate (forced permeation draws; the score
    function beside it), and the finite difference jumps wherever a crossing
    decision flips, so the reference is the least-squares slope of L over
    +-15 %, seven points; both are averaged over 8 seeds and compared within
    their statistical error.
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
    assert abs(r["d_diffusivity_pathwise"] / want - 1) < 0.01, (r["d_diffusivity_pathwise"], want)
    # the time-rescaling estimate is unbiased here too, with more spread
    big = dict(kw, npar=16 * NPAR)
    rb = adj(wave, **big)
    want_b = fd(lambda D: loss(wave, D=D, **big), 2.0, 2e-3)
    assert abs(rb["d_diffusivity"] / want_b - 1) < 0.03, (rb["d_diffusivity"], want_b)


def test_diffusivity_gradient_voxelised_axon_time_rescaling():
    wave = base_waves()
    kw = dict(kappa=0.0, t2=(1e6, 70.0, 70.0), npar=16 * NPAR)
    r = adj(wave, **kw)
    want = slope(lambda D: loss(wave, D=D, **kw), 2.0, 0.05)
    assert abs(r["d_diffusivity"] / want - 1) < 0.03, (r["d_diffusivity"], want)
    assert r["d_diffusivity_pathwise"] / want < 0.6   # the frozen-event term misses the corner jumps


def test_adjoint_sums_equal_the_oracle_walker_set():
    """rms_adjoint_run's gradients against the oracle's FP64 adjoint
    (or_adjoint_split) of the same 4096 walkers and seed, on flat planes
    with partial permeation (kappa = 0.05): every gradient, the loss and the
    signal sums agree to FP32 accuracy."""
    import pyoracle
    wave = base_waves()
    n, D, kap, t2 = 4096, 2.0, 0.05, (1e6, 70.0, 60.0)
    lab = planes()
    sim = make(wave, D=D, kappa=kap, t2=t2, lab=lab, npar=n)
    r = sim.adjoint(WEIGHTS.reshape(-1) / n, seed=5)
    step, t2s, pij, td = pyoracle.reference_tables(DT, RES, [0.0, D, D], list(t2), 100, TN, kappa=kap)
    job = pyoracle.Job(lab, dt=DT, tn=TN, npar=n, res=RES, step=step, t2_steps=t2s, pij=pij, seed=5, timepoints=100,
                       td=td, wave=wave, boundary=pyoracle.BOUNDARY_PERIODIC)
    sums = pyoracle.adjoint_split(job, WEIGHTS.reshape(-1) / n)
    want = pyoracle.adjoint_gradients(job, sums, D, t2, kappa=kap)
    assert sums["E"] != 0.0   # partial permeation draws were made
    np.testing.assert_allclose(r["sigw"], sums["sigw"], rtol=0, atol=1e-4 * n)
    assert r["loss"] == pytest.approx(want["loss"], rel=1e-4, abs=1e-6)
    scale = np.abs(want["d_wave"]).max()
    np.testing.assert_allclose(r["d_wave"], want["d_wave"], rtol=0, atol=1e-3 * scale)
    assert r["d_diffusivity_pathwise"] == pytest.approx(want["d_diffusivity_pathwise"], rel=2e-3), "pathwise D"
    # the score, forced-draw and time-rescaling sums are differences of larger
    # sums: FP32 per walker shows at 1e-3
    for k in ("d_diffusivity", "d_kappa", "d_kappa_score"):
        assert r[k] == pytest.approx(want[k], rel=1e-2), k
    np.testing.assert_allclose(r["d_t2"][:3], want["d_t2"], rtol=2e-3, atol=1e-12)


def test_kappa_gradient_permeable_axon():
    """The kappa gradient (forced draws) against the +-15 % slope of the loss,
    both averaged over 8 seeds (262144 walkers each): on this axon the slope
    is the noisier of the two (crossing decisions flip in jumps; measured on
    the oracle at 65536 walkers: score-function spread ~17 %, slope spread
    ~45 % per seed; the forced draws spread less than the score function).
    The means must agree within 3 standard errors of their difference (from
    the seed spreads) and within 40 %; the forced draws' seed spread must be
    below the score function's."""
    wave = base_waves()
    kw = dict(kappa=0.05, t2=(1e6, 70.0, 70.0), npar=4 * NPAR)
    adjs, scores, slopes = [], [], []
    for seed in range(5, 13):
        sim = make(wave, **kw)
        r = sim.adjoint(WEIGHTS.reshape(-1) / kw["npar"], seed=seed)
        adjs.append(r["d_kappa"])
        scores.append(r["d_kappa_score"])
        sim.close()

        def f(k):
            sk = make(wave, **dict(kw, kappa=k))
            sk.run(seed=seed, precision="split")
            v = float((sk.get("sigw").reshape(-1, 2) * WEIGHTS).sum() / kw["npar"])
            sk.close()
            return v

        slopes.append(slope(f, 0.05, 0.15))
    a, b = np.mean(adjs), np.mean(slopes)
    se = np.sqrt(np.var(adjs, ddof=1) / len(adjs) + np.var(slopes, ddof=1) / len(slopes))
    assert abs(a - b) < 3 * se, (adjs, slopes)
    assert abs(a / b - 1) < 0.4, (a, b)
    assert np.std(adjs) < np.std(scores), (adjs, scores)


def test_jacobian_rows_equal_the_oracle():
    """rms_adjoint_jacobian's rows against the oracle's FP64 adjoint
    (or_adjoint_split) with a unit weight on each signal sum, on flat planes
    with partial permeation (kappa = 0.05), where the FP32 and FP64 walks
    cannot part: D (time rescaling), kappa (forced draws and score function)
    and T2 agree to FP32 accuracy."""
    import pyoracle
    wave = base_waves()
    n, D, kap, t2 = 4096, 2.0, 0.05, (1e6, 70.0, 60.0)
    lab = planes()
    sim = make(wave, D=D, kappa=kap, t2=t2, lab=lab, npar=n)
    J = sim.jacobian(seed=5)
    step, t2s, pij, td = pyoracle.reference_tables(DT, RES, [0.0, D, D], list(t2), 100, TN, kappa=kap)
    job = pyoracle.Job(lab, dt=DT, tn=TN, npar=n, res=RES, step=step, t2_steps=t2s, pij=pij, seed=5, timepoints=100,
                       td=td, wave=wave, boundary=pyoracle.BOUNDARY_PERIODIC)
    for j in range(wave.shape[0]):
        for sk in range(2):
            g = np.zeros((wave.shape[0], 2))
            g[j, sk] = 1.0
            sums = pyoracle.adjoint_split(job, g.reshape(-1))
            want = pyoracle.adjoint_gradients(job, sums, D, t2, kappa=kap)
            for key, col in (("d_diffusivity", "D"), ("d_kappa", "kappa"), ("d_kappa_score", "kappa_score")):
                assert J[col][j, sk] == pytest.approx(want[key], rel=1e-2, abs=1e-5 * n), (j, sk, key)
            np.testing.assert_allclose(J["T2"][j, sk], want["d_t2"], rtol=2e-3, atol=1e-9 * n)


@pytest.mark.parametrize("kappa", [0.05, 0.0])
def test_jacobian_rows_equal_one_hot_adjoints(kappa):
    """rms_adjoint_jacobian's row for each waveform's cos and sin sum equals
    rms_adjoint_run with a unit weight on that sum (the same walkers and
    estimators; only the order of FP32 operations differs), for D, kappa
    (forced draws and score function) and T2; with kappa = 0 no draw is made
    and the kappa columns are 0."""
    wave = base_waves()
    n = 16384
    sim = make(wave, kappa=kappa, npar=n)
    J = sim.jacobian(seed=5)
    for j in range(wave.shape[0]):
        for sk in range(2):
            g = np.zeros((wave.shape[0], 2))
            g[j, sk] = 1.0
            r = sim.adjoint(g.reshape(-1), seed=5)
            assert J["D"][j, sk] == pytest.approx(r["d_diffusivity"], rel=1e-3, abs=1e-6 * n), (j, sk)
            assert J["kappa"][j, sk] == pytest.approx(r["d_kappa"], rel=1e-3, abs=1e-6 * n), (j, sk)
            assert J["kappa_score"][j, sk] == pytest.approx(r["d_kappa_score"], rel=1e-6, abs=1e-9 * n), (j, sk)
            np.testing.assert_allclose(J["T2"][j, sk], r["d_t2"][:3], rtol=1e-6, atol=1e-12 * n)
    np.testing.assert_allclose(J["sigw"], r["sigw"], rtol=1e-12)
    if kappa == 0.0:
        assert not J["kappa"].any() and not J["kappa_score"].any()


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
    # the one-pass Jacobian contracted with the loss weights is the backward pass's gradient
    J = adjoint.signal_jacobian(wave.detach(), 2.0, 0.05, [1e6, 80.0, 60.0], setup)
    Wt = torch.from_numpy(WEIGHTS)
    # the adjoint forms s0 cos(phi) in FP32, the forward walk in FP64
    np.testing.assert_allclose(J["signal"].numpy(), S.detach().numpy(), rtol=1e-5, atol=1e-9)
    assert float((J["D"] * Wt).sum()) == pytest.approx(D.grad.item(), rel=1e-3, abs=1e-9)
    assert float((J["kappa"] * Wt).sum()) == pytest.approx(kap.grad.item(), rel=1e-3, abs=1e-9)
    np.testing.assert_allclose((J["T2"] * Wt[:, :, None]).sum(dim=(0, 1)).numpy(), t2.grad.numpy(), rtol=1e-5,
                               atol=1e-10)


@pytest.mark.parametrize("boundary,shard", [("periodic", None), ("mirror", None), ("periodic", (5000, 16384))])
def test_grouped_forced_walks_equal_the_single_launch(monkeypatch, boundary, shard):
    """The default reverse pass (pass 1 alone, recording the bin displacement
    sums, a_jw, the time-rescaling sums and the checkpoints; dL/dwave reduced
    from the records; then the forced walks grouped by resume step, each from
    its checkpoint) gives the single launch's gradients and Jacobian: the same
    walkers, draws and FP32 walk.  The forced walks and the Jacobian's
    time-rescaling sums are the same FP32 arithmetic (only the FP64 sums'
    order differs); dL/dwave and the weighted time-rescaling sum are summed in
    another order (float).  2000 steps of 20-step bins checkpoint every 480
    steps (5 resume steps); also on a walker shard that does not start at
    walker 0."""
    wave = base_waves()
    n = 16384

    def both(grouped):
        monkeypatch.setenv("RMS_ADJOINT_GROUPED", "1" if grouped else "0")
        sim = engine.Sim(lattice(), dt=DT, tn=TN, npar=n, res=RES, diffusivity=[0.0, 2.0, 2.0],
                         t2=[1e6, 80.0, 60.0], wave=wave, timepoints=100, permeation="kappa", kappa=0.05,
                         boundary=boundary)
        r = sim.adjoint(WEIGHTS.reshape(-1) / n, seed=5, walker_range=shard)
        J = sim.jacobian(seed=5, walker_range=shard)
        sim.close()
        return r, J

    r1, J1 = both(True)
    r0, J0 = both(False)
    assert r0["d_kappa"] != 0.0
    for k in ("loss", "d_diffusivity_pathwise", "d_kappa_score", "d_kappa"):
        assert r1[k] == pytest.approx(r0[k], rel=1e-7, abs=1e-15), k
    assert r1["d_diffusivity"] == pytest.approx(r0["d_diffusivity"], rel=1e-4), "d_diffusivity"
    scale = np.abs(r0["d_wave"]).max()
    np.testing.assert_allclose(r1["d_wave"], r0["d_wave"], rtol=0, atol=1e-5 * scale)
    np.testing.assert_allclose(r1["d_t2"], r0["d_t2"], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(r1["sigw"], r0["sigw"], rtol=1e-12)
    for k in ("D", "kappa", "kappa_score", "T2", "sigw"):
        np.testing.assert_allclose(J1[k], J0[k], rtol=1e-7, atol=1e-12 * n, err_msg=k)


def test_grouped_reverse_pass_without_permeation(monkeypatch):
    """Impermeable membranes (kappa = 0): no forced walks; the records of
    pass 1 still give the single launch's dL/dwave, D and T2 gradients."""
    wave = base_waves()
    n = 16384
    out = []
    for grouped in ("1", "0"):
        monkeypatch.setenv("RMS_ADJOINT_GROUPED", grouped)
        sim = make(wave, kappa=0.0, npar=n)
        out.append((sim.adjoint(WEIGHTS.reshape(-1) / n, seed=5), sim.jacobian(seed=5)))
        sim.close()
    (r1, J1), (r0, J0) = out
    assert r1["d_kappa"] == 0.0 and r0["d_kappa"] == 0.0
    assert r1["d_diffusivity"] == pytest.approx(r0["d_diffusivity"], rel=1e-4)
    scale = np.abs(r0["d_wave"]).max()
    np.testing.assert_allclose(r1["d_wave"], r0["d_wave"], rtol=0, atol=1e-5 * scale)
    for k in ("D", "T2", "sigw"):
        np.testing.assert_allclose(J1[k], J0[k], rtol=1e-7, atol=1e-12 * n, err_msg=k)


def test_timing_reports_the_reverse_pass_on_a_fresh_simulation():
    """rms_sim_last_timing after an adjoint call on a simulation that has not
    run forward: the reverse pass's device time, positive."""
    sim = make(base_waves(), npar=4096)
    sim.adjoint(WEIGHTS.reshape(-1) / 4096, seed=5)
    walk_ms, run_ms = sim.timing()
    assert walk_ms > 0.0 and run_ms > 0.0
    sim.close()


def test_reverse_pass_in_walker_chunks_equals_one_chunk(monkeypatch):
    """200000 walkers with the scratch capped at 130 MiB against one chunk.
    Records per walker: 1936 bytes for the weighted form (100 bins x 3
    floats, a_jw, 4 checkpoints, the summary and bucket entries) -- chunks of
    70,400, 70,400 and 59,200 walkers; 720 bytes for the Jacobian -- 189,312
    and 10,688.  The chunks' sums add up to the whole run's gradients and
    Jacobian (float and FP64 sums in another order only)."""
    wave = base_waves()
    n = 200000

    def run(cap):
        if cap:
            monkeypatch.setenv("RMS_ADJOINT_SCRATCH_MB", str(cap))
        else:
            monkeypatch.delenv("RMS_ADJOINT_SCRATCH_MB", raising=False)
        sim = make(wave, npar=n)
        r = sim.adjoint(WEIGHTS.reshape(-1) / n, seed=5)
        J = sim.jacobian(seed=5)
        sim.close()
        return r, J

    r1, J1 = run(130)
    r0, J0 = run(0)
    for k in ("loss", "d_diffusivity_pathwise", "d_kappa_score", "d_kappa"):
        assert r1[k] == pytest.approx(r0[k], rel=1e-7, abs=1e-15), k
    assert r1["d_diffusivity"] == pytest.approx(r0["d_diffusivity"], rel=1e-5), "d_diffusivity"
    scale = np.abs(r0["d_wave"]).max()
    np.testing.assert_allclose(r1["d_wave"], r0["d_wave"], rtol=0, atol=1e-5 * scale)
    np.testing.assert_allclose(r1["d_t2"], r0["d_t2"], rtol=1e-9, atol=1e-15)
    for k in ("D", "kappa", "kappa_score", "T2", "sigw"):
        np.testing.assert_allclose(J1[k], J0[k], rtol=1e-7, atol=1e-12 * n, err_msg=k)
