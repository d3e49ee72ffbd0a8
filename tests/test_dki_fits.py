"""DKI fits of a signal table (rms_dki_shell, rms_dki_lls, rms_akc_shell,
rms_akc_lls): host functions of the library, checked on the CPU.

  - on a signal that follows the DKI model exactly, both fits recover the
    model's directional D(n) and K(n) at directions outside the table;
  - on noisy signals the library equals the numpy restatement of
    analysis/readRMS.m (rms_b200.analysis) to 1e-9;
  - rank-deficient tables give MATLAB's basic solution, as the restatement's
    LAPACK pivoted QR does.
"""
import numpy as np
import pytest

from rms_b200 import analysis, engine


def fib_dirs(n):
    """n unit vectors spread over the sphere (golden-angle spiral)."""
    k = np.arange(n) + 0.5
    z = 1.0 - 2.0 * k / n
    phi = np.pi * (3.0 - np.sqrt(5.0)) * k
    r = np.sqrt(1.0 - z * z)
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def model(seed=0):
    """A diffusion tensor D and fourth-order coefficients w (D_cnt / W_cnt
    multiplicities as readRMS.m): D(n) = n.D.n, D(n)^2 K(n) = sum W_cnt w n4."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    D = q @ np.diag([2.0, 1.2, 0.6]) @ q.T
    d6 = D[analysis.D_IND[:, 0], analysis.D_IND[:, 1]]
    w = rng.uniform(0.1, 0.6, size=15) * np.array([1, .2, .2, .4, .2, .4, .2, .2, .2, .2, 1, .2, .4, .2, 1])
    return d6, w


def dn_kn(d6, w, n):
    Dn = analysis.ndir2(n) @ (analysis.D_CNT * d6)
    Wn = analysis.ndir4(n) @ (analysis.W_CNT * w)
    return Dn, Wn / Dn ** 2


def table(ndirs=30, bvals=(0.5, 1.0, 1.5, 2.0)):
    dirs = fib_dirs(ndirs)
    bvec = np.repeat(dirs, len(bvals), axis=0)
    bval = np.tile(np.asarray(bvals), ndirs)
    return bvec, bval


def model_signal(d6, w, bvec, bval, T):
    Dn, Kn = dn_kn(d6, w, bvec)
    logS = -bval * Dn + bval ** 2 * Dn ** 2 * Kn / 6.0
    return np.tile(np.exp(logS), (T, 1))


def test_shell_fit_recovers_the_model():
    d6, w = model(1)
    bvec, bval = table()
    td = np.array([5.0, 10.0, 20.0])
    sig = model_signal(d6, w, bvec, bval, 3)
    dt = engine.dki_shell(sig, bvec, bval, td)
    probe = fib_dirs(7)[[0, 3, 6]] @ np.linalg.qr(np.random.default_rng(3).normal(size=(3, 3)))[0]
    K, D = engine.akc_shell(dt, probe, td)
    Dw, Kw = dn_kn(d6, w, probe)
    np.testing.assert_allclose(D, np.tile(Dw, (3, 1)), rtol=1e-9)
    np.testing.assert_allclose(K, np.tile(Kw, (3, 1)), rtol=1e-8)
    # <x^2> tensor = 2 t D with multiplicities folded in (n2 carries none)
    np.testing.assert_allclose(dt[:, :6], 2.0 * td[:, None] * analysis.D_CNT * d6, rtol=1e-9)


def test_lls_fit_recovers_the_model():
    d6, w = model(2)
    bvec, bval = table(bvals=(1.0, 2.0, 2.5))
    sig = model_signal(d6, w, bvec, bval, 2)
    # b = 0 rows with a zero direction, as scanners write them (normalised to 0 / 1)
    bvec = np.vstack([np.zeros((2, 3)), bvec])
    bval = np.concatenate([[0.0, 0.0], bval])
    sig = np.hstack([np.ones((2, 2)), sig])
    dt = engine.dki_lls(sig, bvec, bval)
    np.testing.assert_allclose(dt[:, :6], np.tile(d6, (2, 1)), rtol=1e-8, atol=1e-12)
    np.testing.assert_allclose(dt[:, 6:], np.tile(w, (2, 1)), rtol=1e-7, atol=1e-10)
    probe = fib_dirs(5)
    K, D = engine.akc_lls(dt, probe * 3.0)       # directions need not be unit
    Dw, Kw = dn_kn(d6, w, probe)
    np.testing.assert_allclose(D[0], Dw, rtol=1e-8)
    np.testing.assert_allclose(K[0], Kw, rtol=1e-7)


@pytest.mark.parametrize("intercept", [False, True])
def test_shell_fit_equals_the_numpy_restatement(intercept):
    d6, w = model(4)
    # with the intercept (PGSE), each b-value appears twice per direction
    # (two diffusion times): more rows per direction than distinct b-values
    bvec, bval = table(ndirs=20, bvals=(0.5, 1.0, 2.0, 0.5, 1.0, 2.0) if intercept else (0.5, 1.0, 2.0))
    rng = np.random.default_rng(5)
    T = 6
    sig = model_signal(d6, w, bvec, bval, T) * (1.0 + 0.02 * rng.normal(size=(T, bval.size)))
    # shuffle the measurements: the fit groups rows by direction, in any order
    p = rng.permutation(bval.size)
    sig, bvec, bval = sig[:, p], bvec[p], bval[p]
    td = np.linspace(2.0, 30.0, T)
    got = engine.dki_shell(sig, bvec, bval, td, intercept=intercept)
    want = analysis.dki_shell(sig, bvec, bval, td, intercept=intercept)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
    n = fib_dirs(9)
    for a, b in zip(engine.akc_shell(got, n, td), analysis.akc_shell(want, n, td)):
        np.testing.assert_allclose(a, b, rtol=1e-8)


def test_lls_fit_equals_the_numpy_restatement():
    d6, w = model(6)
    bvec, bval = table(ndirs=32, bvals=(1.0, 2.0, 3.0))
    rng = np.random.default_rng(7)
    sig = model_signal(d6, w, bvec, bval, 4) * (1.0 + 0.01 * rng.normal(size=(4, bval.size)))
    got = engine.dki_lls(sig, bvec, bval)
    want = analysis.dki_lls(sig, bvec, bval)
    np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12 * np.abs(want).max())
    n = fib_dirs(6)
    for a, b in zip(engine.akc_lls(got, n), analysis.akc_lls(want, n)):
        np.testing.assert_allclose(a, b, rtol=1e-8)


def test_rank_deficient_tables_give_matlabs_basic_solution():
    """A \\ y on a rank-deficient A is the basic solution of QR with column
    pivoting (what MATLAB returns, with a warning); the library equals the
    LAPACK-based restatement on such tables."""
    d6, w = model(0)
    rng = np.random.default_rng(8)
    cases = [
        # 10 directions: 15 fourth-order elements from 10 equations (m < n)
        table(ndirs=10),
        # one b-value more in one direction than the others measure
        (lambda bv: (bv[0], np.where(np.arange(bv[1].size) == 0, 3.0, bv[1])))(table(ndirs=20, bvals=(1.0, 2.0))),
    ]
    for bvec, bval in cases:
        sig = model_signal(d6, w, bvec, bval, 2) * (1.0 + 0.01 * rng.normal(size=(2, bval.size)))
        got = engine.dki_shell(sig, bvec, bval, [5.0, 10.0])
        want = analysis.dki_shell(sig, bvec, bval, [5.0, 10.0])
        np.testing.assert_allclose(got, want, rtol=1e-8, atol=1e-10 * np.abs(want).max())
    # one b-shell: exact dependencies among the 21 columns, with ties in the
    # pivot choice, so which basic solution comes out is the implementation's;
    # it is a least-squares solution with at most rank-many nonzeros
    bvec, bval = table(ndirs=30, bvals=(1.0,))
    sig = model_signal(d6, w, bvec, bval, 1) * (1.0 + 0.01 * rng.normal(size=(1, bval.size)))
    dt = engine.dki_lls(sig, bvec, bval)[0]
    a = np.concatenate([-(bval[:, None] * analysis.ndir2(bvec)) * analysis.D_CNT,
                        (bval[:, None] ** 2 / 6.0 * analysis.ndir4(bvec)) * analysis.W_CNT], axis=1)
    y = np.log(sig[0] + analysis.EPS)
    best = np.linalg.lstsq(a, y, rcond=None)[0]
    assert abs(np.linalg.norm(a @ dt - y) - np.linalg.norm(a @ best - y)) < 1e-10
    assert np.count_nonzero(dt) <= np.linalg.matrix_rank(a) < 21


def test_bad_tables_are_errors():
    d6, w = model(0)
    bvec, bval = table(ndirs=20, bvals=(1.0,))
    with pytest.raises(engine.RmsError) as e:      # one b-value: no K (the reference indexes past X)
        engine.dki_shell(model_signal(d6, w, bvec, bval, 1), bvec, bval, [10.0])
    assert e.value.code == -1
    with pytest.raises(ValueError):
        engine.dki_lls(np.ones((1, 5)), bvec, bval)
    with pytest.raises(ValueError):
        engine.dki_shell(np.ones((2, bval.size)), bvec, bval, [10.0])


def test_narrow_signal_normalises_by_sig0():
    sig0 = np.array([1.0, 0.5])
    sigre = np.array([[0.5, -0.25], [0.25, 0.125]])
    np.testing.assert_array_equal(analysis.narrow_signal(sig0, sigre), [[0.5, 0.25], [0.5, 0.25]])


def test_gradient_tables_are_readable_without_a_run():
    lab = np.ones((8, 8, 8), dtype=np.uint8)
    bvec, bval = table(ndirs=20, bvals=(1.0, 2.0))
    s = engine.Sim(lab, dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0], t2=[80, 80],
                   bval=bval, bvec=bvec)
    np.testing.assert_array_equal(s.get("bval"), bval)
    np.testing.assert_array_equal(s.get("bvec").reshape(-1, 3), bvec)
    assert s.field_size("grad") == 0
    grad = np.array([[20.0, 4.0, 0.05, 1, 0, 0], [30.0, 4.0, 0.04, 0, 0.6, 0.8]])
    p = engine.Sim(lab, dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0], t2=[80, 80], grad=grad)
    np.testing.assert_array_equal(p.get("grad").reshape(-1, 6), grad)
    assert p.field_size("bval") == 0 and p.field_size("bvec") == 0


def test_sim_fits_read_the_run_as_the_matlab_readers_do():
    """Sim.dki_shell / dki_lls form the signal table as readRMS.m (narrow) and
    readRMS_pgse.m (PGSE) do; the run's outputs are stood in for here."""
    lab = np.ones((8, 8, 8), dtype=np.uint8)
    d6, w = model(9)
    bvec, bval = table(ndirs=20, bvals=(1.0, 2.0, 3.0))
    T = 4
    td = np.array([5.0, 10.0, 15.0, 20.0])
    sig0 = np.array([1e4, 0.9e4, 0.8e4, 0.7e4])
    S = model_signal(d6, w, bvec, bval, T)
    s = engine.Sim(lab, dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0], t2=[80, 80],
                   bval=bval, bvec=bvec)
    s.outputs = lambda: dict(sig0=sig0, sigre=-S * sig0[:, None], td=td)
    s.get = (lambda get: (lambda name: td if name == "td" else get(name)))(s.get)
    np.testing.assert_allclose(s.dki_shell(), engine.dki_shell(S, bvec, bval, td), rtol=1e-12)
    np.testing.assert_allclose(s.dki_lls(), engine.dki_lls(S, bvec, bval), rtol=1e-12)
    # PGSE: |sig| as summed over walkers, b from the gradient rows, intercept fit
    from rms_b200 import analysis
    dirs = np.repeat(fib_dirs(20), 4, axis=0)
    Delta = np.tile([20.0, 20.0, 30.0, 30.0], 20)
    bv = np.tile([1.0, 2.0, 1.0, 2.0], 20)
    g = analysis.pgse_gradient_for_b(bv, Delta, 4.0)
    grad = np.column_stack([Delta, np.full(bv.size, 4.0), g, dirs])
    p = engine.Sim(lab, dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0], t2=[80, 80], grad=grad)
    sums = 5e3 * model_signal(d6, w, dirs, bv, 1)[0]
    p.outputs = lambda: dict(sig=sums)
    got = p.dki_shell(td=20.0)
    want = engine.dki_shell(sums[None, :], dirs, analysis.pgse_bval(grad), [20.0], intercept=True)
    np.testing.assert_allclose(got, want, rtol=1e-12)
    with pytest.raises(ValueError):
        p.dki_shell()
    with pytest.raises(ValueError):
        p.dki_lls()
