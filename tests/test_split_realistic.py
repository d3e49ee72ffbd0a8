"""The split walk on one of the reference's realistic lattices, on the CPU.

The oracle's FP64 replay of the engine's split walk (FP32 in-voxel
positions, 4-bit padded lattice, free flight, step-indexed draws) against the
reference walk itself (the oracle's restatement of main.cu), on independent
random streams: the first axon of the reference's mitochondria family
(tests/golden/realistic_mito_1: 100 x 100 x 180 voxels, 0.2 % labelled,
D = [0 2 2/15], T2 = [80 80 20], the reference's Pij rule).  The GPU split
walk equals this replay walker by walker (tests/test_gpu_split.py), so this
ties the engine's fast walk to the reference's physics on real geometry.

Bounds, for N = 32768 walkers per walk and two independent walks, from the
spread measured over 12 seed pairs at 65536 walkers (no bias found: every
z-score of D and K within 1.8): per walk sigma(D)/D <= 0.8 % and
sigma(K) <= 0.037 at 32768 walkers, so a difference has sigma(D)/D <= 1.1 %
and sigma(K) <= 0.052; the checks allow 4.5 and 3.8 of those.
"""
import os

import numpy as np
import pytest

import pyoracle
from conftest import unpack_golden
from rms_b200 import analysis

N = 32768


@pytest.fixture(scope="module")
def walks(tmp_path_factory):
    d = unpack_golden("realistic_mito_1", str(tmp_path_factory.mktemp("mito")), inputs_only=True)
    vals = open(os.path.join(d, "simParamInput.txt")).read().split()
    n1, n2, n3 = (int(x) for x in vals[-3:])
    lab = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8).reshape(n1, n2, n3)
    D, T2 = [0.0, 2.0, 2.0 / 15.0], [80.0, 80.0, 20.0]
    tn, tp = 2000, 100
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, tp, tn)
    threads = max(1, min(16, os.cpu_count() or 1))
    out = {}
    for name, split, seed in (("reference", False, 101), ("split", True, 202)):
        job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=N, res=0.1, step=step, t2_steps=t2s, pij=pij,
                           seed=seed, timepoints=tp, td=td)
        out[name] = pyoracle.run_oracle(job, nthreads=threads, split=split)
    out["volume_fraction"] = np.count_nonzero(lab == 2) / np.count_nonzero(lab)
    return out, td


def test_diffusivity_and_kurtosis_agree(walks):
    out, td = walks
    ref, spl = out["reference"], out["split"]
    Dr, Kr = analysis.axis_dk(ref["sig0"], ref["dx2"], ref["dx4"], td)
    Ds, Ks = analysis.axis_dk(spl["sig0"], spl["dx2"], spl["dx4"], td)
    for i in (19, 49, 99):
        np.testing.assert_allclose(Ds[i], Dr[i], rtol=0.05, err_msg=f"D at t = {td[i]:.3f} ms")
        np.testing.assert_allclose(Ks[i], Kr[i], atol=0.2, err_msg=f"K at t = {td[i]:.3f} ms")
    # a thin axon: across it diffusion is restricted, along it nearly free
    assert Dr[-1].min() < 0.5 * Dr[-1].max()


def test_compartments_and_relaxation_agree(walks):
    out, _ = walks
    ref, spl = out["reference"], out["split"]
    for o in (ref, spl):
        assert np.all(o["npar_count"].sum(axis=1) == N)
    # walkers in the mitochondria (label 2): the fraction is set by the uniform
    # start and stays at the volume fraction (the reference's Pij rule keeps
    # the uniform equilibrium); binomial spread, 5 sigma (over 12 seed pairs at
    # 65536 walkers the two walks differed by z = -1.2 .. -1.6, no bias)
    fr, fs = ref["npar_count"][:, 2] / N, spl["npar_count"][:, 2] / N
    vol = out["volume_fraction"]
    sd = np.sqrt(vol * (1 - vol) / N)
    assert np.all(np.abs(fs - fr) < 5 * np.sqrt(2) * sd)
    assert np.all(np.abs(fr - vol) < 5 * sd) and np.all(np.abs(fs - vol) < 5 * sd)
    # T2-weighted signal (T2 = 20 ms in the mitochondria)
    np.testing.assert_allclose(spl["sig0"] / N, ref["sig0"] / N, rtol=5e-3)


def test_pgse_signal_on_the_undulating_axon():
    """The PGSE signal of the split walk's replay against the reference walk on
    the reference's first undulating axon (tests/golden/realistic_undulation_pgse),
    b = 1 ms/um^2 (Delta 0.3 ms, delta 0.1 ms) along, across and oblique to the
    axon: S ~ 0.21 along it, 0.93-0.96 across.  Per walker Var(cos phi) <= 1/2,
    so a difference of two 32768-walker walks has sigma <= 0.0055; the bar is
    0.025 (two seed pairs differed by 0.009 and 0.003)."""
    import tempfile
    d = unpack_golden("realistic_undulation_pgse", tempfile.mkdtemp(), inputs_only=True)
    lab = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8).reshape(100, 100, 180)
    D, T2, tn = [0.0, 2.0, 2.0], [80.0, 80.0, 80.0], 2000
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, D, T2, 100, tn)
    dirs = np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0], [0.48, 0.6, 0.64], [0.6, 0, 0.8], [0, 0.6, 0.8]])
    g = float(analysis.pgse_gradient_for_b(1.0, 0.3, 0.1))
    grad = np.column_stack([np.full(6, 0.3), np.full(6, 0.1), np.full(6, g), dirs])
    threads = max(1, min(16, os.cpu_count() or 1))
    sig = {}
    for name, split, seed in (("reference", False, 1), ("split", True, 2)):
        job = pyoracle.Job(lab, dt=2e-4, tn=tn, npar=N, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=seed,
                           timepoints=100, td=td, grad=grad)
        sig[name] = pyoracle.run_oracle(job, nthreads=threads, split=split)["sig"] / N
    np.testing.assert_allclose(sig["split"], sig["reference"], atol=0.025)
    assert sig["reference"][0] < 0.3 and sig["reference"][1] > 0.9      # along vs across the axon
