"""Shared test set-up.

Markers: ``gpu`` -- needs a CUDA GPU (B200); everything unmarked runs on CPU.
The oracle (oracle/) is the checker: tests load it only to compare against.
"""
import gzip
import os
import shutil
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200)")


def unpack_golden(name: str, dest: str, inputs_only: bool = False) -> str:
    """Decompress tests/golden/<name>/*.gz into dest; returns dest."""
    src = os.path.join(GOLDEN, name)
    outputs = {"sig0.txt", "dx2.txt", "dx4.txt", "sigRe.txt", "sig.txt", "NPar_count.txt",
               "sim_para.txt", "diff_time.txt"}
    os.makedirs(dest, exist_ok=True)
    for fn in os.listdir(src):
        if not fn.endswith(".gz"):
            continue
        base = fn[:-3]
        if inputs_only and base in outputs:
            continue
        with gzip.open(os.path.join(src, fn), "rb") as f, open(os.path.join(dest, base), "wb") as g:
            shutil.copyfileobj(f, g)
    return dest


def golden_seed(name: str) -> int:
    with open(os.path.join(GOLDEN, name, "SEED")) as f:
        return int(f.read().strip())


def assert_fp64_close(got, want, rtol=1e-9, what=""):
    """Agreement of FP64 sums up to last-bit differences of sin/cos/exp and of
    summation order: |got - want| <= rtol * max(|want| over the row)."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    assert got.shape == want.shape, (what, got.shape, want.shape)
    w2 = want.reshape(want.shape[0], -1) if want.ndim > 1 else want.reshape(1, -1)
    g2 = got.reshape(w2.shape)
    scale = np.maximum(np.abs(w2).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(g2 - w2) / scale
    assert np.all(np.isfinite(g2)), what
    assert err.max() <= rtol, f"{what}: max scaled error {err.max():.3e} > {rtol}"


@pytest.fixture
def tmpdir_path(tmp_path):
    return str(tmp_path)
