"""The reference arm of bench.py stays clear of the engine: it derives the
reference's tables (main.cu:433-458, and the kappa rule of
analysis/interaction.m:437-439) in the oracle, and no engine library is
loaded in its process.  CPU only."""
import os
import subprocess
import sys

import numpy as np

import pyoracle
from rms_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_kappa_tables_equal_the_library_tables():
    for D, kappa, dt in (([0.0, 2.0, 2.0], 0.01, 2e-4), ([0.0, 1.7, 2.3, 0.5], 0.05, 1e-4), ([0.0, 2.0], 0.0, 2e-4)):
        sim = engine.Sim(None, shape=(8, 8, 8), dt=dt, tn=1000, npar=64, res=0.1, diffusivity=D,
                         t2=[80.0] * len(D), bval=[], bvec=np.zeros((0, 3)), permeation="kappa", kappa=kappa)
        step, _, pij, _ = pyoracle.reference_tables(dt, 0.1, D, [80.0] * len(D), kappa=kappa)
        assert np.array_equal(sim.get("pij"), pij), (D, kappa)
        assert np.array_equal(sim.get("step"), step)
        sim.close()


def test_reference_arm_loads_no_engine_library():
    if not pyoracle.ref_available():
        import pytest
        pytest.skip("reference host build not present (make -C oracle)")
    code = f"""
import sys, numpy as np
sys.path.insert(0, {ROOT!r}); sys.path.insert(0, {os.path.join(ROOT, 'oracle')!r})
import bench, pyoracle
from rms_b200 import geometry
lab = geometry.axon_lattice(16, 16, 32, 0.1, seed=1, exterior=2, r0=0.5)
kw = dict(dt=2e-4, tn=1000, npar=4096, res=0.1, diffusivity=[0.0, 2.0, 2.0], t2=[1e12] * 3,
          bval=[], bvec=np.zeros((0, 3)), permeation="kappa", kappa=0.03)
job, n, cores, kind = bench.cpu_reference_rate(lab, kw, target_s=0.2, nthreads=2)
o = pyoracle.run_reference_walkers(job, min(n, 256), cores)
assert o["npar_count"][0].sum() == min(n, 256)
maps = open('/proc/self/maps').read()
print('LOADED_ENGINE' if 'librms.so' in maps else 'CLEAN')
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip().splitlines()[-1] == "CLEAN"
