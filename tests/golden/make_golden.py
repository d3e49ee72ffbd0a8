"""Regenerate the golden run directories under tests/golden/.

Each case is a complete run directory: the reference's text inputs, written
by rms_b200.runio (the layout of analysis/setupRMS.m), and the output files
written by the REFERENCE PROGRAM ITSELF -- hpc_code/lib/main.cu or
main_PGSE.cu compiled for the host through oracle/ref_shim (oracle/_ref),
seed pinned.  Files are stored gzip-compressed.

The realistic cases take their lattices from the reference checkout: the
first axon of the mitochondria family (hpc_code/input/
I_realistic_axon_mitochondria/fiber.mat) with every 6th row of the b-table
hpc_code/btable/btable_5shell_90ndir_b1000.mat and the compartment
parameters the reference's demo uses for that family
(part1_demo3_simulation.m: D = [0 2 2/15], T2 = [80 80 20]); and the first
axon of the undulation family (hpc_code/input/IV_undulation/fiber.mat) under
a PGSE table, walked by main_PGSE.cu.

Needs the reference checkout (to build oracle/_ref); run from the repo root:
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import gzip
import os
import shutil
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle  # noqa: E402
from rms_b200 import geometry, runio  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: $RMS_REFERENCE, else "reference" beside the repository
REF = os.environ.get("RMS_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(
    os.path.dirname(os.path.abspath(__file__))))), "reference"))


def lattice(seed: int) -> np.ndarray:
    """16 x 16 x 24 voxels: a thin axon (label 1) in extra-axonal space
    (label 2), with a null (label 0) slab at x = 0..1 so walkers meet all
    three kinds of face: permeable membrane, impermeable null, lattice wall."""
    lab = geometry.axon_lattice(16, 16, 24, 0.1, seed=seed, exterior=2, r0=0.45)
    lab[:2, :, :] = 0
    return lab


CASES = {
    "narrow_3comp": dict(
        seed=20240611, tn=1000, npar=64, dt=2e-4, res=0.1,
        diffusivity=[0.0, 2.0, 1.0], t2=[80.0, 80.0, 40.0],
        bval=[0.5, 1.0, 1.0, 2.0, 2.0, 3.0],
        bvec=[[1, 0, 0], [0, 1, 0], [0, 0, 1], [0.6, 0.8, 0], [0, 0.6, 0.8], [0.48, 0.6, 0.64]],
    ),
    "pgse_3comp": dict(
        seed=777, tn=2000, npar=64, dt=2e-4, res=0.1,
        diffusivity=[0.0, 2.0, 1.5], t2=[80.0, 70.0, 50.0],
        # Delta, delta, |g|, gx, gy, gz; includes Delta < delta (overlapping lobes),
        # a lobe edge between steps, and a gradient outlasting the walk
        grad=[[0.10, 0.05, 3.0, 1, 0, 0], [0.20, 0.05, 3.0, 0, 1, 0],
              [0.20, 0.1003, 2.0, 0, 0, 1], [0.03, 0.05, 4.0, 0.6, 0.8, 0],
              [0.25, 0.2, 1.0, 0, 0.6, 0.8], [0.30, 0.15, 2.5, 0.48, 0.6, 0.64],
              [0.35, 0.1, 1.5, 1, 0, 0], [0.40, 0.1, 1.5, 0, 0, 1]],
    ),
    "realistic_mito_1": dict(
        seed=31337, tn=2000, npar=64, dt=2e-4, res=0.1,
        diffusivity=[0.0, 2.0, 2.0 / 15.0], t2=[80.0, 80.0, 20.0],
        lattice="realistic", btable="reference",
    ),
    "realistic_undulation_pgse": dict(
        seed=4242, tn=2000, npar=64, dt=2e-4, res=0.1,
        diffusivity=[0.0, 2.0, 2.0], t2=[80.0, 80.0, 80.0],
        # Delta, delta, |g|, gx, gy, gz: along the axon (z), across it, oblique
        grad=[[0.20, 0.10, 3.0, 0, 0, 1], [0.20, 0.10, 3.0, 1, 0, 0], [0.20, 0.10, 3.0, 0, 1, 0],
              [0.30, 0.05, 4.0, 0.48, 0.6, 0.64], [0.35, 0.05, 2.0, 0, 0.6, 0.8]],
        lattice="undulation",
    ),
}


def realistic_lattice(family: str = "I_realistic_axon_mitochondria") -> np.ndarray:
    """The first axon of one of the reference's lattice families: 100 x 100 x
    180 voxels of 0.1 um, labels 0 (outside), 1 (axon) and, in the
    mitochondria family, 2 (mitochondria)."""
    from scipy.io import loadmat
    m = loadmat(os.path.join(REF, "hpc_code", "input", family, "fiber.mat"))
    return np.ascontiguousarray(m["fiber"][0, 0]["shape"], dtype=np.uint8)


def reference_btable():
    """Every 6th row of the reference's 5-shell, 90-direction b-table."""
    from scipy.io import loadmat
    m = loadmat(os.path.join(REF, "hpc_code", "btable", "btable_5shell_90ndir_b1000.mat"))
    return m["bval"].ravel()[::6].tolist(), m["bvec"][::6].tolist()


def main():
    if not pyoracle.ref_available():
        sys.exit("oracle/_ref/librmsref.so is missing: run make -C oracle with the reference present")
    only = set(sys.argv[1:])
    for name, c in CASES.items():
        if only and name not in only:
            continue
        if c.get("lattice") == "realistic":
            lab = realistic_lattice()
        elif c.get("lattice") == "undulation":
            lab = realistic_lattice("IV_undulation")
        else:
            lab = lattice(1)
        if c.get("btable") == "reference":
            c = dict(c)
            c["bval"], c["bvec"] = reference_btable()
        tmp = tempfile.mkdtemp()
        kw = dict(dt=c["dt"], tn=c["tn"], npar=c["npar"], res=c["res"],
                  diffusivity=c["diffusivity"], t2=c["t2"])
        if "grad" in c:
            runio.write_inputs(tmp, lab, grad=c["grad"], **kw)
        else:
            runio.write_inputs(tmp, lab, bval=c["bval"], bvec=c["bvec"], **kw)
        rc = pyoracle.run_reference_main(tmp, "grad" in c, c["seed"])
        if rc != 0:
            sys.exit(f"reference run failed for {name}: {rc}")
        out = os.path.join(HERE, name)
        shutil.rmtree(out, ignore_errors=True)
        os.makedirs(out)
        for fn in sorted(os.listdir(tmp)):
            with open(os.path.join(tmp, fn), "rb") as f, gzip.open(os.path.join(out, fn + ".gz"), "wb", 9) as g:
                g.write(f.read())
        with open(os.path.join(out, "SEED"), "w") as f:
            f.write(f"{c['seed']}\n")
        shutil.rmtree(tmp)
        print("wrote", out)


if __name__ == "__main__":
    main()
