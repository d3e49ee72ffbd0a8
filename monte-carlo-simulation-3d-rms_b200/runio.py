"""Run-directory text formats of the reference simulator.

Writers produce the input files the reference's ``./main_cuda`` reads, in the
layout its MATLAB writer uses (analysis/setupRMS.m:16-69); the PGSE inputs,
for which the reference ships no writer, follow the reader in
hpc_code/lib/main_PGSE.cu:440-445, 495-506.  Readers load the output files
the simulator writes (hpc_code/lib/main.cu:550-615, main_PGSE.cu:596-669), and
the reference's MATLAB geometry and b-table files (hpc_code/input/*/fiber.mat,
hpc_code/btable/*.mat).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

TIMEPOINTS = 1000  # hpc_code/lib/main.cu:35


def _fmt_e(x: float) -> str:
    """MATLAB sprintf('%e') (setupRMS.m:44,49)."""
    return "%e" % x


def _fmt_u(x) -> str:
    """MATLAB sprintf('%u') of an integer-valued double."""
    return "%d" % int(round(x))


def write_lattice(path: str, labels: np.ndarray) -> None:
    """fiber.txt: every label followed by one space, i outer, k fastest, no
    newline (setupRMS.m:17-23); the reader takes NPix1*NPix2*NPix3 integers
    in that order (main.cu:461-466)."""
    lab = np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1)
    with open(path, "wb") as f:
        # the bytes are assembled from digit arrays, 16 M voxels at a time
        step = 1 << 24
        for s in range(0, lab.size, step):
            f.write(_label_text(lab[s:s + step]))


def _label_text(v: np.ndarray) -> bytes:
    """ASCII of "%u " for each uint8 in v, concatenated."""
    v = v.astype(np.int32)
    nd = 1 + (v >= 10) + (v >= 100)          # digits per label
    end = np.cumsum(nd + 1)                  # one past each label's space
    out = np.empty(int(end[-1]) if v.size else 0, dtype=np.uint8)
    if not v.size:
        return b""
    out[end - 1] = ord(" ")
    out[end - 2] = ord("0") + v % 10
    m = nd >= 2
    out[end[m] - 3] = ord("0") + (v[m] // 10) % 10
    m = nd == 3
    out[end[m] - 4] = ord("0") + v[m] // 100
    return out.tobytes()


def write_lattice_binary(path: str, labels: np.ndarray) -> None:
    """fiber.bin: the labels of fiber.txt as raw bytes, i outer, k fastest
    (engine extension; the engine reads it in place of fiber.txt)."""
    np.ascontiguousarray(labels, dtype=np.uint8).reshape(-1).tofile(path)


def write_inputs(target: str, labels: np.ndarray, *, dt: float, tn: int, npar: int,
                 res: float, diffusivity, t2, bval=None, bvec=None, grad=None,
                 lattice: str = "txt") -> None:
    """Write one run directory.

    Narrow-pulse form when ``bval``/``bvec`` are given (setupRMS.m:16-69);
    PGSE form when ``grad`` (Ngrad x 6: Delta, delta, |g|, gx, gy, gz) is
    given (main_PGSE.cu:440-445, 495-506).  Units: ms, um, um^2/ms,
    rad/(um ms) for |g|.  ``lattice``: "txt" (fiber.txt, what the reference
    reads), "bin" (fiber.bin only) or "both".
    """
    os.makedirs(target, exist_ok=True)
    labels = np.asarray(labels)
    if labels.ndim != 3:
        raise ValueError("labels must be a 3-D array (NPix1, NPix2, NPix3)")
    n1, n2, n3 = labels.shape
    d = np.atleast_1d(np.asarray(diffusivity, dtype=np.float64))
    t2a = np.atleast_1d(np.asarray(t2, dtype=np.float64))
    if d.size != t2a.size:
        raise ValueError("diffusivity and T2 need one value per compartment")
    nc = d.size
    pgse = grad is not None
    if pgse == (bval is not None):
        raise ValueError("give either bval/bvec (narrow pulse) or grad (PGSE)")
    if lattice not in ("txt", "bin", "both"):
        raise ValueError("lattice must be 'txt', 'bin' or 'both'")
    if lattice in ("txt", "both"):
        write_lattice(os.path.join(target, "fiber.txt"), labels)
    if lattice in ("bin", "both"):
        write_lattice_binary(os.path.join(target, "fiber.bin"), labels)
    lines = [_fmt_e(dt), _fmt_u(tn), _fmt_u(npar)]
    if not pgse:
        bv = np.atleast_1d(np.asarray(bval, dtype=np.float64))
        bvc = np.asarray(bvec, dtype=np.float64).reshape(-1, 3)
        if bvc.shape[0] != bv.size:
            raise ValueError("bvec must have one row per b-value")
        lines.append(_fmt_u(bv.size))
        with open(os.path.join(target, "bval.txt"), "w") as f:
            f.write("".join("%.8f\n" % x for x in bv))
        with open(os.path.join(target, "bvec.txt"), "w") as f:
            f.write("".join("%.8f\n" % x for x in bvc.reshape(-1)))
    else:
        g = np.asarray(grad, dtype=np.float64).reshape(-1, 6)
        with open(os.path.join(target, "gradient_Ngrad.txt"), "w") as f:
            f.write("%d\n" % g.shape[0])
        with open(os.path.join(target, "gradient_time.txt"), "w") as f:
            f.write("".join(" ".join("%.17g" % x for x in row) + "\n" for row in g))
    lines += [_fmt_u(nc), _fmt_e(res), _fmt_u(n1), _fmt_u(n2), _fmt_u(n3)]
    with open(os.path.join(target, "simParamInput.txt"), "w") as f:
        f.write("".join(x + "\n" for x in lines))
    with open(os.path.join(target, "diffusivity.txt"), "w") as f:
        f.write("".join("%.8f\n" % x for x in d))
    with open(os.path.join(target, "T2.txt"), "w") as f:
        f.write("".join("%.8f\n" % x for x in t2a))


@dataclass
class RunOutputs:
    """The arrays of one finished run directory."""
    sig0: np.ndarray
    dx2: np.ndarray
    dx4: np.ndarray
    npar_count: np.ndarray
    sim_para: np.ndarray
    diff_time: np.ndarray
    sigre: Optional[np.ndarray] = None
    sig: Optional[np.ndarray] = None
    extra: dict = field(default_factory=dict)


def _load(path: str, ncol: Optional[int] = None) -> np.ndarray:
    a = np.loadtxt(path, dtype=np.float64, ndmin=1)
    if ncol is not None:
        a = a.reshape(-1, ncol)
    return a


def read_outputs(root: str) -> RunOutputs:
    """Load a run directory's outputs (the files readRMS.m:30-48 and
    readRMS_pgse.m:31-57 load)."""
    nc = None
    npc = np.loadtxt(os.path.join(root, "NPar_count.txt"), ndmin=2)
    nc = npc.shape[1]
    out = RunOutputs(
        sig0=_load(os.path.join(root, "sig0.txt")),
        dx2=_load(os.path.join(root, "dx2.txt"), 6),
        dx4=_load(os.path.join(root, "dx4.txt"), 15),
        npar_count=npc.reshape(-1, nc),
        sim_para=_load(os.path.join(root, "sim_para.txt")),
        diff_time=_load(os.path.join(root, "diff_time.txt")),
    )
    p_sigre = os.path.join(root, "sigRe.txt")
    p_sig = os.path.join(root, "sig.txt")
    if os.path.exists(p_sigre):
        out.sigre = np.loadtxt(p_sigre, ndmin=2)
    if os.path.exists(p_sig):
        out.sig = _load(p_sig)
    return out


# ---- the reference's MATLAB data files (MAT v5) ----

def read_fiber_mat(path: str) -> list:
    """The lattices of a geometry file in the reference's layout
    (hpc_code/input/*/fiber.mat, read by part1_demo3_simulation.m:28-31): a
    struct array ``fiber`` whose elements hold ``shape`` (a uint8 label
    lattice, [NPix1, NPix2, NPix3]) and ``voxel_size`` (um).  Returns a list of
    (labels, voxel_size), labels C-contiguous uint8 in the engine's layout (k
    fastest, as fiber.txt is written)."""
    from scipy.io import loadmat
    m = loadmat(path)
    if "fiber" not in m:
        raise ValueError(f"{path}: no 'fiber' variable")
    fib = m["fiber"].ravel()
    out = []
    for f in fib:
        lab = np.ascontiguousarray(np.asarray(f["shape"]), dtype=np.uint8)
        if lab.ndim != 3:
            raise ValueError(f"{path}: a fiber shape is not a 3-D lattice")
        out.append((lab, float(np.asarray(f["voxel_size"]).ravel()[0])))
    return out


def read_btable_mat(path: str):
    """A b-table in the reference's layout (hpc_code/btable/*.mat, read by
    part1_demo3_simulation.m:35-37): ``bval`` [Nbvec] (ms/um^2) and ``bvec``
    [Nbvec, 3].  Returns (bval, bvec) as float64 arrays."""
    from scipy.io import loadmat
    m = loadmat(path)
    bval = np.asarray(m["bval"], dtype=np.float64).ravel()
    bvec = np.asarray(m["bvec"], dtype=np.float64).reshape(-1, 3)
    if bvec.shape[0] != bval.size:
        raise ValueError(f"{path}: bval and bvec disagree in length")
    return bval, bvec
