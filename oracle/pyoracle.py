"""oracle/pyoracle.py -- TEST INFRASTRUCTURE (the oracle), not product code.

ctypes front end for the two CPU checkers built by oracle/Makefile:

  _build/liboracle.so  the plain-C restatement of the reference walk (rms_oracle.c)
  _ref/librmsref.so    the reference simulator itself (hpc_code/lib/main.cu,
                       main_PGSE.cu) compiled for the host through ref_shim/

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "librmsref.so")

MODE_NARROW, MODE_PGSE, MODE_WAVEFORM = 0, 1, 2
BOUNDARY_MIRROR, BOUNDARY_PERIODIC = 0, 1


class OrParams(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("npar", C.c_int64), ("tn", C.c_int), ("timepoints", C.c_int),
        ("nite", C.c_int), ("nc", C.c_int), ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int),
        ("boundary", C.c_int), ("res", C.c_double), ("dt", C.c_double), ("seed", C.c_uint64),
        ("step", C.POINTER(C.c_double)), ("t2", C.POINTER(C.c_double)),
        ("pij", C.POINTER(C.c_double)), ("labels", C.POINTER(C.c_uint8)),
        ("nbvec", C.c_int), ("bval", C.POINTER(C.c_double)), ("bvec", C.POINTER(C.c_double)),
        ("td", C.POINTER(C.c_double)), ("ngrad", C.c_int), ("grad", C.POINTER(C.c_double)),
        ("nwave", C.c_int), ("nbins", C.c_int), ("wave", C.POINTER(C.c_double)),
        ("rule", C.c_int), ("no_flight", C.c_int),
    ]


class OrOutputs(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in
                ("sig0", "dx2", "dx4", "sigre", "sig", "npar_count", "sigw")]


class OrTrace(C.Structure):
    _fields_ = [("w0", C.c_int64), ("nw", C.c_int64), ("init_voxel", C.POINTER(C.c_int32)),
                ("voxel", C.POINTER(C.c_int32)), ("events", C.POINTER(C.c_uint32)),
                ("pos", C.POINTER(C.c_double)), ("binmean", C.POINTER(C.c_double))]


_lib = None
_ref = None


def oracle_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        _lib = C.CDLL(ORACLE_SO)
        _lib.or_run.restype = C.c_int
        _lib.or_run_parallel.restype = C.c_int
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference host build missing: {REF_SO}")
        _ref = C.CDLL(REF_SO)
        for f in ("ref_narrow_main_dir", "ref_pgse_main_dir", "ref_run_narrow",
                  "ref_run_pgse", "ref_max_threads"):
            getattr(_ref, f).restype = C.c_int
    return _ref


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def reference_tables(dt: float, res: float, diffusivity, t2, timepoints: int = 1000,
                     tn: Optional[int] = None, kappa: Optional[float] = None):
    """Derived tables exactly as hpc_code/lib/main.cu:421-458, 484-487 computes
    them: step (voxels), T2/dt, Pij, TD.  With ``kappa`` (um/ms) the
    permeation probability between two labelled compartments follows the
    membrane permeability instead: the 3-D rule of analysis/interaction.m:
    437-439, P = (2/3) kappa ds / D_i with ds = sqrt(6 D_i dt), used as
    P / (1 + P) (the library's RMS_PERM_KAPPA)."""
    d = [float(x) for x in diffusivity]
    nc = len(d)
    step = np.array([math.sqrt(6.0 * dt * x) / res for x in d])
    t2s = np.array([float(x) / dt for x in t2])
    pij = np.zeros(nc * nc)
    for i in range(nc):
        for j in range(nc):
            if i == 0 or j == 0:
                pij[i * nc + j] = 0.0
            elif i == j:
                pij[i * nc + j] = 1.0
            elif kappa is not None:
                ds = math.sqrt(6.0 * d[i] * dt)
                P = 2.0 / 3.0 * float(kappa) * ds / d[i] if d[i] > 0.0 else 0.0
                pij[i * nc + j] = P / (1.0 + P)
            else:
                pij[i * nc + j] = min(1.0, math.sqrt(d[j] / d[i]))
    td = None
    if tn is not None:
        ts = tn // timepoints
        td = np.array([(i * ts + 1) * dt for i in range(timepoints)])
    return step, t2s, pij, td


class Job:
    """One simulation job in the oracle's terms (tables already derived)."""

    def __init__(self, labels, *, dt, tn, npar, res, step, t2_steps, pij, seed,
                 timepoints=1000, nite=4, boundary=BOUNDARY_MIRROR,
                 bval=None, bvec=None, td=None, grad=None, wave=None, rule=0, no_flight=False):
        self.labels = np.ascontiguousarray(labels, dtype=np.uint8)
        self.n1, self.n2, self.n3 = self.labels.shape
        self.dt, self.tn, self.npar, self.res = float(dt), int(tn), int(npar), float(res)
        self.step = np.ascontiguousarray(step, dtype=np.float64)
        self.t2 = np.ascontiguousarray(t2_steps, dtype=np.float64)
        self.pij = np.ascontiguousarray(pij, dtype=np.float64)
        self.nc = self.step.size
        self.seed = int(seed)
        self.timepoints, self.nite, self.boundary = int(timepoints), int(nite), int(boundary)
        self.mode = MODE_WAVEFORM if wave is not None else (MODE_PGSE if grad is not None else MODE_NARROW)
        # general waveforms [nwave, nbins, 3] (split replay only)
        self.wave = np.ascontiguousarray(wave if wave is not None else np.zeros((0, 0, 3)), dtype=np.float64)
        self.nwave, self.nbins = (self.wave.shape[0], self.wave.shape[1]) if wave is not None else (0, 0)
        self.rule = int(rule)
        self.no_flight = int(bool(no_flight))   # split replay: every step through the face loop
        self.bval = np.ascontiguousarray(bval if bval is not None else np.zeros(0), dtype=np.float64)
        self.bvec = np.ascontiguousarray(bvec if bvec is not None else np.zeros(0), dtype=np.float64).reshape(-1)
        self.nbvec = self.bval.size if self.mode == MODE_NARROW else 0
        if td is None:
            ts = self.tn // self.timepoints
            td = np.array([(i * ts + 1) * self.dt for i in range(self.timepoints)])
        self.td = np.ascontiguousarray(td, dtype=np.float64)
        self.grad = np.ascontiguousarray(grad if grad is not None else np.zeros(0), dtype=np.float64).reshape(-1)
        self.ngrad = self.grad.size // 6

    def params(self) -> OrParams:
        return OrParams(
            self.mode, self.npar, self.tn, self.timepoints, self.nite, self.nc, self.n1,
            self.n2, self.n3, self.boundary, self.res, self.dt, self.seed,
            _dp(self.step), _dp(self.t2), _dp(self.pij),
            self.labels.ctypes.data_as(C.POINTER(C.c_uint8)),
            self.nbvec, _dp(self.bval), _dp(self.bvec), _dp(self.td),
            self.ngrad, _dp(self.grad), self.nwave, self.nbins, _dp(self.wave), self.rule, self.no_flight)

    def empty_outputs(self):
        T = self.timepoints
        return dict(sig0=np.zeros(T), dx2=np.zeros((T, 6)), dx4=np.zeros((T, 15)),
                    sigre=np.zeros((T, max(self.nbvec, 0))), sig=np.zeros(self.ngrad),
                    npar_count=np.zeros((T, self.nc)), sigw=np.zeros((max(self.nwave, 0), 2)))


def _out_struct(o):
    return OrOutputs(*(_dp(o[k]) for k in ("sig0", "dx2", "dx4", "sigre", "sig", "npar_count", "sigw")))


def run_oracle(job: Job, w_begin: int = 0, w_end: Optional[int] = None, nthreads: int = 1,
               trace_walkers: int = 0, split: bool = False):
    """Walk walkers [w_begin, w_end) with the C restatement.  With
    ``trace_walkers`` > 0 the first that many walkers of the range also
    return their per-step voxel and event traces (single thread).  With
    ``split`` the FP64 replay of the engine's split-precision walk runs instead
    of the reference walk."""
    lib = oracle_lib()
    run1 = lib.or_run_split if split else lib.or_run
    runp = lib.or_run_split_parallel if split else lib.or_run_parallel
    if w_end is None:
        w_end = job.npar
    o = job.empty_outputs()
    p = job.params()
    outs = _out_struct(o)
    if trace_walkers:
        nw = int(trace_walkers)
        tr_init = np.zeros(nw, dtype=np.int32)
        tr_vox = np.zeros((nw, job.tn), dtype=np.int32)
        tr_ev = np.zeros((nw, job.tn), dtype=np.uint32)
        tr_pos = np.zeros((nw, job.tn, 3))
        tr_bin = np.zeros((nw, max(job.nbins, 1), 3))
        tr = OrTrace(w_begin, nw, tr_init.ctypes.data_as(C.POINTER(C.c_int32)),
                     tr_vox.ctypes.data_as(C.POINTER(C.c_int32)),
                     tr_ev.ctypes.data_as(C.POINTER(C.c_uint32)), _dp(tr_pos), _dp(tr_bin))
        rc = run1(C.byref(p), C.c_int64(w_begin), C.c_int64(w_end), C.byref(outs), C.byref(tr))
        o["trace"] = dict(init_voxel=tr_init, voxel=tr_vox, events=tr_ev, pos=tr_pos, binmean=tr_bin)
    elif nthreads > 1:
        rc = runp(C.byref(p), C.c_int64(w_begin), C.c_int64(w_end), C.c_int(nthreads), C.byref(outs))
    else:
        rc = run1(C.byref(p), C.c_int64(w_begin), C.c_int64(w_end), C.byref(outs), None)
    if rc != 0:
        raise RuntimeError(f"or_run failed: {rc}")
    return o


def stream_doubles(seed: int, walker: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    oracle_lib().or_stream_doubles(C.c_uint64(seed), C.c_uint64(walker), C.c_int(n), _dp(out))
    return out


def stream_floats(seed: int, walker: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    oracle_lib().or_stream_floats(C.c_uint64(seed), C.c_uint64(walker), C.c_int(n),
                                  out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def split_dir_uniforms(seed: int, walker: int, nsteps: int) -> np.ndarray:
    out = np.zeros(2 * nsteps, dtype=np.float32)
    oracle_lib().or_split_dir_uniforms(C.c_uint64(seed), C.c_uint64(walker), C.c_int(nsteps),
                                       out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def split_domain_floats(seed: int, walker: int, dom: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    oracle_lib().or_split_domain_floats(C.c_uint64(seed), C.c_uint64(walker), C.c_uint32(dom), C.c_int(n),
                                        out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def philox4x32_10(ctr, key) -> np.ndarray:
    c = np.array(ctr, dtype=np.uint32)
    k = np.array(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    u32p = C.POINTER(C.c_uint32)
    oracle_lib().or_philox4x32_10(c.ctypes.data_as(u32p), k.ctypes.data_as(u32p),
                                  out.ctypes.data_as(u32p))
    return out


def run_reference_main(run_dir: str, pgse: bool, seed: int) -> int:
    """Run the reference program's main() in ``run_dir`` (the process
    contract of part1_demo3_simulation.m:86-90), seed pinned."""
    lib = ref_lib()
    os.environ["RMS_REF_SEED"] = str(int(seed))
    try:
        fn = lib.ref_pgse_main_dir if pgse else lib.ref_narrow_main_dir
        return fn(run_dir.encode())
    finally:
        os.environ.pop("RMS_REF_SEED", None)


def run_reference_walkers(job: Job, nsample: int, nthreads: int):
    """The reference's own propagate() on walkers [0, nsample) of the job,
    OpenMP over walkers (the timed CPU baseline).  Labels go in as int32 like
    the reference's APix (main.cu:461)."""
    if job.timepoints != 1000 or job.nite != 4 or job.boundary != BOUNDARY_MIRROR:
        raise ValueError("the reference build supports only its own constants")
    lib = ref_lib()
    apix = np.ascontiguousarray(job.labels, dtype=np.int32)
    ip = apix.ctypes.data_as(C.POINTER(C.c_int))
    o = job.empty_outputs()
    if job.mode == MODE_NARROW:
        rc = lib.ref_run_narrow(
            C.c_ulonglong(job.seed), job.tn, job.npar, C.c_int64(nsample), job.nbvec, job.nc,
            C.c_double(job.res), _dp(job.step), job.n1, job.n2, job.n3, _dp(job.t2),
            _dp(job.pij), _dp(job.bval), _dp(job.bvec), ip, _dp(job.td), nthreads,
            _dp(o["sig0"]), _dp(o["dx2"]), _dp(o["dx4"]), _dp(o["sigre"]), _dp(o["npar_count"]))
    else:
        rc = lib.ref_run_pgse(
            C.c_ulonglong(job.seed), job.tn, job.npar, C.c_int64(nsample), job.nc,
            C.c_double(job.res), C.c_double(job.dt), _dp(job.step), job.n1, job.n2, job.n3,
            job.ngrad, _dp(job.grad), _dp(job.t2), _dp(job.pij), ip, nthreads,
            _dp(o["sig0"]), _dp(o["dx2"]), _dp(o["dx4"]), _dp(o["sig"]), _dp(o["npar_count"]))
    if rc != 0:
        raise RuntimeError(f"reference run failed: {rc}")
    return o


def ref_max_threads() -> int:
    return int(ref_lib().ref_max_threads())


def contract_phases_fp64(pos, wave, chunk: int = 65536):
    """FP64 restatement of the multi-waveform phase contraction
    (rms_contract_phases): for float inputs pos [nwalk, nbins, 3] and
    wave [nwave, nbins, 3], phi = pos . wave over (bin, axis) in float64, and
    the per-waveform sums of cos(phi) and sin(phi), [nwave, 2].  Test
    infrastructure: the checker of the GPU contraction."""
    P = np.asarray(pos, dtype=np.float32).reshape(len(pos), -1).astype(np.float64)
    W = np.asarray(wave, dtype=np.float32).reshape(len(wave), -1).astype(np.float64)
    out = np.zeros((W.shape[0], 2))
    for a in range(0, P.shape[0], chunk):
        phi = P[a:a + chunk] @ W.T
        out[:, 0] += np.cos(phi).sum(axis=0)
        out[:, 1] += np.sin(phi).sum(axis=0)
    return out


def adjoint_split(job: "Job", gup, w_begin: int = 0, w_end: Optional[int] = None):
    """Walker sums of the split walk's adjoint in waveform mode (or_adjoint_split,
    the FP64 restatement of csrc/rms_adjoint.cu): dict with L, LE, path, E,
    LT [nc], sigw [nwave, 2], TR (time rescaling), F (forced permeation
    decisions: the sum of nb Pij (1 - Pij) (L[crossed] - L[reflected])) and
    dwave [nbins, nwave, 3] (sum of a_jw X_wb, um)."""
    lib = oracle_lib()
    if w_end is None:
        w_end = job.npar
    g = np.ascontiguousarray(np.asarray(gup, dtype=np.float64).reshape(-1))
    sums = np.zeros(4 + job.nc + 2 * job.nwave + 2)
    dw = np.zeros(job.nbins * job.nwave * 3)
    p = job.params()
    rc = lib.or_adjoint_split(C.byref(p), _dp(g), C.c_int64(w_begin), C.c_int64(w_end), _dp(sums), _dp(dw))
    if rc != 0:
        raise RuntimeError(f"or_adjoint_split failed: {rc}")
    nc, nw = job.nc, job.nwave
    return dict(L=sums[0], LE=sums[1], path=sums[2], E=sums[3], LT=sums[4:4 + nc].copy(),
                sigw=sums[4 + nc:4 + nc + 2 * nw].reshape(-1, 2).copy(), TR=sums[4 + nc + 2 * nw],
                F=sums[5 + nc + 2 * nw],
                dwave=dw.reshape(job.nbins, job.nwave, 3))


def adjoint_gradients(job: "Job", sums: dict, D: float, t2, kappa: Optional[float] = None, nwalk: Optional[int] = None):
    """The gradients the library's host code forms from the adjoint walker sums
    (monte-carlo-simulation-3d-rms_b200/csrc/rms_api.cpp, run_adjoint):
    dL/dwave = dt sum a X; dL/dlog P from the forced decisions (F), beside the
    score function with the mean loss as baseline; dL/dD by time rescaling,
    (TR - F [kappa mode] or TR - F / 2) / D; the pathwise
    dL/dD = (path l / 2 - F / 2 [kappa mode]) / D (l = sqrt(6 D dt)/res);
    dL/dkappa = F / kappa (score / kappa as d_kappa_score);
    dL/dT2_c = sum L t_c dt / T2_c^2."""
    n = job.npar if nwalk is None else nwalk
    score = sums["LE"] - sums["L"] / n * sums["E"]
    F = sums["F"]
    step = float(job.step[1 if job.nc > 1 else 0])
    kap = kappa is not None
    d_wave = job.dt * np.transpose(sums["dwave"], (1, 0, 2))
    d_D = (sums["TR"] - (F if kap else 0.5 * F)) / D
    d_D_path = (sums["path"] * step / 2.0 - (F / 2.0 if kap else 0.0)) / D
    d_kappa = F / kappa if kap and kappa > 0 else 0.0
    d_kappa_score = score / kappa if kap and kappa > 0 else 0.0
    t2 = np.asarray(t2, dtype=np.float64)
    d_t2 = sums["LT"] * job.dt / t2 ** 2
    return dict(d_wave=d_wave, d_diffusivity=d_D, d_diffusivity_pathwise=d_D_path, d_kappa=d_kappa,
                d_kappa_score=d_kappa_score, d_t2=d_t2, loss=sums["L"])
