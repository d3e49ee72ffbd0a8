"""ctypes binding of librms (include/rms.h).

The engine's compute path is the compiled library; this module only marshals
arrays across the C ABI.  There is no Python or CPU fallback: if librms.so is
missing, or no GPU is present when a run is requested, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_build", "librms.so")
CLI_PATH = os.path.join(PKG_DIR, "_build", "rms_main")

MODE = {"narrow": 0, "pgse": 1, "waveform": 2, "auto": -1}
BOUNDARY = {"mirror": 0, "periodic": 1}
PERMEATION = {"reference": 0, "kappa": 1, "table": 2}
PRECISION = {"compat": 0, "split": 1}
FIELD = {"sig0": 0, "dx2": 1, "dx4": 2, "sigre": 3, "sig": 4, "npar_count": 5, "td": 6,
         "diffusivity": 7, "step": 8, "pij": 9, "sigw": 10, "bval": 11, "bvec": 12, "grad": 13,
         "sim_para": 14}
ERRORS = {-1: "ARG", -2: "IO", -3: "FORMAT", -4: "RANGE", -5: "CUDA", -6: "NOMEM",
          -7: "STATE", -8: "TIMEOUT"}

# The C ABI's exported names (include/rms.h), checked by the CPU tests.
EXPORTS = ("rms_sim_create", "rms_sim_load_dir", "rms_sim_set_lattice", "rms_sim_run",
           "rms_sim_field_size", "rms_sim_get", "rms_sim_get_trace", "rms_sim_get_trace_positions",
           "rms_sim_write_dir",
           "rms_sim_last_timing", "rms_batch_run", "rms_last_error", "rms_sim_destroy",
           "rms_rng_doubles", "rms_rng_floats", "rms_philox4x32_10", "rms_version",
           "rms_split_variant", "rms_rng_split", "rms_sim_run_noalloc", "rms_contract_phases",
           "rms_adjoint_run", "rms_adjoint_jacobian", "rms_autotune", "rms_batch_graph_create", "rms_graph_run", "rms_graph_destroy",
           "rms_sim_cumulants", "rms_combine_cumulants", "rms_sim_set_tube_lattice",
           "rms_dki_shell", "rms_dki_lls", "rms_akc_shell", "rms_akc_lls")
CONTRACT = {"fp32": 0, "bf16x3": 1, "bf16x3_presplit": 2}

_DP = C.POINTER(C.c_double)


class RmsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rms error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [
        ("mode", C.c_int), ("dt", C.c_double), ("tn", C.c_int), ("npar", C.c_int64),
        ("nc", C.c_int), ("res", C.c_double), ("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int),
        ("diffusivity", _DP), ("t2", _DP),
        ("nbvec", C.c_int), ("bval", _DP), ("bvec", _DP),
        ("ngrad", C.c_int), ("grad", _DP),
        ("nwave", C.c_int), ("nbins", C.c_int), ("wave", _DP),
        ("timepoints", C.c_int), ("nite", C.c_int), ("boundary", C.c_int),
        ("permeation", C.c_int), ("kappa", C.c_double), ("pij", _DP),
        ("membrane_rule", C.c_int),
    ]


RULE = {"reflect": 0, "reject": 1, "leap": 2}


class RunOpts(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64), ("precision", C.c_int), ("device", C.c_int),
        ("stream", C.c_void_p), ("trace_walkers", C.c_int), ("variant", C.c_int),
        ("walker_begin", C.c_int64), ("walker_end", C.c_int64),
        ("traj_out", C.c_void_p), ("traj_split", C.c_int),
        ("shard_index", C.c_int), ("shard_count", C.c_int),
    ]


def _opts(seed=0, precision="split", device=0, stream=None, trace_walkers=0, variant=0, walker_range=None,
          traj_out=0, traj_split=False, shard=None) -> RunOpts:
    """rms_run_opts of a call; ``shard`` = (index, count) walks only that
    shard of every simulation's walkers (one rank's part of a job or batch)."""
    w0, w1 = walker_range if walker_range is not None else (0, 0)
    si, sc = shard if shard is not None else (0, 0)
    st = None if stream is None else C.c_void_p(int(stream))
    return RunOpts(int(seed) & ((1 << 64) - 1), PRECISION[precision], int(device), st, int(trace_walkers),
                   int(variant), int(w0), int(w1), C.c_void_p(int(traj_out)) if traj_out else None,
                   1 if traj_split else 0, int(si), int(sc))


class AdjointGrads(C.Structure):
    _fields_ = [("d_wave", _DP), ("d_diffusivity", C.c_double), ("d_kappa", C.c_double),
                ("d_t2", C.c_double * 8), ("loss", C.c_double), ("sigw", _DP),
                ("d_diffusivity_pathwise", C.c_double), ("d_kappa_score", C.c_double)]


_lib = None


def lib():
    """Load librms.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"librms.so not built: {LIB_PATH} "
                               "(run __graft_entry__.build() or make -C monte-carlo-simulation-3d-rms_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        L.rms_last_error.restype = C.c_char_p
        L.rms_version.restype = C.c_char_p
        for name in EXPORTS:
            if name not in ("rms_last_error", "rms_version", "rms_sim_destroy", "rms_graph_destroy"):
                getattr(L, name).restype = C.c_int
        L.rms_sim_destroy.restype = None
        L.rms_sim_create.argtypes = [C.POINTER(Config), C.POINTER(C.c_void_p)]
        L.rms_sim_load_dir.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_void_p)]
        L.rms_sim_set_lattice.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int]
        L.rms_sim_run.argtypes = [C.c_void_p, C.POINTER(RunOpts)]
        L.rms_sim_field_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
        L.rms_sim_get.argtypes = [C.c_void_p, C.c_int, _DP, C.c_size_t]
        L.rms_sim_get_trace.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_uint32), C.c_size_t, C.c_size_t]
        L.rms_sim_get_trace_positions.argtypes = [C.c_void_p, _DP, C.c_size_t, C.c_size_t]
        L.rms_sim_write_dir.argtypes = [C.c_void_p, C.c_char_p]
        L.rms_sim_last_timing.argtypes = [C.c_void_p, _DP, _DP]
        L.rms_batch_run.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(RunOpts)]
        L.rms_sim_destroy.argtypes = [C.c_void_p]
        L.rms_rng_doubles.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _DP]
        L.rms_rng_floats.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_float)]
        L.rms_philox4x32_10.argtypes = [C.POINTER(C.c_uint32)] * 3
        L.rms_sim_run_noalloc.argtypes = [C.c_void_p, C.POINTER(RunOpts), C.c_void_p, C.c_void_p, C.c_void_p]
        L.rms_rng_split.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_float)]
        L.rms_split_variant.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.rms_batch_graph_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(RunOpts), C.POINTER(C.c_void_p)]
        L.rms_graph_run.argtypes = [C.c_void_p, C.c_uint64]
        L.rms_graph_destroy.argtypes = [C.c_void_p]
        L.rms_graph_destroy.restype = None
        L.rms_sim_set_tube_lattice.argtypes = [C.c_void_p, _DP, _DP, _DP, C.c_int, C.c_int, C.c_int]
        L.rms_sim_cumulants.argtypes = [C.c_void_p, _DP, C.c_int, _DP, _DP]
        L.rms_combine_cumulants.argtypes = [C.c_int, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP]
        L.rms_dki_shell.argtypes = [C.c_int, C.c_int, _DP, _DP, _DP, _DP, C.c_int, _DP]
        L.rms_dki_lls.argtypes = [C.c_int, C.c_int, _DP, _DP, _DP, _DP]
        L.rms_akc_shell.argtypes = [C.c_int, _DP, C.c_int, _DP, _DP, _DP, _DP]
        L.rms_akc_lls.argtypes = [C.c_int, _DP, C.c_int, _DP, _DP, _DP]
        L.rms_autotune.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.POINTER(RunOpts), C.POINTER(C.c_int), _DP]
        L.rms_adjoint_run.argtypes = [C.c_void_p, C.POINTER(RunOpts), _DP, C.POINTER(AdjointGrads)]
        L.rms_adjoint_jacobian.argtypes = [C.c_void_p, C.POINTER(RunOpts), _DP, _DP]
        L.rms_contract_phases.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int, C.c_int,
                                          C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]
        _lib = L
    return _lib


def _check(rc: int):
    if rc != 0:
        raise RmsError(rc, lib().rms_last_error().decode(errors="replace"))


def _arr(x, dtype=np.float64):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype).reshape(-1))


def _ptr(a: Optional[np.ndarray]):
    return a.ctypes.data_as(_DP) if a is not None and a.size else None


class Sim:
    """One simulation (an ``rms_sim``): configuration, lattice, results."""

    def __init__(self, labels=None, *, dt, tn, npar, res, diffusivity, t2, nc=None,
                 shape=None, bval=None, bvec=None, grad=None, wave=None, timepoints=0, nite=0,
                 boundary="mirror", permeation="reference", kappa=0.0, pij=None, rule="reflect"):
        """``wave``: general waveforms, array [nwave, nbins, 3] (phase per um of
        a bin's displacement sum, per ms: phase_j = dt sum_b wave[j, b] . X_b);
        selects the waveform mode (SPLIT walk only)."""
        self._h = C.c_void_p()
        d = _arr(diffusivity)
        t2a = _arr(t2)
        mode = "waveform" if wave is not None else ("pgse" if grad is not None else "narrow")
        wv = None
        if wave is not None:
            wv = np.ascontiguousarray(np.asarray(wave, dtype=np.float64))
            if wv.ndim != 3 or wv.shape[2] != 3:
                raise ValueError("wave must be [nwave, nbins, 3]")
        if labels is not None:
            labels = np.ascontiguousarray(labels, dtype=np.uint8)
            shape = labels.shape
        if shape is None:
            raise ValueError("give labels or shape")
        self._keep = [d, t2a]
        bv = _arr(bval if bval is not None else [])
        bvc = _arr(bvec if bvec is not None else [])
        gr = _arr(grad if grad is not None else [])
        pj = _arr(pij) if pij is not None else None
        self._keep += [bv, bvc, gr, pj, wv]
        self.wave_shape = wv.shape if wv is not None else None
        self.nc = int(nc or d.size)
        cfg = Config(MODE[mode], float(dt), int(tn), int(npar), int(nc or d.size), float(res),
                     int(shape[0]), int(shape[1]), int(shape[2]), _ptr(d), _ptr(t2a),
                     bv.size if mode == "narrow" else 0, _ptr(bv), _ptr(bvc),
                     gr.size // 6 if mode == "pgse" else 0, _ptr(gr),
                     wv.shape[0] if wv is not None else 0, wv.shape[1] if wv is not None else 0,
                     _ptr(wv.reshape(-1)) if wv is not None else None,
                     int(timepoints), int(nite), BOUNDARY[boundary], PERMEATION[permeation],
                     float(kappa), _ptr(pj), RULE[rule])
        _check(lib().rms_sim_create(C.byref(cfg), C.byref(self._h)))
        self.mode = mode
        self.shape = tuple(int(x) for x in shape)
        self.tn = int(tn)
        if labels is not None:
            self.set_lattice(labels)

    @classmethod
    def from_dir(cls, path: str, mode: str = "auto") -> "Sim":
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        self._keep = []
        self.wave_shape = None
        _check(lib().rms_sim_load_dir(path.encode(), MODE[mode], C.byref(self._h)))
        if mode == "auto":
            mode = "pgse" if os.path.exists(os.path.join(path, "gradient_time.txt")) else "narrow"
        self.mode = mode
        vals = open(os.path.join(path, "simParamInput.txt")).read().split()
        self.tn = int(vals[1])
        self.shape = tuple(int(v) for v in vals[-3:])
        self.nc = int(vals[4 if mode == "narrow" else 3])
        return self

    def set_lattice(self, labels: np.ndarray):
        lab = np.ascontiguousarray(labels, dtype=np.uint8)
        if lab.ndim != 3:
            raise ValueError("labels must be 3-D")
        _check(lib().rms_sim_set_lattice(self._h, lab.ctypes.data_as(C.POINTER(C.c_uint8)),
                                         *[int(x) for x in lab.shape]))

    def set_tube_lattice(self, r2, cx, cy, inside: int = 1, outside: int = 0, device: int = 0):
        """Build the lattice on the GPU from per-slice tables (geometry.axon_slices)."""
        a, b, c = _arr(r2), _arr(cx), _arr(cy)
        if not (a.size == b.size == c.size == self.shape[2]):
            raise ValueError("one radius^2 and centre per z slice")
        _check(lib().rms_sim_set_tube_lattice(self._h, _ptr(a), _ptr(b), _ptr(c), int(inside), int(outside), int(device)))

    def run(self, seed: int = 0, precision: str = "compat", device: int = 0, stream=None,
            trace_walkers: int = 0, variant: int = 0, walker_range=None, traj_out: int = 0,
            traj_split: bool = False, shard=None):
        """``traj_out``: device address of a float32 [walkers, nbins, 3] buffer
        for the bins' mean displacements (waveform mode, SPLIT); with
        ``traj_split`` the same bytes hold BF16 hi parts then lo parts (the
        input of contract_phases(method="bf16x3_presplit")).  ``shard`` =
        (index, count): walk only that shard of the walkers."""
        opts = _opts(seed, precision, device, stream, trace_walkers, variant, walker_range, traj_out, traj_split,
                     shard)
        _check(lib().rms_sim_run(self._h, C.byref(opts)))
        return self

    def run_noalloc(self, d_labels: int, d_rows: int, d_sig: int = 0, seed: int = 0, device: int = 0,
                    stream=None, walker_range=None):
        """The split walk on caller-owned device buffers (raw device addresses),
        allocating nothing; see rms_sim_run_noalloc in include/rms.h."""
        opts = _opts(seed, "split", device, stream, walker_range=walker_range)
        _check(lib().rms_sim_run_noalloc(self._h, C.byref(opts), C.c_void_p(int(d_labels)),
                                         C.c_void_p(int(d_rows)), C.c_void_p(int(d_sig)) if d_sig else None))
        return self

    def adjoint(self, g_sigw, seed: int = 0, device: int = 0, stream=None, walker_range=None) -> dict:
        """Gradients of L = sum_j g_sigw[j, 0] C_j + g_sigw[j, 1] S_j (the
        waveform-mode signal sums) for the walk ``run(seed, "split")`` makes;
        see rms_adjoint_run in include/rms.h."""
        if self.wave_shape is None:
            raise ValueError("the adjoint needs a waveform-mode simulation")
        nw, nb, _ = self.wave_shape
        g = _arr(g_sigw)
        if g.size != 2 * nw:
            raise ValueError("g_sigw must hold (cos, sin) weights per waveform")
        opts = _opts(seed, "split", device, stream, walker_range=walker_range)
        dwave = np.zeros(nw * nb * 3)
        sigw = np.zeros(2 * nw)
        out = AdjointGrads(_ptr(dwave), 0.0, 0.0, (C.c_double * 8)(), 0.0, _ptr(sigw), 0.0, 0.0)
        _check(lib().rms_adjoint_run(self._h, C.byref(opts), _ptr(g), C.byref(out)))
        return dict(d_wave=dwave.reshape(nw, nb, 3), d_diffusivity=out.d_diffusivity, d_kappa=out.d_kappa,
                    d_t2=np.array(out.d_t2[:]), loss=out.loss, sigw=sigw.reshape(nw, 2),
                    d_diffusivity_pathwise=out.d_diffusivity_pathwise, d_kappa_score=out.d_kappa_score)

    JAC_COLS = {"D": 0, "kappa": 1, "kappa_score": 2, "T2": 3}

    def jacobian(self, seed: int = 0, device: int = 0, stream=None, walker_range=None) -> dict:
        """d(signal sums)/d(D, kappa, T2) for every waveform in one adjoint run
        (rms_adjoint_jacobian): arrays [nwave, 2] (cos sum, sin sum) per
        parameter -- "D", "kappa" (forced draws), "kappa_score", and "T2"
        [nwave, 2, nc] -- and the run's own sums "sigw" [nwave, 2]."""
        if self.wave_shape is None:
            raise ValueError("the adjoint needs a waveform-mode simulation")
        nw = self.wave_shape[0]
        opts = _opts(seed, "split", device, stream, walker_range=walker_range)
        jac = np.zeros(2 * nw * 11)
        sigw = np.zeros(2 * nw)
        _check(lib().rms_adjoint_jacobian(self._h, C.byref(opts), _ptr(jac), _ptr(sigw)))
        j = jac.reshape(nw, 2, 11)
        nc = self.nc
        return dict(D=j[:, :, 0].copy(), kappa=j[:, :, 1].copy(), kappa_score=j[:, :, 2].copy(),
                    T2=j[:, :, 3:3 + nc].copy(), sigw=sigw.reshape(nw, 2))

    def cumulants(self, dirs=None):
        """(D, K), [timepoints, ndir], along unit directions dirs [ndir, 3]
        (default x, y, z); readRMS.m's formulas, computed in the library."""
        d = None if dirs is None else _arr(dirs)
        ndir = 3 if d is None else d.size // 3
        T = self.field_size("sig0")
        D, K = np.zeros(T * ndir), np.zeros(T * ndir)
        _check(lib().rms_sim_cumulants(self._h, _ptr(d) if d is not None else None, ndir, _ptr(D), _ptr(K)))
        return D.reshape(T, ndir), K.reshape(T, ndir)

    def signal_table(self):
        """(sig, bvec [m, 3], bval [m]) of the last run, formed as the MATLAB
        readers form them: narrow pulses |sigRe| / sig0 [T, m] against bval.txt
        and bvec.txt (readRMS.m:38-48); PGSE |sig| [1, m] (the walker sum, not
        normalised, as readRMS_pgse.m:56 reads it) against
        b = |g|^2 delta^2 (Delta - delta/3) and the gradient directions
        (readRMS_pgse.m:48-53)."""
        from . import analysis
        o = self.outputs()
        if self.mode == "narrow":
            return analysis.narrow_signal(o["sig0"], o["sigre"]), self.get("bvec").reshape(-1, 3), self.get("bval")
        if self.mode == "pgse":
            g = self.get("grad").reshape(-1, 6)
            return np.abs(o["sig"]).reshape(1, -1), g[:, 3:6], analysis.pgse_bval(g)
        raise ValueError("signal tables exist for narrow-pulse and PGSE runs")

    def dki_shell(self, td=None):
        """Shell-wise DKI fit of the last run, dt [T, 21] (rms_dki_shell):
        narrow pulses as readRMS.m's dki_shell (td: the run's diffusion times);
        PGSE as readRMS_pgse.m's, with the intercept column that absorbs the
        walker count, for the diffusion time td of its one row (required)."""
        sig, bvec, bval = self.signal_table()
        if self.mode == "pgse":
            if td is None:
                raise ValueError("a PGSE table has one row: give its diffusion time td")
            return dki_shell(sig, bvec, bval, np.atleast_1d(td), intercept=True)
        return dki_shell(sig, bvec, bval, self.get("td") if td is None else td)

    def dki_lls(self):
        """Linear least-squares DKI fit of the last narrow-pulse run, dt [T, 21]
        (readRMS.m's dki_lls, rms_dki_lls)."""
        if self.mode != "narrow":
            raise ValueError("the LLS fit reads a normalised signal: narrow-pulse runs (or call dki_lls)")
        return dki_lls(*self.signal_table())

    def field_size(self, name: str) -> int:
        n = C.c_size_t()
        _check(lib().rms_sim_field_size(self._h, FIELD[name], C.byref(n)))
        return n.value

    def get(self, name: str) -> np.ndarray:
        n = self.field_size(name)
        out = np.zeros(n)
        _check(lib().rms_sim_get(self._h, FIELD[name], _ptr(out) if n else None, n))
        return out

    def outputs(self) -> dict:
        T = self.field_size("sig0")
        o = dict(sig0=self.get("sig0"), dx2=self.get("dx2").reshape(T, 6),
                 dx4=self.get("dx4").reshape(T, 15), td=self.get("td"))
        nc = self.field_size("diffusivity")
        o["npar_count"] = self.get("npar_count").reshape(T, nc)
        if self.mode == "narrow":
            o["sigre"] = self.get("sigre").reshape(T, -1)
        elif self.mode == "pgse":
            o["sig"] = self.get("sig")
        else:
            o["sigw"] = self.get("sigw").reshape(-1, 2)
        return o

    def trace(self, nwalkers: int) -> dict:
        tr_init = np.zeros(nwalkers, dtype=np.int32)
        vox = np.zeros((nwalkers, self.tn), dtype=np.int32)
        ev = np.zeros((nwalkers, self.tn), dtype=np.uint32)
        _check(lib().rms_sim_get_trace(self._h, tr_init.ctypes.data_as(C.POINTER(C.c_int32)),
                                       vox.ctypes.data_as(C.POINTER(C.c_int32)),
                                       ev.ctypes.data_as(C.POINTER(C.c_uint32)), nwalkers, self.tn))
        pos = np.zeros((nwalkers, self.tn, 3))
        _check(lib().rms_sim_get_trace_positions(self._h, _ptr(pos), nwalkers, self.tn))
        return dict(init_voxel=tr_init, voxel=vox, events=ev, pos=pos)

    def write_dir(self, path: str):
        _check(lib().rms_sim_write_dir(self._h, path.encode()))

    def timing(self):
        """(walk kernel ms, whole run ms) of the last run, from CUDA events."""
        a, b = C.c_double(), C.c_double()
        _check(lib().rms_sim_last_timing(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().rms_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def batch_run(sims, seed: int = 0, precision: str = "compat", device: int = 0, stream=None, variant: int = 0,
              shard=None):
    """Walk a batch of simulations (SPLIT: one persistent launch; COMPAT: one
    launch per simulation).  ``shard`` = (index, count): every simulation
    walks only that shard of its walkers (a rank's part of the batch)."""
    arr = (C.c_void_p * len(sims))(*[s._h.value for s in sims])
    opts = _opts(seed, precision, device, stream, variant=variant, shard=shard)
    _check(lib().rms_batch_run(arr, len(sims), C.byref(opts)))


def contract_phases(d_pos: int, nwalk: int, nbins: int, d_wave: int, nwave: int, d_out: int,
                    method: str = "bf16x3", stream=None) -> float:
    """Multi-waveform phase contraction on device buffers (raw device
    addresses): d_pos float32 [nwalk, nbins, 3], d_wave float32
    [nwave, nbins, 3], d_out float64 [nwave, 2] receives the sums of cos and
    sin of phi = pos . wave.  Returns the kernel's device time (ms)."""
    ms = C.c_float()
    st = None if stream is None else C.c_void_p(int(stream))
    _check(lib().rms_contract_phases(C.c_void_p(int(d_pos)), int(nwalk), int(nbins), C.c_void_p(int(d_wave)),
                                     int(nwave), CONTRACT[method], C.c_void_p(int(d_out)), st, C.byref(ms)))
    return ms.value


def combine_cumulants(f, Ds, Ks):
    """Volume-weighted D, K of several axons (part1_demo4_analysis.m:88-90):
    f [naxons], Ds/Ks [naxons, T, ndir] -> (D, K) [T, ndir]."""
    Ds, Ks = np.asarray(Ds, dtype=np.float64), np.asarray(Ks, dtype=np.float64)
    na, T, nd = Ds.shape
    D, K = np.zeros(T * nd), np.zeros(T * nd)
    _check(lib().rms_combine_cumulants(na, T, nd, _ptr(_arr(f)), _ptr(_arr(Ds)), _ptr(_arr(Ks)), _ptr(D), _ptr(K)))
    return D.reshape(T, nd), K.reshape(T, nd)


def _signal_table(sig, bvec, bval):
    sig = np.atleast_2d(np.asarray(sig, dtype=np.float64))
    bvec = _arr(bvec)
    bval = _arr(bval)
    T, m = sig.shape
    if bvec.size != 3 * m or bval.size != m:
        raise ValueError("sig [T, m] needs bvec [m, 3] and bval [m]")
    return np.ascontiguousarray(sig), bvec, bval, T, m


def dki_shell(sig, bvec, bval, td, intercept=False):
    """Shell-wise DKI fit (readRMS.m:51-78; intercept=True: readRMS_pgse.m:60-89)
    of sig [T, m] (e.g. analysis.narrow_signal): dt [T, 21], the 6 <x^2> and 15
    <x^4> tensor elements per timepoint (rms_dki_shell)."""
    sig, bvec, bval, T, m = _signal_table(sig, bvec, bval)
    tdv = _arr(td)
    if tdv.size != T:
        raise ValueError("td needs one value per timepoint")
    dt = np.zeros(T * 21)
    _check(lib().rms_dki_shell(T, m, _ptr(sig), _ptr(bvec), _ptr(bval), _ptr(tdv), int(bool(intercept)), _ptr(dt)))
    return dt.reshape(T, 21)


def dki_lls(sig, bvec, bval):
    """Linear least-squares DKI fit (readRMS.m:80-91) of sig [T, m]: the 21
    coefficients per timepoint, dt [T, 21] (rms_dki_lls)."""
    sig, bvec, bval, T, m = _signal_table(sig, bvec, bval)
    dt = np.zeros(T * 21)
    _check(lib().rms_dki_lls(T, m, _ptr(sig), _ptr(bvec), _ptr(bval), _ptr(dt)))
    return dt.reshape(T, 21)


def akc_shell(dt, dirs, td):
    """(K, D) [T, ndir] along dirs [ndir, 3] from a shell fit (readRMS.m:105-112)."""
    dt = np.ascontiguousarray(np.atleast_2d(np.asarray(dt, dtype=np.float64)))
    d, tdv = _arr(dirs), _arr(td)
    T, nd = dt.shape[0], d.size // 3
    D, K = np.zeros(T * nd), np.zeros(T * nd)
    _check(lib().rms_akc_shell(T, _ptr(dt), nd, _ptr(d), _ptr(tdv), _ptr(D), _ptr(K)))
    return K.reshape(T, nd), D.reshape(T, nd)


def akc_lls(dt, dirs):
    """(K, D) [T, ndir] along dirs [ndir, 3] from an LLS fit (the DKI signal model)."""
    dt = np.ascontiguousarray(np.atleast_2d(np.asarray(dt, dtype=np.float64)))
    d = _arr(dirs)
    T, nd = dt.shape[0], d.size // 3
    D, K = np.zeros(T * nd), np.zeros(T * nd)
    _check(lib().rms_akc_lls(T, _ptr(dt), nd, _ptr(d), _ptr(D), _ptr(K)))
    return K.reshape(T, nd), D.reshape(T, nd)


class Graph:
    """A batch launch captured as a CUDA graph (rms_batch_graph_create) and
    replayed per seed (rms_graph_run); results land in the simulations."""

    def __init__(self, sims, seed: int = 0, device: int = 0, stream=None, variant: int = 0, shard=None):
        self._h = C.c_void_p()
        self.sims = list(sims)
        arr = (C.c_void_p * len(sims))(*[s._h.value for s in sims])
        opts = _opts(seed, "split", device, stream, variant=variant, shard=shard)
        _check(lib().rms_batch_graph_create(arr, len(sims), C.byref(opts), C.byref(self._h)))

    def run(self, seed: int):
        # the captured launch refers to its simulations: a closed one (or a
        # closed graph) would leave it pointing at freed memory
        if not (self._h and self._h.value):
            raise RmsError(-7, "the graph is closed")
        if any(not (s._h and s._h.value) for s in self.sims):
            raise RmsError(-7, "a simulation of the graph was closed: create the graph again")
        _check(lib().rms_graph_run(self._h, int(seed) & ((1 << 64) - 1)))

    def close(self):
        if self._h and self._h.value:
            lib().rms_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(sims, seed: int = 0, device: int = 0, stream=None, shard=None):
    """(variant, [walk ms per variant]) of the SPLIT walk for this batch; pass
    the variant to run()/batch_run().  Cached per job class."""
    arr = (C.c_void_p * len(sims))(*[s._h.value for s in sims])
    opts = _opts(seed, "split", device, stream, shard=shard)
    v = C.c_int()
    ms = np.zeros(len(split_variants()))
    _check(lib().rms_autotune(arr, len(sims), C.byref(opts), C.byref(v), _ptr(ms)))
    return v.value, ms


def rng_doubles(seed: int, walker: int, n: int) -> np.ndarray:
    out = np.zeros(n)
    _check(lib().rms_rng_doubles(seed, walker, n, _ptr(out)))
    return out


def rng_floats(seed: int, walker: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    _check(lib().rms_rng_floats(seed, walker, n, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def rng_split(seed: int, walker: int, domain: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.float32)
    _check(lib().rms_rng_split(seed, walker, domain, n, out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def philox4x32_10(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    p = C.POINTER(C.c_uint32)
    _check(lib().rms_philox4x32_10(c.ctypes.data_as(p), k.ctypes.data_as(p), out.ctypes.data_as(p)))
    return out


def split_variants():
    """[(k, block, min_blocks_per_sm)] of the SPLIT walk's launch variants."""
    out, k = [], 1
    while True:
        b, m = C.c_int(), C.c_int()
        if lib().rms_split_variant(k, C.byref(b), C.byref(m)) != 0:
            return out
        out.append((k, b.value, m.value))
        k += 1


def version() -> str:
    return lib().rms_version().decode()
