#!/usr/bin/env python
"""Walker-steps/s of the B200 random-walk engine (one JSON line on rank 0).

Workload ``batch`` (default; the batched form the metric names): 64 axons,
lattices of log-uniform voxel counts between 64x64x256 and 256x256x2048,
5e7 walkers per GPU in proportion to intra-axonal volume, D0 ~ U(1.5, 2.5)
um^2/ms and kappa ~ U(0, 0.05) um/ms per axon, 20,000 steps, moments only,
all walked by ONE persistent split-precision launch (rms_batch_run).
Workload ``production``: a 256 x 256 x 2048 label lattice at 0.1 um
(one undulating, caliber-varying axon, label 1, in extra-axonal space, label
2), 1e7 walkers per GPU, 50,000 steps of dt = 2e-4 ms, D = 2 um^2/ms in both
compartments, membrane permeability kappa = 0.01 um/ms, T2 = 80 / 60 ms, and
the PGSE signal of 30 directions x b in {0..5} ms/um^2 x Delta in {4, 5, 6} ms
at delta = 4 ms (540 gradients; Delta + delta fits the 10 ms walk).
``production-full``: the same with Delta in {4, ..., 10} ms (1260 gradients),
which needs 70,000 steps (Delta + delta = 14 ms).
Workload ``single``: the 64 x 64 x 512 single-axon lattice (labels 0/1),
1e5 walkers, 5,000 steps, impermeable, no T2, periodic walls, moments every
10 steps.  Inputs are synthetic and seeded.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-cuda]
                  [--precision split|compat] [--workload batch|production|single|contraction|adjoint]
                  [--scaling strong|weak] [--plain-steps P]

Several ranks (torchrun, one per GPU) split the batch: every rank walks its
shard of every axon's walkers (walker ids, and so random streams, are the whole
job's), and the per-axon sums are added in rank order (--scaling strong, the
default); --scaling weak gives every rank the whole batch on its own seeds.

``value``: walker-steps/s of the whole job, lattice already resident on the
GPU, timed with CUDA events on the launching stream (max over ranks).
``e2e``: the same through the public API with the lattice handed over from
pinned host memory and the results read back (and, with several ranks, summed
across them) every step (host clock around synchronised steps).
``plain``: the plain form on the same job -- the FP64 walk in the reference's
arithmetic (COMPAT), one launch per axon -- timed the same way; the metric is
value / plain.  ``error``: D(t) and K(t) of the timed split walk against the
FP64 replay of the same walkers (oracle), on a walker subset of four axons.
``reference_cuda``: the reference's own CUDA programs (main.cu, main_PGSE.cu
built unchanged for sm_100a) beside rms_main on one run directory each.
``--impl reference`` times the reference simulator's own step loop
(hpc_code/lib/main.cu or main_PGSE.cu compiled for the host, all cores) on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "walker-steps/s on 1 B200 (batched/split-prec vs plain) at stated D(t)/K(t) error"
UNIT = "walker-steps/s"
# Algorithmic work per walker-step (the step kernel's roofline model): one
# label gather per face crossing, 0.73 crossings per step at
# step/voxel = 0.49, each a 32-byte sector -> 23.4 B; 105 thread-ops.
BYTES_PER_WALKER_STEP = 23.4
OPS_PER_WALKER_STEP = 105.0
BATCH_SEED_STEP = 0x9E3779B97F4A7C15   # batch member k walks with seed + k * this (include/rms.h)


def fib_directions(n: int) -> np.ndarray:
    """n near-uniform unit vectors (Fibonacci sphere)."""
    i = np.arange(n) + 0.5
    z = 1.0 - 2.0 * i / n
    r = np.sqrt(1.0 - z * z)
    phi = np.pi * (1.0 + 5 ** 0.5) * i
    return np.column_stack([r * np.cos(phi), r * np.sin(phi), z])


def workload(name: str, world: int, walkers: int | None = None, tn: int | None = None,
             timepoints: int | None = None, scaling: str = "strong"):
    """(lattice(s), Sim keywords, walkers per GPU, config) of a workload; the
    config is the same dict in both arms (this engine and the reference)."""
    lab, sim_kw, per_gpu, cfg = _workload(name, world, scaling)
    if timepoints:
        if isinstance(sim_kw, list):
            sim_kw = [dict(kw, timepoints=int(timepoints)) for kw in sim_kw]
        else:
            sim_kw["timepoints"] = int(timepoints)
        cfg["workload"] += f" [timepoints overridden: {timepoints}]"
    if isinstance(sim_kw, list):
        if walkers:
            scale = walkers / per_gpu
            sim_kw = [dict(kw, npar=max(32, int(kw["npar"] * scale))) for kw in sim_kw]
            per_gpu = sum(kw["npar"] for kw in sim_kw)
            cfg["walkers"] = per_gpu
            cfg["workload"] += f" [walkers overridden: {per_gpu}]"
        if tn:
            sim_kw = [dict(kw, tn=int(tn)) for kw in sim_kw]
            cfg["steps_per_walk"] = int(tn)
            cfg["workload"] += f" [steps overridden: {tn}]"
        return lab, sim_kw, per_gpu, cfg
    if walkers:
        per_gpu = int(walkers)
        sim_kw["npar"] = per_gpu * world
        cfg["walkers_per_gpu"] = per_gpu
        cfg["workload"] += f" [walkers/GPU overridden: {per_gpu}]"
    if tn:
        sim_kw["tn"] = int(tn)
        cfg["steps_per_walk"] = int(tn)
        cfg["workload"] += f" [steps overridden: {tn}]"
    return lab, sim_kw, per_gpu, cfg


def _workload(name: str, world: int, scaling: str = "strong"):
    from rms_b200 import analysis, geometry
    if name in ("production", "production-full"):
        # 50,000 steps of 2e-4 ms walk 10 ms: Delta + delta fits for Delta <= 6 ms.
        # production-full walks the whole Delta range 4..10 ms: 70,000 steps.
        full = name == "production-full"
        tn = 70_000 if full else 50_000
        deltas = (4.0, 5.0, 6.0, 7.0, 8.0, 9.0, 10.0) if full else (4.0, 5.0, 6.0)
        lab = geometry.axon_lattice(256, 256, 2048, 0.1, seed=0, exterior=2)
        dirs = fib_directions(30)
        rows = []
        for Delta in deltas:
            for b in (0.0, 1.0, 2.0, 3.0, 4.0, 5.0):
                g = float(analysis.pgse_gradient_for_b(b, Delta, 4.0))
                for d in dirs:
                    rows.append([Delta, 4.0, g, *d])
        per_gpu = 10_000_000
        sim_kw = dict(dt=2e-4, tn=tn, npar=per_gpu * world, res=0.1,
                      diffusivity=[0.0, 2.0, 2.0], t2=[80.0, 80.0, 60.0],
                      grad=np.array(rows), permeation="kappa", kappa=0.01)
        cfg = dict(workload=f"{name}: 256x256x2048 lattice, 1e7 walkers/GPU, {tn} steps, "
                            f"kappa=0.01 um/ms, T2 80/60 ms, PGSE {len(rows)} gradients "
                            f"(Delta {deltas[0]:g}..{deltas[-1]:g} ms, delta 4 ms)",
                   lattice=[256, 256, 2048], walkers_per_gpu=per_gpu, steps_per_walk=tn,
                   ngrad=len(rows), mode="pgse",
                   l2="flushed between timed steps (256 MiB write); the packed lattice is 68 MB",
                   parallelism=f"walker shards x{world} (weak: 1e7 walkers per rank)")
    elif name == "batch":
        # 64 axons, lattices of log-uniform voxel counts between 64x64x256 and
        # 256x256x2048, walkers proportional to the intra-axonal volume (5e7 in
        # all), D0 ~ U(1.5, 2.5) um^2/ms and kappa ~ U(0, 0.05) um/ms per axon
        rng = np.random.default_rng(2)
        shapes = geometry.batch_sizes(64, seed=0)
        lattices = [geometry.axon_lattice(*shp, 0.1, seed=100 + k, exterior=2) for k, shp in enumerate(shapes)]
        intra = np.array([max(1, int(np.count_nonzero(l == 1))) for l in lattices], dtype=np.float64)
        total = 50_000_000
        npar = np.maximum(32, np.round(total * intra / intra.sum()).astype(np.int64))
        D0 = rng.uniform(1.5, 2.5, 64)
        kap = rng.uniform(0.0, 0.05, 64)
        sims_kw = [dict(dt=2e-4, tn=20_000, npar=int(npar[k]), res=0.1,
                        diffusivity=[0.0, float(D0[k]), float(D0[k])], t2=[1e12, 1e12, 1e12],
                        bval=[], bvec=np.zeros((0, 3)), permeation="kappa", kappa=float(kap[k]))
                   for k in range(64)]
        weak = scaling == "weak"
        cfg = dict(workload="batch: 64 axons, lattices 64x64x256..256x256x2048 (log-uniform voxels), "
                            "5e7 walkers in proportion to intra-axonal volume, D0~U(1.5,2.5), "
                            "kappa~U(0,0.05), 20000 steps, moments only",
                   axons=64, lattice_voxels=int(sum(l.size for l in lattices)),
                   walkers=int(npar.sum()) * (world if weak else 1), steps_per_walk=20_000,
                   mode="narrow (no b-table)",
                   l2="flushed between timed steps (256 MiB write); the 64 lattices (1.71 GB) are larger than L2",
                   parallelism=(f"{world} rank(s), each walking the whole batch on its own seeds (weak)" if weak else
                                f"{world} rank(s), each walking its 1/{world} shard of every axon's walkers "
                                "(strong; per-axon sums added in rank order)"))
        return lattices, sims_kw, int(npar.sum()), cfg
    elif name == "single":
        lab = geometry.axon_lattice(64, 64, 512, 0.1, seed=0, exterior=0)
        per_gpu = 100_000
        sim_kw = dict(dt=2e-4, tn=5_000, npar=per_gpu * world, res=0.1, diffusivity=[0.0, 2.0],
                      t2=[1e12, 1e12], bval=[], bvec=np.zeros((0, 3)), timepoints=500,
                      boundary="periodic")
        cfg = dict(workload="single: 64x64x512 axon, 1e5 walkers/GPU, 5000 steps, moments every 10 steps",
                   lattice=[64, 64, 512], walkers_per_gpu=per_gpu, steps_per_walk=5_000,
                   mode="narrow", l2="flushed between timed steps (256 MiB write)",
                   parallelism=f"walker shards x{world} (weak: 1e5 walkers per rank)")
    else:
        raise SystemExit(f"unknown workload {name}")
    return lab, sim_kw, per_gpu, cfg


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        mhz, maxmhz, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                maxmhz = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not mhz:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": maxmhz, "reasons": sorted(reasons),
                "samples": len(mhz)}


def cpu_reference_rate(lab, sim_kw, target_s: float, nthreads: int | None = None):
    """The reference's own step loop (oracle/_ref: hpc_code/lib/main_PGSE.cu or
    main.cu compiled for the host) on the first n walkers of the job, all
    cores; n is chosen so one sample takes about target_s seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    dt, tn = sim_kw["dt"], sim_kw["tn"]
    # the derived tables (main.cu:433-458; the kappa rule of interaction.m:437-439)
    # from the oracle: this arm loads nothing of the engine
    kap = sim_kw.get("kappa") if sim_kw.get("permeation") == "kappa" else None
    step, t2s, pij, _ = pyoracle.reference_tables(dt, sim_kw["res"], sim_kw["diffusivity"], sim_kw["t2"],
                                                  kappa=kap)
    timepoints = sim_kw.get("timepoints", 0) or 1000
    kw = dict(dt=dt, tn=tn, npar=sim_kw["npar"], res=sim_kw["res"], step=step, t2_steps=t2s,
              pij=pij, seed=1, timepoints=1000)
    if "grad" in sim_kw:
        job = pyoracle.Job(lab, grad=sim_kw["grad"], **kw)
    else:
        job = pyoracle.Job(lab, bval=sim_kw.get("bval", []), bvec=sim_kw.get("bvec", np.zeros((0, 3))), **kw)
    kind = "reference"
    if not pyoracle.ref_available():
        raise RuntimeError("oracle/_ref/librmsref.so missing")
    if timepoints != 1000 or sim_kw.get("boundary", "mirror") != "mirror":
        # the reference build has fixed 1000 records and mirror walls: time its loop as is
        pass
    nthreads = nthreads or pyoracle.ref_max_threads()
    # probe with doubling walker counts until a probe lasts a second, then scale
    n = 2 * nthreads
    while True:
        t0 = time.perf_counter()
        pyoracle.run_reference_walkers(job, n, nthreads)
        dt_probe = time.perf_counter() - t0
        if dt_probe >= 1.0 or n >= job.npar:
            break
        n = min(job.npar, 2 * n)
    n = int(max(nthreads, min(job.npar, n * target_s / max(dt_probe, 1e-3))))
    return job, n, nthreads, kind


def run_reference_cuda(args):
    """The reference's own CUDA programs beside this engine's drop-in, process
    against process on one run directory each: main.cu and main_PGSE.cu built
    unchanged for sm_100a (oracle/_ref/main_cuda, main_pgse_cuda) and rms_main
    (split and compat precision).  Workload: the 64x64x512 single-axon lattice
    in the reference's file contract (mirror walls, 1000 records), 1e6 walkers
    x 5000 steps; narrow pulses b = 1, 2 ms/um^2 along x and z, and PGSE with
    6 directions x b = 1, 2 ms/um^2 at Delta = 0.6 ms, delta = 0.2 ms.  Each
    process is timed by the wall clock: all read fiber.txt, create a CUDA
    context, walk, and write the output files.  D(t) and K(t) along x and z at
    the last record come from each one's output files (readRMS.m formulas); the
    reference seeds cuRAND from /dev/random, so they agree within Monte-Carlo
    error, not bit for bit."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    npar, tn = args.walkers or args.refcuda_walkers, args.tn or 5_000
    runs = reference_cuda_runs(npar, tn)
    ref = runs.get("reference main.cu", {}) if isinstance(runs, dict) else {}
    line = {"metric": METRIC, "value": ref.get("walker_steps_per_s"), "unit": UNIT, "n_gpus": 1,
            "higher_is_better": True, "impl": "reference-cuda", "data": "synthetic (seeded)",
            "config": {"workload": f"64x64x512 axon (mirror walls, 1000 records), {npar} walkers, {tn} steps: "
                                   "the reference's CUDA programs (narrow pulse, PGSE) and rms_main on the same "
                                   "run directories, wall time per process (text I/O and context creation included)"},
            "runs": runs}
    print(json.dumps(line), flush=True)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    world = int(os.environ.get("WORLD_SIZE", "1"))
    lab, sim_kw, per_gpu, cfg = workload(args.workload, world, args.walkers, args.tn, args.timepoints,
                                         args.scaling)
    if isinstance(lab, list):
        # a batch: time the reference loop on the axon with the most walkers
        k = int(np.argmax([kw["npar"] for kw in sim_kw]))
        lab, sim_kw = lab[k], sim_kw[k]
    try:
        job, n, cores, kind = cpu_reference_rate(lab, sim_kw, target_s=6.0)
    except Exception as e:  # the build is missing on this machine
        print(json.dumps({"impl": "reference", "unavailable": f"reference host build: {e}"}))
        return
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        pyoracle.run_reference_walkers(job, n, cores)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    per_step = float(np.mean(times))
    rate = n * job.tn / per_step
    sample = (f"walkers [0,{n}) of the job x {job.tn} steps per timed step, reference "
              f"propagate() (oracle/_ref) on {cores} host threads")
    line = {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True,
        "scaling": args.scaling if args.workload == "batch" else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": cfg, "impl": "reference",
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


class SingleJob:
    """One simulation; rank r walks walker shard r of a world * per_gpu job."""

    def __init__(self, lab, kw, per_gpu, rank, device, stream):
        from rms_b200 import engine, shards
        self.lab, self.kw = lab, kw
        self.w0, self.w1 = shards.walker_shard(per_gpu, rank)
        self.sim = engine.Sim(lab, **kw)
        self.device, self.stream = device, stream
        self.walker_steps = (self.w1 - self.w0) * kw["tn"]
        self.launches_per_step = 1
        self.pinned = None

    def tune(self, precision):
        # SPLIT: the walk kernel alone (rows added into the totals);
        # COMPAT: the walk, then the ordered reduce of the rows (and of the signals)
        if precision == "compat":
            self.launches_per_step = 2 + (1 if self.sim.mode == "pgse" else 0)

    def run(self, seed, precision):
        self.sim.run(seed=seed, precision=precision, device=self.device, stream=self.stream,
                     walker_range=(self.w0, self.w1))

    def walk_ms(self):
        return self.sim.timing()[0]

    def pin_inputs(self):
        """The caller's input lattice in pinned host memory (made before the
        end-to-end timing: it stands for inputs the caller already holds)."""
        import torch
        if self.pinned is None:
            self.pinned = torch.from_numpy(np.ascontiguousarray(self.lab)).pin_memory().numpy()

    def reload_inputs(self):
        self.pin_inputs()
        self.sim.set_lattice(self.pinned)

    def outputs(self):
        return self.sim.outputs()

    def input_bytes(self):
        return int(self.lab.nbytes)

    def cpu_case(self):
        return self.lab, self.kw

    def close(self):
        self.sim.close()


class BatchJob:
    """Many axons walked by one launch (rms_batch_run, or its captured CUDA
    graph).  Strong scaling: rank r walks shard r of every axon's walkers, so
    the ranks together walk the one job once.  Weak scaling: every rank walks
    the whole batch on its own seeds."""

    def __init__(self, labs, kws, rank, world, device, stream, scaling="strong"):
        from rms_b200 import engine
        self.engine = engine
        self.labs, self.kws = labs, kws
        self.sims = [engine.Sim(l, **kw) for l, kw in zip(labs, kws)]
        self.rank, self.world, self.device, self.stream = rank, world, device, stream
        self.weak = scaling == "weak"
        self.shard = None if (self.weak or world == 1) else (rank, world)
        self.seed_offset = (rank << 40) if self.weak else 0
        if self.shard is None:
            self.walker_steps = sum(kw["npar"] * kw["tn"] for kw in kws)
        else:
            self.walker_steps = sum((kw["npar"] * (rank + 1) // world - kw["npar"] * rank // world) * kw["tn"]
                                    for kw in kws)
        # split: one persistent walk (multi-axon launches sum into the axon
        # totals, no separate reduction); compat: one walk + one reduction per axon
        self.launches_per_step = 1
        self.pinned = None
        self.variant, self.variant_ms = 0, None
        self.graph = None

    def tune(self, precision):
        """Pick the split walk's launch variant for this batch (rms_autotune)
        and capture the batch launch as a CUDA graph (rms_batch_graph_create)."""
        if precision == "split":
            self.variant, self.variant_ms = self.engine.autotune(self.sims, seed=1, device=self.device,
                                                                  stream=self.stream, shard=self.shard)
            self.graph = self.engine.Graph(self.sims, seed=0, device=self.device, stream=self.stream,
                                           variant=self.variant, shard=self.shard)
        else:
            self.launches_per_step = 2 * len(self.sims)

    def run(self, seed, precision):
        if self.graph is not None and precision == "split":
            self.graph.run(seed + self.seed_offset)
            return
        self.engine.batch_run(self.sims, seed=seed + self.seed_offset, precision=precision,
                              device=self.device, stream=self.stream,
                              variant=self.variant if precision == "split" else 0, shard=self.shard)

    def walk_ms(self):
        return self.sims[0].timing()[0]

    def pin_inputs(self):
        """The caller's input lattices in pinned host memory (made before the
        end-to-end timing: they stand for inputs the caller already holds)."""
        import torch
        if self.pinned is None:
            self.pinned = [torch.from_numpy(np.ascontiguousarray(l)).pin_memory().numpy() for l in self.labs]

    def reload_inputs(self):
        if self.graph is not None:
            self.graph.close()   # a new lattice ends the captured launch: e2e walks through rms_batch_run
            self.graph = None
        self.pin_inputs()
        for sim, lab in zip(self.sims, self.pinned):
            sim.set_lattice(lab)

    def outputs(self):
        out = {}
        for k, sim in enumerate(self.sims):
            for f, v in sim.outputs().items():
                out[f"{k}/{f}"] = v
        return out

    def input_bytes(self):
        return int(sum(l.nbytes for l in self.labs))

    def cpu_case(self):
        k = int(np.argmax([kw["npar"] for kw in self.kws]))
        return self.labs[k], self.kws[k]

    def error_vs_fp64(self, seed, nsub=16384, axons=None, nthreads=None):
        """D(t), K(t) of the split walk against the oracle's FP64 replay of
        the same walkers: walkers [0, nsub) of four axons (the smallest, two
        in between, the largest lattice), walked with the seed the timed step
        gave each axon.  Bar: D within 0.5 %, K within 2 % (absolute 0.02
        where |K| < 1), records 50 on."""
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle
        from rms_b200 import analysis
        sizes = np.array([l.size for l in self.labs])
        order = np.argsort(sizes, kind="stable")
        if axons is None:
            axons = sorted({int(order[0]), int(order[len(order) // 3]), int(order[2 * len(order) // 3]),
                            int(order[-1])})
        nthreads = nthreads or os.cpu_count() or 1
        per_axon, dD_max, dK_max = [], 0.0, 0.0
        sl = slice(50, None)
        for k in axons:
            kw, sim = self.kws[k], self.sims[k]
            n = int(min(nsub, kw["npar"]))
            sk = (seed + self.seed_offset + k * BATCH_SEED_STEP) & ((1 << 64) - 1)
            got = sim.run(seed=sk, precision="split", device=self.device, stream=self.stream,
                          walker_range=(0, n)).outputs()
            kap = kw["kappa"] if kw.get("permeation") == "kappa" else None
            step, t2s, pij, td = pyoracle.reference_tables(kw["dt"], kw["res"], kw["diffusivity"], kw["t2"],
                                                           1000, kw["tn"], kappa=kap)
            job = pyoracle.Job(self.labs[k], dt=kw["dt"], tn=kw["tn"], npar=kw["npar"], res=kw["res"], step=step,
                               t2_steps=t2s, pij=pij, seed=sk, td=td, bval=[], bvec=np.zeros((0, 3)))
            t0 = time.perf_counter()
            want = pyoracle.run_oracle(job, 0, n, nthreads=nthreads, split=True)
            cpu_s = time.perf_counter() - t0
            Dg, Kg = analysis.axis_dk(got["sig0"], got["dx2"], got["dx4"], got["td"])
            Dw, Kw = analysis.axis_dk(want["sig0"], want["dx2"], want["dx4"], got["td"])
            dD = float(np.abs(Dg[sl] / Dw[sl] - 1).max())
            dK = float((np.abs(Kg[sl] - Kw[sl]) / np.maximum(np.abs(Kw[sl]), 1.0)).max())
            counts_equal = bool(np.array_equal(got["npar_count"].sum(axis=1), want["npar_count"].sum(axis=1)))
            per_axon.append({"axon": int(k), "lattice": list(self.labs[k].shape), "walkers": n,
                             "dD_rel": dD, "dK": dK, "D_late": [round(float(x), 5) for x in Dw[-1]],
                             "K_late": [round(float(x), 4) for x in Kw[-1]], "walker_count_conserved": counts_equal,
                             "replay_s": round(cpu_s, 2)})
            dD_max, dK_max = max(dD_max, dD), max(dK_max, dK)
        return {"dD_max": dD_max, "dK_max": dK_max, "bar": {"dD": 0.005, "dK": 0.02},
                "within_bar": bool(dD_max <= 0.005 and dK_max <= 0.02),
                "against": "FP64 replay of the same walkers and random streams (oracle or_run_split)",
                "definition": "max over records 50..999 and axes x, y, z of |D/D64 - 1| and "
                              "|K - K64| / max(|K64|, 1)",
                "steps_per_walk": int(self.kws[0]["tn"]), "per_axon": per_axon}

    def close(self):
        if self.graph is not None:
            self.graph.close()
        for sim in self.sims:
            sim.close()


def issue_peak(sm_mhz):
    """Thread-instruction issue peak of a B200: 148 SMs x 4 schedulers x 32
    lanes per clock, at the SM clock sampled during the timed region."""
    return 148 * 4 * 32 * (sm_mhz or 1965.0) * 1e6


def profile_figures(precision, workload):
    """Per-walker-step figures of the ncu capture summarised in profiles/
    (measured on a smaller case of the same kernel and workload shape)."""
    out = {}
    prof = os.path.join(ROOT, "profiles", f"walk_{precision}_kernel__{workload}.md")
    if os.path.exists(prof):
        for ln in open(prof):
            for key in ("traffic_bytes_per_walker_step", "warp_inst_per_warp_step", "issue_active"):
                if ln.startswith(key + ":"):
                    out[key] = float(ln.split(":")[1].split()[0])
    return out


def reference_cuda_runs(npar, tn, nthreads=None):
    """The reference's own CUDA programs beside rms_main, process against
    process: see run_reference_cuda.  Returns the runs dict."""
    exe = os.path.join(ROOT, "oracle", "_ref", "main_cuda")
    exe_pgse = os.path.join(ROOT, "oracle", "_ref", "main_pgse_cuda")
    ours = os.path.join(ROOT, "monte-carlo-simulation-3d-rms_b200", "_build", "rms_main")
    import shutil
    import tempfile
    from rms_b200 import analysis, geometry, runio
    if not (os.path.exists(exe) and os.path.exists(exe_pgse) and os.path.exists(ours)):
        return {"unavailable": "oracle/_ref/main_cuda, main_pgse_cuda or rms_main not built"}
    lab = geometry.axon_lattice(64, 64, 512, 0.1, seed=0, exterior=0)
    base = dict(dt=2e-4, tn=tn, npar=npar, res=0.1, diffusivity=[0.0, 2.0], t2=[1e12, 1e12])
    narrow = dict(base, bval=[1.0, 2.0], bvec=[[1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    # PGSE: 6 directions x b in {1, 2} ms/um^2 at Delta = 0.6 ms, delta = 0.2 ms (fits the 1 ms walk)
    dirs = fib_directions(6)
    from rms_b200 import analysis as an
    grad = np.array([[0.6, 0.2, float(an.pgse_gradient_for_b(b, 0.6, 0.2)), *d] for b in (1.0, 2.0) for d in dirs])
    pgse = dict(base, grad=grad)
    top = tempfile.mkdtemp(prefix="rms_refcuda_")
    runs = {}
    try:
        for name, cmd, kw in (("reference main.cu", [exe], narrow),
                              ("rms_main split (narrow)", [ours, "--precision", "split", "--seed", "7"], narrow),
                              ("rms_main compat (narrow)", [ours, "--precision", "compat", "--seed", "7"], narrow),
                              ("reference main_PGSE.cu", [exe_pgse], pgse),
                              ("rms_main split (pgse)", [ours, "--precision", "split", "--seed", "7"], pgse),
                              ("rms_main compat (pgse)", [ours, "--precision", "compat", "--seed", "7"], pgse)):
            d = os.path.join(top, "".join(c if c.isalnum() else "_" for c in name))
            runio.write_inputs(d, lab, lattice="txt", **kw)
            t0 = time.perf_counter()
            try:
                r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=900)
            except subprocess.TimeoutExpired:
                runs[name] = {"error": "timed out after 900 s"}
                continue
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                runs[name] = {"error": f"exit {r.returncode}: {(r.stderr or r.stdout)[-300:]}"}
                continue
            sig0 = np.loadtxt(os.path.join(d, "sig0.txt"))
            dx2 = np.loadtxt(os.path.join(d, "dx2.txt"))
            dx4 = np.loadtxt(os.path.join(d, "dx4.txt"))
            td = np.loadtxt(os.path.join(d, "diff_time.txt"))
            D, K = analysis.axis_dk(sig0, dx2, dx4, td)
            runs[name] = {"wall_s": round(wall, 3), "walker_steps_per_s": npar * tn / wall,
                          "D_x": float(D[-1, 0]), "D_z": float(D[-1, 2]),
                          "K_x": float(K[-1, 0]), "K_z": float(K[-1, 2])}
            if "grad" in kw:
                sig = np.atleast_1d(np.loadtxt(os.path.join(d, "sig.txt")))
                runs[name]["S_over_S0"] = [round(float(x), 5) for x in sig / sig0[-1]]
    finally:
        shutil.rmtree(top, ignore_errors=True)
    for prog in ("narrow", "pgse"):
        ref = runs.get("reference main.cu" if prog == "narrow" else "reference main_PGSE.cu", {})
        ours_s = runs.get(f"rms_main split ({prog})", {})
        if ref.get("wall_s") and ours_s.get("wall_s"):
            runs[f"process_ratio_split_{prog}"] = ref["wall_s"] / ours_s["wall_s"]
    return runs


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    # under torchrun the ranks' exchange goes through NCCL even for one rank,
    # so a one-GPU torchrun run walks the same code path as several GPUs
    dist_on = world > 1 or "TORCHELASTIC_RUN_ID" in os.environ
    if dist_on:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    lab, sim_kw, per_gpu, cfg = workload(args.workload, world, args.walkers, args.tn, args.timepoints,
                                         args.scaling)
    stream = torch.cuda.current_stream()
    sh = stream.cuda_stream
    batch = isinstance(lab, list)
    if batch:
        job = BatchJob(lab, sim_kw, rank, world, local, sh, scaling=args.scaling)
    else:
        job = SingleJob(lab, sim_kw, per_gpu, rank, local, sh)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    precision = args.precision

    def barrier():
        if dist_on:
            dist.barrier()

    def max_over_ranks(*vals):
        if not dist_on:
            return vals
        t = torch.tensor(vals, dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return tuple(float(x) for x in t)

    def sum_over_ranks(x):
        if not dist_on:
            return x
        t = torch.tensor([float(x)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        return float(t[0])

    # every rank's walker-steps, summed: the units all ranks walked per step
    total_walker_steps = sum_over_ranks(job.walker_steps)

    if hasattr(job, "tune"):
        job.tune(precision)   # outside the timed region
    for i in range(args.warmup):
        job.run(1000 + i, precision)
    walk_ms = []
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    timed_seed = 2000
    with ClockSampler(local) as clk:
        e0.record(stream)
        for i in range(args.steps):
            flush.zero_()
            job.run(timed_seed + i, precision)
            walk_ms.append(job.walk_ms())
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms, walk = max_over_ranks(e0.elapsed_time(e1) / args.steps, float(np.mean(walk_ms)))
    value = total_walker_steps / (ms * 1e-3)
    clocks = clk.summary()

    # the plain form on the same job: the FP64 walk in the reference's
    # arithmetic (COMPAT), one launch per axon, each rank its own shard
    plain = None
    if args.plain_steps > 0 and precision == "split":
        if batch:
            small = int(np.argmin([l.size for l in job.labs]))
            job.sims[small].run(seed=999, precision="compat", device=local, stream=sh,
                                walker_range=(0, min(4096, job.kws[small]["npar"])))   # module load, untimed
        else:
            job.run(999, "compat")
        pms = []
        for i in range(args.plain_steps):
            barrier()
            torch.cuda.synchronize()
            flush.zero_()
            e0.record(stream)
            job.run(timed_seed + i, "compat")
            e1.record(stream)
            torch.cuda.synchronize()
            pms.append(e0.elapsed_time(e1))
        (pms_max,) = max_over_ranks(float(np.mean(pms)))
        pval = total_walker_steps / (pms_max * 1e-3)
        plain = {"value": pval, "unit": UNIT, "ms_per_step": pms_max, "steps": args.plain_steps,
                 "form": "COMPAT: FP64 positions and sums in the reference's operation order, one launch "
                         "(walk + ordered reduction) per axon, the same walkers and seeds",
                 "batched_split_over_plain": value / pval, "target": 3.0}

    # end to end through the public API: lattices from pinned host memory,
    # results read back (and summed across ranks), every step
    e2e_steps = max(1, min(args.steps, 3))
    job.pin_inputs()
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        job.reload_inputs()
        job.run(3000 + i, precision)
        out = job.outputs()
        if dist_on:
            # the whole job's result: rank-order sum of the shards' accumulators
            from rms_b200 import shards
            out = shards.gather_sum({k: v for k, v in out.items() if not k.endswith("td")}, device="cuda")
    torch.cuda.synchronize()
    (e2e_s,) = max_over_ranks((time.perf_counter() - t0) / e2e_steps)
    d2h = int(sum(v.nbytes for v in out.values()))
    h2d = job.input_bytes()

    # the split walk's D(t), K(t) error against the FP64 replay (rank 0, one GPU)
    error = None
    if batch and precision == "split" and rank == 0 and world == 1 and not args.no_error:
        error = job.error_vs_fp64(timed_seed)

    # roofline of the walk kernel (the dominant launch): issue-bound (the
    # algorithmic thread-op model against the issue peak), with the byte model
    # and the measured DRAM traffic beside it
    walker_steps = job.walker_steps
    prof = profile_figures(precision, args.workload)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    ops_rate = walker_steps * OPS_PER_WALKER_STEP / (walk * 1e-3)
    ipeak = issue_peak(clocks.get("sm_mhz"))
    traffic = prof["traffic_bytes_per_walker_step"] * walker_steps if "traffic_bytes_per_walker_step" in prof else None
    roofline = {
        "bound": "issue", "achieved": ops_rate / 1e12, "peak": ipeak / 1e12, "unit": "T thread-op/s",
        "frac": ops_rate / ipeak, "traffic": traffic,
        "model": f"{OPS_PER_WALKER_STEP:.0f} algorithmic thread-ops/walker-step x {walker_steps:.3g} walker-steps / "
                 f"walk kernel {walk:.1f} ms; peak 148 SM x 128 lanes x {clocks.get('sm_mhz') or 1965:.0f} MHz",
        "executed": ({"warp_inst_per_warp_step": prof["warp_inst_per_warp_step"],
                      "issue_slot_frac": walker_steps / 32 * prof["warp_inst_per_warp_step"] / (walk * 1e-3)
                                         / (ipeak / 32),
                      "source": f"ncu smsp__inst_executed, profiles/walk_{precision}_kernel__{args.workload}.md"}
                     if "warp_inst_per_warp_step" in prof else None),
        "bytes": {"model_gbs": walker_steps * BYTES_PER_WALKER_STEP / (walk * 1e-3) / 1e9,
                  "model": f"{BYTES_PER_WALKER_STEP} B/walker-step (0.73 label gathers x 32 B sector)",
                  "measured_dram_gbs": (traffic / (walk * 1e-3) / 1e9) if traffic else None,
                  "hbm_peak_gbs": hbm_peak,
                  "peak_source": "measured hbm_gbs" if "hbm_gbs" in peaks else "fallback"},
    }

    refcuda = None
    if rank == 0 and world == 1 and not args.no_reference_cuda and args.workload == "batch":
        refcuda = reference_cuda_runs(args.refcuda_walkers, 5000)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                sys.path.insert(0, os.path.join(ROOT, "oracle"))
                import pyoracle
                clab, ckw = job.cpu_case()
                cjob, n, cores, kind = cpu_reference_rate(clab, ckw, target_s=15.0)
                t0 = time.perf_counter()
                pyoracle.run_reference_walkers(cjob, n, cores)
                el = time.perf_counter() - t0
                cpu = {"value": n * cjob.tn / el, "unit": UNIT, "cores": cores, "kind": kind,
                       "sample": f"walkers [0,{n}) x {cjob.tn} steps of the axon with the most walkers, reference "
                                 f"propagate() (oracle/_ref) on {cores} host threads, {el:.1f} s"}
            except Exception as e:
                cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": args.scaling if batch else "weak",
            "vs_baseline": None, "dtype": "f64" if precision == "compat" else "f32+i32 (f64 sums)",
            "data": "synthetic (seeded axon lattices)",
            "config": cfg,
            "setup": dict(precision=precision,
                          **({"launch": "CUDA graph replay (rms_graph_run) of one persistent split launch",
                              "launch_variant": int(job.variant),
                              "autotune_walk_ms": [round(float(x), 2) for x in job.variant_ms]}
                             if getattr(job, "variant_ms", None) is not None else {})),
            "roofline": roofline,
            "walk_ms": walk,
            "plain": plain,
            "error": error,
            "e2e": {"value": total_walker_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": job.launches_per_step * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "reference_cuda": refcuda,
        }
        print(json.dumps(line), flush=True)
    job.close()
    if dist_on:
        dist.destroy_process_group()


ADJOINT_METRIC = ("walker-steps/s of the forward walk differentiated by the adjoint (all its passes in the "
                  "time) of the waveform-mode signal")


def run_adjoint_bench(args):
    """Gradients of the waveform signal: the 64x64x512 single-axon lattice
    with a label-2 exterior (periodic walls), 1e6 walkers, dt = 2e-4 ms, 5000
    steps, one smooth random gradient waveform of 1000 bins x 3 axes
    (|gamma g| <= 0.0214 rad/(um ms), i.e. 80 mT/m) turned to 16 directions,
    D = 2 um^2/ms, kappa = 0.02 um/ms, T2 = 80 / 60 ms.  Times the forward walk
    and the adjoint, and checks every gradient against a central finite
    difference with common random numbers (h = 1e-3 relative)."""
    import torch
    from rms_b200 import engine, geometry, waveforms
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    npar = args.walkers or 1_000_000
    dt, tn, nb, nw = 2e-4, 5000, 1000, 16
    lab = geometry.axon_lattice(64, 64, 512, 0.1, seed=0, exterior=2)
    g = waveforms.random_smooth(1, nb, 0.0214, seed=3)[0]
    rng = np.random.default_rng(1)
    R = np.stack([np.linalg.qr(rng.normal(size=(3, 3)))[0] for _ in range(nw)])
    W = rng.normal(size=(nw, 2))
    par = dict(D=2.0, kappa=0.02, t2=np.array([1e6, 80.0, 60.0]))

    def sim(gg, D, kappa, t2):
        return engine.Sim(lab, dt=dt, tn=tn, npar=npar, res=0.1, diffusivity=[0.0, D, D], t2=list(t2),
                          wave=np.einsum("jab,nb->jna", R, gg), timepoints=1000, boundary="periodic",
                          permeation="kappa", kappa=kappa)

    if args.launches_once:
        # one forward walk, one weighted reverse pass and one Jacobian, nothing
        # else: the launch list of the job for a profiler
        s1 = sim(g, **par)
        s1.run(seed=9, precision="split")
        fwd = s1.timing()[0]
        s1.adjoint(W.reshape(-1) / npar, seed=9)
        adj = s1.timing()[0]
        s1.jacobian(seed=9)
        print(json.dumps({"workload": "adjoint, one of each", "walkers": npar, "forward_ms": fwd, "adjoint_ms": adj,
                          "jacobian_ms": s1.timing()[0]}), flush=True)
        return

    def signal(gg=g, D=par["D"], kappa=par["kappa"], t2=par["t2"], seed=9):
        """Normalised signal per direction, [nw, 2] (cos, sin sums / walkers)."""
        s_ = sim(gg, D, kappa, t2)
        s_.run(seed=seed, precision="split")
        v = s_.get("sigw").reshape(-1, 2) / npar
        s_.close()
        return v

    def loss(**kw):
        return float((signal(**kw) * W).sum())

    s0 = sim(g, **par)
    for _ in range(args.warmup):
        s0.run(seed=9, precision="split")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s0.run(seed=9, precision="split")
    fwd_s = time.perf_counter() - t0
    fwd_ms = s0.timing()[0]
    for _ in range(args.warmup):
        s0.adjoint(W.reshape(-1) / npar, seed=9)   # allocates the reverse pass's records once
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = s0.adjoint(W.reshape(-1) / npar, seed=9)
    adj_s = time.perf_counter() - t0
    adj_ms = s0.timing()[0]
    dg = np.einsum("jab,jna->nb", R, r["d_wave"])      # chain rule through the rotations
    h = 1e-3
    d = np.random.default_rng(4).normal(size=g.shape) * np.abs(g).max()
    checks = {}
    fd_dir = (loss(gg=g + h * d) - loss(gg=g - h * d)) / (2 * h)
    checks["waveform (random direction)"] = (float((dg * d).sum()), fd_dir)
    for c in (1, 2):
        t2p, t2m = par["t2"].copy(), par["t2"].copy()
        t2p[c] *= 1 + h
        t2m[c] *= 1 - h
        checks[f"T2[{c}]"] = (float(r["d_t2"][c]), (loss(t2=t2p) - loss(t2=t2m)) / (2 * h * par["t2"][c]))
    checks["D"] = (r["d_diffusivity"], (loss(D=2.0 * (1 + h)) - loss(D=2.0 * (1 - h))) / (2 * h * 2.0))
    checks["kappa"] = (r["d_kappa"], (loss(kappa=0.02 * (1 + h)) - loss(kappa=0.02 * (1 - h))) / (2 * h * 0.02))
    out = {k: {"adjoint": a, "finite_difference": f, "rel_err": abs(a / f - 1) if f else None}
           for k, (a, f) in checks.items()}
    # D and kappa act through discontinuous events (crossing decisions, face
    # hits at voxel corners): the h = 1e-3 difference is dominated by those
    # jumps, so a least-squares slope over +-5 % (7 points, same seed) is
    # reported beside it
    for k, x0, f in (("D", 2.0, lambda x: loss(D=x)), ("kappa", 0.02, lambda x: loss(kappa=x))):
        xs = x0 * (1 + 0.05 * np.linspace(-1, 1, 7))
        coef, cov = np.polyfit(xs, [f(x) for x in xs], 1, cov=True)
        sl = float(coef[0])
        out[k]["slope_5pct"] = sl
        out[k]["slope_std_err"] = float(np.sqrt(cov[0, 0]))   # from the fit's residuals (jumps)
        out[k]["rel_err_vs_slope"] = abs(out[k]["adjoint"] / sl - 1) if sl else None
    # spread of the Monte Carlo estimators: the same walkers as 8 shards, each
    # shard's gradient scaled to the whole job; standard error of their mean
    shard_g = {"D": [], "D_pathwise": [], "kappa": []}
    for k in range(8):
        rk = s0.adjoint(W.reshape(-1) / npar, seed=9, walker_range=(npar * k // 8, npar * (k + 1) // 8))
        shard_g["D"].append(8 * rk["d_diffusivity"])
        shard_g["D_pathwise"].append(8 * rk["d_diffusivity_pathwise"])
        shard_g["kappa"].append(8 * rk["d_kappa"])
    for key, name in (("D", "D"), ("kappa", "kappa")):
        se = float(np.std(shard_g[key], ddof=1) / np.sqrt(8))
        out[name]["std_err"] = se
        ref = out[name]["slope_5pct"]
        out[name]["z_vs_slope"] = (out[name]["adjoint"] - ref) / se if se > 0 else None
    # the frozen-event (pathwise) D estimate beside the time-rescaling one
    se_p = float(np.std(shard_g["D_pathwise"], ddof=1) / np.sqrt(8))
    out["D"]["pathwise"] = {"value": r["d_diffusivity_pathwise"], "std_err": se_p,
                            "rel_err_vs_slope": abs(r["d_diffusivity_pathwise"] / out["D"]["slope_5pct"] - 1)}
    per_dir = per_direction_checks(s0, signal, npar, nw, par, h)
    # the forward walk's walker-steps, differentiated: pass 1 walks them again
    # with its records, the forced walks about half of them once more
    ws = npar * tn
    line = {
        "metric": ADJOINT_METRIC, "value": ws / (adj_ms * 1e-3), "unit": "walker-steps/s", "n_gpus": 1, "steps": 1,
        "warmup": args.warmup, "ms_per_step": adj_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+i32 (f64 sums)", "data": "synthetic (seeded axon lattice and waveform)",
        "config": {"workload": f"adjoint: 64x64x512 axon + label-2 exterior, {npar} walkers, {tn} steps, "
                               f"waveform {nb} bins x 3 turned to {nw} directions, periodic walls",
                   "walkers": npar, "steps_per_walk": tn, "nbins": nb, "nwave": nw, "parallelism": "1 GPU"},
        "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
        "e2e": {"value": ws / adj_s, "unit": "walker-steps/s", "h2d_bytes_per_step": int(lab.nbytes),
                "d2h_bytes_per_step": int(r["d_wave"].nbytes)},
        # adjoint_kernel pass 1, adjoint_dwave_kernel, adjoint_kernel forced walks
        "gradient_checks": out, "signal_gradients": per_dir, "loss": r["loss"], "gpu_launches": 3,
    }
    print(json.dumps(line), flush=True)


def per_direction_checks(s0, signal, npar, nw, par, h, seeds=range(21, 29)):
    """dS_j/dtheta for each direction's signal S_j = mean s0 cos(phi_j) (the
    reference's PGSE signal, main_PGSE.cu:348-357) and theta = D, kappa, T2:
    every direction's Jacobian row from one reverse pass (rms_adjoint_jacobian),
    against central finite differences with common random numbers (h
    relative) and the least-squares slope over +-5 % (7 points).  Every
    estimate is repeated over independent seeds and compared as seed means
    with standard errors from the seed spread: with common random numbers the
    7 points of one slope share their walkers, so a fit's residuals
    understate its error."""
    t2 = par["t2"]
    names = ("D", "kappa", "T2[1]", "T2[2]")
    x0s = {"D": par["D"], "kappa": par["kappa"], "T2[1]": t2[1], "T2[2]": t2[2]}
    ns = len(seeds)
    adj = {k: np.zeros((ns, nw)) for k in names + ("kappa_score",)}
    fd = {k: np.zeros((ns, nw)) for k in names}
    sl = {k: np.zeros((ns, nw)) for k in ("D", "kappa")}

    def vary(name, x, seed):
        if name == "D":
            return signal(D=x, seed=seed)[:, 0]
        if name == "kappa":
            return signal(kappa=x, seed=seed)[:, 0]
        tt = t2.copy()
        tt[int(name[3])] = x
        return signal(t2=tt, seed=seed)[:, 0]

    jac_ms = []
    for si, seed in enumerate(seeds):
        J = s0.jacobian(seed=seed)
        jac_ms.append(s0.timing()[0])
        adj["D"][si] = J["D"][:, 0] / npar
        adj["kappa"][si] = J["kappa"][:, 0] / npar
        adj["kappa_score"][si] = J["kappa_score"][:, 0] / npar
        adj["T2[1]"][si] = J["T2"][:, 0, 1] / npar
        adj["T2[2]"][si] = J["T2"][:, 0, 2] / npar
        for name, x0 in x0s.items():
            fd[name][si] = (vary(name, x0 * (1 + h), seed) - vary(name, x0 * (1 - h), seed)) / (2 * h * x0)
        for name in ("D", "kappa"):
            xs = x0s[name] * (1 + 0.05 * np.linspace(-1, 1, 7))
            ys = np.stack([vary(name, x, seed) for x in xs])          # [7, nw]
            sl[name][si] = np.polyfit(xs, ys, 1)[0]

    def mse(a):
        return a.mean(axis=0), a.std(axis=0, ddof=1) / np.sqrt(ns)

    res = {}
    for name in names:
        a, ase = mse(adj[name])
        f, fse = mse(fd[name])
        ent = {"adjoint": a.tolist(), "adjoint_std_err": ase.tolist(), "finite_difference": f.tolist(),
               "finite_difference_std_err": fse.tolist(), "rel_err_vs_fd": np.abs(a / f - 1).tolist(),
               "z_vs_fd": ((a - f) / np.hypot(ase, fse)).tolist()}
        ref = f
        if name in sl:
            b, bse = mse(sl[name])
            ent.update(slope_5pct=b.tolist(), slope_std_err=bse.tolist(), rel_err_vs_slope=np.abs(a / b - 1).tolist(),
                       z_vs_slope=((a - b) / np.hypot(ase, bse)).tolist())
            ref = b
        if name == "kappa":
            c, cse = mse(adj["kappa_score"])
            ent["score_function"] = {"value": c.tolist(), "std_err": cse.tolist()}
        rel = np.abs(a / ref - 1)
        ent["summary"] = {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
                          "max_rel_err_vs_fd": float(np.max(ent["rel_err_vs_fd"])),
                          "median_rel_std_err": float(np.median(np.abs(ase / a))),
                          "median_abs_z": float(np.median(np.abs(ent.get("z_vs_slope", ent["z_vs_fd"]))))}
        res[name] = ent
    return {"of": "S_j = mean over walkers of s0 cos(phi_j), each of the 16 directions", "walkers_per_seed": npar,
            "seeds": list(seeds), "h": h, "jacobian_ms": float(np.median(jac_ms)), **res}


CONTRACT_METRIC = "walker-waveform phases/s of the multi-waveform phase contraction (signal mean(cos, sin))"


def run_contraction(args):
    """The multi-waveform phase contraction: positions of 1e7 walkers on 256
    time bins x 3 axes (FP32, from the engine's own walk in waveform mode:
    the 64x64x512 axon with label-2 exterior, kappa = 0.01 um/ms, 20480 steps
    of dt = 5e-4 ms, bin means) contracted against 1024 seeded smooth random
    waveforms with b in [0, 10] ms/um^2.  Times the BF16 hi/lo tensor-core
    method (value) and the FP32 CUDA-core method, and states the signal error
    of both against an FP64 evaluation on the first 65536 walkers, per b."""
    import torch
    from rms_b200 import engine, geometry, waveforms
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and int(os.environ.get("RANK", "0")) != 0:
        return   # one GPU: the positions of one walk fill 30.7 GB of its memory
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    nwalk = args.walkers or 10_000_000
    nbins, nwave, per_bin, dt, D0 = 256, 1024, 80, 5e-4, 2.0
    tn = nbins * per_bin
    stream = torch.cuda.current_stream()
    lab = geometry.axon_lattice(64, 64, 512, 0.1, seed=0, exterior=2)
    dtb = dt * per_bin
    w = waveforms.random_smooth(nwave, nbins, 1.0, seed=4)
    b = np.linspace(0.0, 10.0, nwave)
    w = waveforms.scale_to_b(w, dtb, np.maximum(b, 1e-9))
    wave = np.ascontiguousarray((w * dtb).astype(np.float32))     # phase per um of a bin's position
    # positions: the split walk's bin means (waveform mode, one zero waveform)
    sim = engine.Sim(lab, dt=dt, tn=tn, npar=nwalk, res=0.1, diffusivity=[0.0, D0, D0], t2=[1e12] * 3,
                     wave=np.zeros((1, nbins, 3)), timepoints=nbins, boundary="periodic",
                     permeation="kappa", kappa=0.01)
    pos = torch.empty((nwalk, nbins, 3), dtype=torch.float32, device="cuda")
    sim.run(seed=5, precision="split", stream=stream.cuda_stream, traj_out=pos.data_ptr())
    torch.cuda.synchronize()
    d_wave = torch.from_numpy(wave).cuda()
    out = torch.empty((nwave, 2), dtype=torch.float64, device="cuda")

    def call(method, n=nwalk):
        return engine.contract_phases(pos.data_ptr(), n, nbins, d_wave.data_ptr(), nwave, out.data_ptr(),
                                      method=method, stream=stream.cuda_stream)

    for _ in range(args.warmup):
        call("bf16x3")
    torch.cuda.synchronize()
    kms = []
    with ClockSampler(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            kms.append(call("bf16x3"))
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    k_ms = float(np.mean(kms))
    S_tc = out.cpu().numpy() / nwalk
    f32_ms = call("fp32")
    S_f32 = out.cpu().numpy() / nwalk
    # the same walk writing its bin means as BF16 pairs: the contraction reads
    # them through TMA, no conversion
    pos_split = torch.empty_like(pos)
    sim.run(seed=5, precision="split", stream=stream.cuda_stream, traj_out=pos_split.data_ptr(), traj_split=True)
    torch.cuda.synchronize()

    def call_split():
        return engine.contract_phases(pos_split.data_ptr(), nwalk, nbins, d_wave.data_ptr(), nwave, out.data_ptr(),
                                      method="bf16x3_presplit", stream=stream.cuda_stream)

    for _ in range(args.warmup):
        call_split()
    ps_ms = float(np.mean([call_split() for _ in range(args.steps)]))
    S_ps = out.cpu().numpy() / nwalk
    del pos_split
    flops = 2.0 * nwalk * 3 * nbins * nwave

    # end to end through the API: waveforms from pinned host memory, the
    # signal read back; positions are the walk's device output
    h_wave = torch.from_numpy(wave).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.steps, 3))):
        d_wave.copy_(h_wave, non_blocking=True)
        call("bf16x3")
        sig = out.cpu()
    e2e_s = (time.perf_counter() - t0) / max(1, min(args.steps, 3))

    # signal error against FP64 on a sample, per b (bins of 1 ms/um^2)
    ns = min(nwalk, 65536)
    call("bf16x3", ns)
    s_tc = out.cpu().numpy() / ns
    call("fp32", ns)
    s_f32 = out.cpu().numpy() / ns
    P = pos[:ns].reshape(ns, -1).double().cpu().numpy()
    phi = P @ wave.reshape(nwave, -1).astype(np.float64).T
    s64 = np.stack([np.cos(phi).mean(0), np.sin(phi).mean(0)], axis=1)
    errs = []
    for lo in range(10):
        m = (b >= lo) & (b < lo + 1) if lo < 9 else (b >= 9)
        errs.append({"b": [lo, lo + 1], "bf16x3": float(np.abs(s_tc[m] - s64[m]).max()),
                     "fp32": float(np.abs(s_f32[m] - s64[m]).max()),
                     "S_mean": float(s64[m, 0].mean())})

    # CPU: FP32 matmul + cos/sin in numpy on all host cores, a bounded sample
    nc = 8192
    Pc = pos[:nc].reshape(nc, -1).cpu().numpy()
    Wc = wave.reshape(nwave, -1)
    t0 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t0 < 10.0:
        ph = Pc @ Wc.T
        np.cos(ph).sum(0), np.sin(ph).sum(0)
        reps += 1
    cpu_s = (time.perf_counter() - t0) / reps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("bf16_tflops", 1590.0))
    achieved = flops / (k_ms * 1e-3) / 1e12
    line = {
        "metric": CONTRACT_METRIC, "value": nwalk * nwave / (ms * 1e-3), "unit": "phases/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 hi/lo x3 (f32 accumulate, f64 sums)",
        "data": "synthetic (seeded walk positions, seeded random waveforms)",
        "config": {"workload": f"contraction: {nwalk} walkers x {nbins} bins x 3 axes (FP32 positions of the "
                               f"engine's walk, {tn} steps) against {nwave} waveforms, b in [0, 10] ms/um^2",
                   "walkers": nwalk, "nbins": nbins, "nwave": nwave, "K": 3 * nbins,
                   "l2": "inputs (30.7 GB of positions) larger than L2", "parallelism": "1 GPU"},
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "model": f"2 M K N = {flops:.3g} algorithmic FLOP / contraction kernel {k_ms:.2f} ms "
                              "(three BF16 products execute 3x that; peak: measured bf16_tflops, burst)"},
        "kernel_ms": k_ms,
        "fp32_cuda_cores": {"kernel_ms": f32_ms, "tflops": flops / (f32_ms * 1e-3) / 1e12,
                            "max_abs_diff_vs_bf16x3": float(np.abs(S_f32 - S_tc).max())},
        "bf16x3_presplit": {"kernel_ms": ps_ms, "tflops": flops / (ps_ms * 1e-3) / 1e12,
                            "frac_of_peak": flops / (ps_ms * 1e-3) / 1e12 / peak,
                            "max_abs_diff_vs_bf16x3": float(np.abs(S_ps - S_tc).max()),
                            "input": "bin means written by the walk as BF16 hi/lo pairs (traj_split), read by TMA"},
        "signal_error_vs_fp64": {"sample_walkers": ns, "per_b": errs},
        "e2e": {"value": nwalk * nwave / e2e_s, "unit": "phases/s", "h2d_bytes_per_step": int(wave.nbytes),
                "d2h_bytes_per_step": int(sig.numel() * 8)},
        "gpu_launches": 2 * args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": {"value": nc * nwave / cpu_s, "unit": "phases/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": f"numpy FP32 matmul + cos/sin, {nc} walkers x {nwave} "
                                                   f"waveforms x K={3 * nbins}, {reps} reps in ~10 s"},
    }
    print(json.dumps(line), flush=True)
    sim.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-cuda"])
    ap.add_argument("--precision", default="split", choices=["split", "compat"])
    ap.add_argument("--workload", default="batch",
                    choices=["production", "production-full", "batch", "single", "contraction", "adjoint"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--walkers", type=int, default=None, help="walkers per GPU (smaller case, e.g. for ncu)")
    ap.add_argument("--launches-once", action="store_true",
                    help="adjoint workload: one forward walk, reverse pass and Jacobian only (for a launch list)")
    ap.add_argument("--plain-steps", type=int, default=1,
                    help="timed runs of the plain FP64 walk on the same job (0: none)")
    ap.add_argument("--scaling", default="strong", choices=["strong", "weak"],
                    help="batch under several ranks: split the one job (strong) or walk it per rank (weak)")
    ap.add_argument("--no-error", action="store_true", help="skip the D/K error against the FP64 replay")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip the reference's own CUDA programs beside rms_main")
    ap.add_argument("--refcuda-walkers", type=int, default=1_000_000,
                    help="walkers of the reference-CUDA comparison (64x64x512 axon, 5000 steps)")
    ap.add_argument("--tn", type=int, default=None, help="steps per walk (smaller case, e.g. for ncu)")
    ap.add_argument("--timepoints", type=int, default=None,
                    help="records per walk (keep steps/record when shortening the walk)")
    args = ap.parse_args()
    if args.workload == "adjoint":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint"}))
        else:
            run_adjoint_bench(args)
    elif args.workload == "contraction":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no waveform contraction "
                                                                  "(its only gradient form is the PGSE pair)"}))
        else:
            run_contraction(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    elif args.impl == "reference-cuda":
        run_reference_cuda(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
