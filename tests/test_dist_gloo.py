"""Walker sharding across two ranks (gloo, CPU): each rank walks its shard
and the FP64 accumulators are summed in rank order; the result equals the
unsharded job (counts exactly, sums to 1e-12).  The walk itself is the
oracle here, standing in for the GPU kernel on this CPU-only check of the
rank logic (rms_b200.shards, used by bench.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import pyoracle
from rms_b200 import geometry, shards


def _job():
    lab = geometry.axon_lattice(12, 12, 16, 0.1, seed=3, exterior=2, r0=0.4)
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, [0, 2.0, 1.0], [80, 80, 40], 1000, 1000)
    return pyoracle.Job(lab, dt=2e-4, tn=1000, npar=60, res=0.1, step=step, t2_steps=t2s, pij=pij,
                        seed=5, td=td, bval=[1.0], bvec=[[1, 0, 0]])


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    job = _job()
    w0, w1 = shards.split_range(job.npar, rank, world)
    o = pyoracle.run_oracle(job, w0, w1)
    fields = {k: o[k] for k in ("sig0", "dx2", "dx4", "sigre", "npar_count")}
    tot = shards.gather_sum(fields)
    if rank == 0:
        q.put({k: v.copy() for k, v in tot.items()})
    dist.barrier()
    dist.destroy_process_group()


def _batch():
    """Three axons of uneven lattices and walker counts (one with fewer
    walkers than ranks), as a batch would hold them."""
    jobs = []
    for k, (shape, npar) in enumerate((((12, 12, 16), 37), ((10, 14, 20), 64), ((8, 8, 12), 1))):
        lab = geometry.axon_lattice(*shape, 0.1, seed=10 + k, exterior=2, r0=0.35)
        step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, [0, 2.0, 1.5], [80, 80, 40], 1000, 1000,
                                                       kappa=0.02 * k)
        jobs.append(pyoracle.Job(lab, dt=2e-4, tn=1000, npar=npar, res=0.1, step=step, t2_steps=t2s, pij=pij,
                                 seed=100 + k, td=td, bval=[1.0], bvec=[[0, 0, 1]]))
    return jobs


def _batch_rank(rank, world, port, q):
    """One rank of a batch split into shards: walkers [npar r / N, npar (r+1) / N)
    of every axon (what rms_run_opts.shard_index/shard_count selects in the
    library), then the per-axon sums added across ranks in rank order."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    fields = {}
    for k, job in enumerate(_batch()):
        w0, w1 = shards.split_range(job.npar, rank, world)
        o = pyoracle.run_oracle(job, w0, w1) if w1 > w0 else job.empty_outputs()
        for f in ("sig0", "dx2", "dx4", "sigre", "npar_count"):
            fields[f"{k}/{f}"] = o[f]
    tot = shards.gather_sum(fields)
    if rank == 0:
        q.put({k: v.copy() for k, v in tot.items()})
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_batch_shards_sum_to_the_whole_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for k, job in enumerate(_batch()):
        whole = pyoracle.run_oracle(job)
        assert np.array_equal(got[f"{k}/npar_count"], whole["npar_count"]), k
        for f in ("sig0", "dx2", "dx4", "sigre"):
            np.testing.assert_allclose(got[f"{k}/{f}"], whole[f], rtol=1e-12,
                                       atol=1e-12 * np.abs(whole[f]).max())


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_shards_sum_to_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    whole = pyoracle.run_oracle(_job())
    assert np.array_equal(got["npar_count"], whole["npar_count"])
    for k in ("sig0", "dx2", "dx4", "sigre"):
        np.testing.assert_allclose(got[k], whole[k], rtol=1e-12, atol=1e-12 * np.abs(whole[k]).max())


def _adjoint_job():
    """Permeable flat planes (kappa = 0.05), 2 waveforms of 20 bins."""
    from rms_b200 import waveforms
    lab = np.full((12, 8, 8), 2, dtype=np.uint8)
    lab[(np.arange(12) // 3) % 2 == 0] = 1
    dt, tn, nb = 5e-4, 400, 20
    wave = waveforms.scale_to_b(waveforms.random_smooth(2, nb, 1.0, seed=7), dt * tn / nb, [0.5, 1.0])
    step, t2s, pij, td = pyoracle.reference_tables(dt, 0.1, [0.0, 2.0, 2.0], [1e6, 70.0, 60.0], 20, tn, kappa=0.05)
    job = pyoracle.Job(lab, dt=dt, tn=tn, npar=96, res=0.1, step=step, t2_steps=t2s, pij=pij, seed=3,
                       timepoints=20, td=td, wave=wave, boundary=pyoracle.BOUNDARY_PERIODIC)
    gup = np.array([0.3, -1.1, 0.7, 0.2]) / job.npar
    return job, gup


def _adjoint_grads(job, gup, w0, w1):
    sums = pyoracle.adjoint_split(job, gup, w0, w1)
    return pyoracle.adjoint_gradients(job, sums, 2.0, [1e6, 70.0, 60.0], kappa=0.05, nwalk=w1 - w0)


def _adjoint_rank(rank, world, port, q):
    """One rank's walker shard of the reverse pass (the oracle's FP64 adjoint
    standing in for rms_adjoint_run with walker_range), then
    shards.adjoint_sum."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    job, gup = _adjoint_job()
    w0, w1 = shards.split_range(job.npar, rank, world)
    tot = shards.adjoint_sum(_adjoint_grads(job, gup, w0, w1))
    if rank == 0:
        q.put(tot)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_adjoint_shards_sum_to_the_whole_job():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_adjoint_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    job, gup = _adjoint_job()
    whole = _adjoint_grads(job, gup, 0, job.npar)
    assert whole["d_kappa"] != 0.0   # permeation draws were forced
    for k in ("d_diffusivity", "d_diffusivity_pathwise", "d_kappa", "loss"):
        assert got[k] == pytest.approx(whole[k], rel=1e-12, abs=1e-15), k
    for k in ("d_wave", "d_t2"):
        np.testing.assert_allclose(got[k], whole[k], rtol=1e-12, atol=1e-12 * np.abs(whole[k]).max(), err_msg=k)
    # the score with per-shard baselines: the sum of the two shards' estimates
    halves = [_adjoint_grads(job, gup, *shards.split_range(job.npar, r, 2))["d_kappa_score"] for r in range(2)]
    assert got["d_kappa_score"] == pytest.approx(sum(halves), rel=1e-12, abs=1e-15)


def test_shard_ranges_cover_the_job():
    for npar, world in ((10, 3), (1, 2), (1000003, 8)):
        rs = [shards.split_range(npar, r, world) for r in range(world)]
        assert rs[0][0] == 0 and rs[-1][1] == npar
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
    assert shards.walker_shard(100, 3) == (300, 400)
