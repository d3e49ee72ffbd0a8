"""Batched runs (rms_batch_run): many axons with uneven lattices and walker
counts walked by one persistent split launch.  Axon k uses seed + k * phi64
(include/rms.h), so each must equal its own rms_sim_run with that seed --
the same walkers, the same arithmetic: compartment counts equal, FP64 sums
equal up to summation order."""
import numpy as np
import pytest

from conftest import assert_fp64_close
from rms_b200 import engine, geometry

pytestmark = pytest.mark.gpu
PHI64 = 0x9E3779B97F4A7C15


def axon_sims(mode="narrow"):
    rng = np.random.default_rng(11)
    sims = []
    shapes = [(16, 16, 40), (24, 20, 32), (12, 12, 64), (32, 32, 24), (20, 16, 16)]
    for k, shp in enumerate(shapes):
        lab = geometry.axon_lattice(*shp, 0.1, seed=k, exterior=2, r0=float(rng.uniform(0.4, 0.9)))
        D1 = float(rng.uniform(1.5, 2.5))
        kw = dict(dt=2e-4, tn=1000, npar=int(rng.integers(300, 5000)), res=0.1,
                  diffusivity=[0, D1, 2.0], t2=[80, 80, 60], permeation="kappa",
                  kappa=float(rng.uniform(0, 0.05)))
        if mode == "pgse":
            kw["grad"] = np.array([[0.1, 0.05, 2.0, 1, 0, 0], [0.15, 0.05, 3.0, 0, 0.6, 0.8]])
        else:
            kw["bval"], kw["bvec"] = [1.0, 2.0], [[1, 0, 0], [0, 0, 1]]
        sims.append(engine.Sim(lab, **kw))
    return sims


@pytest.mark.parametrize("mode", ["narrow", "pgse"])
def test_batch_equals_single_runs(mode):
    sims = axon_sims(mode)
    seed = 77
    engine.batch_run(sims, seed=seed, precision="split")
    batched = [s.outputs() for s in sims]
    for k, s in enumerate(sims):
        single = s.run(seed=(seed + k * PHI64) % (1 << 64), precision="split").outputs()
        assert np.array_equal(batched[k]["npar_count"], single["npar_count"]), k
        for f in ("sig0", "dx2", "dx4") + (("sig",) if mode == "pgse" else ("sigre",)):
            assert_fp64_close(batched[k][f], single[f], 1e-9, f"axon {k} {f}")


def test_batch_compat_is_serial_equivalent():
    sims = axon_sims()[:2]
    engine.batch_run(sims, seed=5, precision="compat")
    b = [s.outputs() for s in sims]
    for k, s in enumerate(sims):
        one = s.run(seed=(5 + k * PHI64) % (1 << 64), precision="compat").outputs()
        for f in one:
            assert np.array_equal(b[k][f], one[f]), (k, f)


def test_batch_rejects_mixed_schedules():
    sims = axon_sims()[:2]
    lab = np.ones((8, 8, 8), dtype=np.uint8)
    other = engine.Sim(lab, dt=2e-4, tn=2000, npar=10, res=0.1, diffusivity=[0, 2.0], t2=[80, 80],
                       bval=[1.0, 2.0], bvec=[[1, 0, 0], [0, 0, 1]])
    with pytest.raises(engine.RmsError) as e:
        engine.batch_run(sims + [other], seed=1, precision="split")
    assert e.value.code == -1


def test_autotune_picks_a_variant_and_caches_it():
    import time
    sims = axon_sims()
    v, ms = engine.autotune(sims, seed=3)
    nv = len(engine.split_variants())
    assert 1 <= v <= nv and ms.shape == (nv,) and np.all(ms > 0)
    assert ms[v - 1] == ms.min()
    t0 = time.perf_counter()
    v2, ms2 = engine.autotune(sims, seed=3)
    assert v2 == v and np.array_equal(ms, ms2) and time.perf_counter() - t0 < 0.05   # cached
    # the variant changes the launch shape only: the same walkers, the same counts
    engine.batch_run(sims, seed=5, precision="split", variant=v)
    tuned = [s.outputs() for s in sims]
    engine.batch_run(sims, seed=5, precision="split", variant=1)
    for s, o in zip(sims, tuned):
        p = s.outputs()
        np.testing.assert_array_equal(p["npar_count"], o["npar_count"])
        assert_fp64_close(p["dx2"], o["dx2"], 1e-9, "dx2")


def test_graph_replays_equal_batch_runs():
    sims = axon_sims("pgse")
    g = engine.Graph(sims, seed=0)
    for seed in (21, 22):
        g.run(seed)
        replay = [s.outputs() for s in sims]
        engine.batch_run(sims, seed=seed, precision="split")
        for s, o in zip(sims, replay):
            p = s.outputs()
            np.testing.assert_array_equal(p["npar_count"], o["npar_count"])
            assert_fp64_close(p["dx2"], o["dx2"], 1e-9, "dx2")
            np.testing.assert_allclose(p["sig"], o["sig"], rtol=1e-9, atol=1e-9)
    assert not np.array_equal(replay[0]["dx2"], sims[0].outputs()["dx2"] * 0)
    # a new lattice invalidates the captured launch
    sims[1].set_lattice(geometry.axon_lattice(24, 20, 32, 0.1, seed=9, exterior=2, r0=0.5))
    with pytest.raises(engine.RmsError):
        g.run(23)
    g.close()


def test_one_simulation_graph_equals_a_plain_run():
    # a graph of one simulation walks it in the table form (seeds from device
    # memory); the walkers and their draws are those of rms_sim_run
    sims = axon_sims()[:1]
    g = engine.Graph(sims, seed=0)
    g.run(31)
    o = sims[0].outputs()
    sims[0].run(seed=31, precision="split")
    p = sims[0].outputs()
    np.testing.assert_array_equal(p["npar_count"], o["npar_count"])
    assert_fp64_close(p["dx2"], o["dx2"], 1e-9, "dx2")
    g.close()


@pytest.mark.parametrize("precision", ["split", "compat"])
def test_batch_shards_sum_to_the_whole_batch(precision):
    """A batch split into ranks' shards (shard r of N of every axon's walkers,
    rms_run_opts.shard_index/shard_count): the shards' sums add up to the
    unsharded batch -- counts exactly, FP64 sums up to their order.  Three
    shards, one of them empty for the smallest axon (npar < shards)."""
    sims = axon_sims()[:3]
    tiny = engine.Sim(geometry.axon_lattice(12, 12, 16, 0.1, seed=4, exterior=2, r0=0.4), dt=2e-4, tn=1000, npar=2,
                      res=0.1, diffusivity=[0, 2.0, 2.0], t2=[80, 80, 60], bval=[1.0, 2.0],
                      bvec=[[1, 0, 0], [0, 0, 1]])
    sims.append(tiny)
    engine.batch_run(sims, seed=9, precision=precision)
    whole = [s.outputs() for s in sims]
    parts = []
    for r in range(3):
        engine.batch_run(sims, seed=9, precision=precision, shard=(r, 3))
        parts.append([s.outputs() for s in sims])
    for k in range(len(sims)):
        cnt = sum(p[k]["npar_count"] for p in parts)
        assert np.array_equal(cnt, whole[k]["npar_count"]), k
        for f in ("sig0", "dx2", "dx4", "sigre"):
            assert_fp64_close(sum(p[k][f] for p in parts), whole[k][f], 1e-9, f"axon {k} {f}")
    # the graph walks the same shard
    g = engine.Graph(sims, seed=0, shard=(1, 3)) if precision == "split" else None
    if g is not None:
        g.run(9)
        for k, s in enumerate(sims):
            np.testing.assert_array_equal(s.outputs()["npar_count"], parts[1][k]["npar_count"])
        g.close()


def test_shard_arguments_are_checked():
    sims = axon_sims()[:1]
    for bad in ((3, 3), (-1, 2)):
        with pytest.raises(engine.RmsError) as e:
            engine.batch_run(sims, seed=1, precision="split", shard=bad)
        assert e.value.code == -1
    with pytest.raises(engine.RmsError):
        sims[0].run(seed=1, precision="split", walker_range=(0, 10), shard=(0, 2))


def test_batch_with_a_wider_lattice_encoding_repacks_its_members():
    """A simulation walked alone packs its lattice 4 bits a voxel (Nc <= 7);
    walked in a batch with an Nc = 8 member every lattice is packed 8 bits a
    voxel.  The member must be packed again, not walked on its 4-bit cells:
    its batch result equals its own run with the batch seed."""
    sims = axon_sims()[:2]
    lab8 = geometry.axon_lattice(16, 16, 24, 0.1, seed=3, exterior=2, r0=0.5)
    lab8[:, :, :4][lab8[:, :, :4] == 2] = 7
    wide = engine.Sim(lab8, dt=2e-4, tn=1000, npar=500, res=0.1, diffusivity=[0, 2.0, 2.0, 1, 1, 1, 1, 1.5],
                      t2=[80.0] * 8, permeation="kappa", kappa=0.02, bval=[1.0, 2.0], bvec=[[1, 0, 0], [0, 0, 1]])
    alone = [s.run(seed=(3 + k * PHI64) % (1 << 64), precision="split").outputs() for k, s in enumerate(sims)]
    engine.batch_run(sims + [wide], seed=3, precision="split")
    for k, s in enumerate(sims):
        o = s.outputs()
        assert np.array_equal(o["npar_count"], alone[k]["npar_count"]), k
        assert_fp64_close(o["dx2"], alone[k]["dx2"], 1e-9, f"axon {k} dx2")
