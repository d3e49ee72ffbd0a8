"""Host side of the C ABI (include/rms.h), no GPU needed: the library loads
and exports every declared entry point, configurations are validated with
error codes instead of the reference's silent misreads, and the derived tables
equal the reference's (hpc_code/lib/main.cu:433-458, 484-487)."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import pyoracle
from conftest import ROOT, unpack_golden
from rms_b200 import engine, geometry, runio


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rms.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(rms_\w+)\s*\(", src, flags=re.M))


def test_library_exports_every_declared_function():
    lib = engine.lib()
    decl = declared_functions()
    assert len(decl) >= 16
    for name in decl:
        assert hasattr(lib, name), name
    assert set(engine.EXPORTS) <= decl


def test_cli_binary_built():
    assert os.access(engine.CLI_PATH, os.X_OK)


def small_sim(**over):
    lab = geometry.axon_lattice(12, 12, 16, 0.1, seed=2, exterior=2, r0=0.4)
    kw = dict(dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0, 1.0], t2=[80, 80, 40],
              bval=[1.0], bvec=[[1, 0, 0]])
    kw.update(over)
    return engine.Sim(lab, **kw)


def test_derived_tables_match_reference_formulas():
    s = small_sim(diffusivity=[0, 2.0, 1.0, 0.5], t2=[80, 80, 40, 20])
    step, t2s, pij, td = pyoracle.reference_tables(2e-4, 0.1, [0, 2.0, 1.0, 0.5], [80, 80, 40, 20], 1000, 1000)
    assert np.array_equal(s.get("step"), step)
    assert np.array_equal(s.get("pij"), pij)
    assert np.array_equal(s.get("td"), td)
    assert np.array_equal(s.get("diffusivity"), [0, 2.0, 1.0, 0.5])


def test_kappa_permeation_formula():
    # analysis/interaction.m:437-439: P = 2/3 kappa ds / D0, then P / (1 + P)
    s = small_sim(permeation="kappa", kappa=0.01)
    p = s.get("pij").reshape(3, 3)
    for a, D in ((1, 2.0), (2, 1.0)):
        ds = math.sqrt(6 * D * 2e-4)
        P = 2.0 / 3.0 * 0.01 * ds / D
        assert p[a, 3 - a] == pytest.approx(P / (1 + P), rel=1e-15)
    assert p[1, 1] == 1.0 and p[0, 1] == 0.0 and p[1, 0] == 0.0


def test_pij_table_is_used_as_given():
    t = np.array([[0, 0, 0], [0, 1, 0.25], [0, 0.5, 1]], dtype=float)
    s = small_sim(permeation="table", pij=t)
    assert np.array_equal(s.get("pij"), t.ravel())


@pytest.mark.parametrize("over,code", [
    (dict(t2=[80, 0, 40]), -4),                      # T2 = 0 -> 0/0 in the reference
    (dict(tn=999), -4),                              # TN below the 1000 records
    (dict(diffusivity=[0, 2.0, 300.0]), -4),         # step >= one voxel
    (dict(dt=-1.0), -4),
    (dict(diffusivity=[0] + [1.0] * 9, t2=[80] * 10), -4),   # Nc above the kernels' limit
    # NaN parameters (the reference would walk with them)
    (dict(dt=float("nan")), -4),
    (dict(res=float("nan")), -4),
    (dict(t2=[80, float("nan"), 40]), -4),
    (dict(diffusivity=[0, float("nan"), 1.0]), -4),
    (dict(permeation="kappa", kappa=float("nan")), -4),
])
def test_invalid_configurations_are_rejected(over, code):
    with pytest.raises(engine.RmsError) as e:
        small_sim(**over)
    assert e.value.code == code


def test_lattice_validation():
    s = small_sim()
    with pytest.raises(engine.RmsError) as e:
        s.set_lattice(np.full((12, 12, 16), 3, dtype=np.uint8))   # label >= Nc
    assert e.value.code == -4
    with pytest.raises(engine.RmsError):
        s.set_lattice(np.zeros((12, 12, 16), dtype=np.uint8))     # nothing to start in
    with pytest.raises(engine.RmsError) as e:
        s.set_lattice(np.ones((12, 12, 15), dtype=np.uint8))      # wrong shape
    assert e.value.code == -1


def test_lattice_check_reports_the_first_bad_voxel():
    # the check scans in 255-voxel blocks: bad labels on and around block edges
    s = small_sim()
    n = 12 * 12 * 16
    for first in (0, 254, 255, 256, 509, 510, n - 1):
        lab = np.ones(n, dtype=np.uint8)
        lab[first] = 5
        if first + 7 < n:
            lab[first + 7] = 3
        with pytest.raises(engine.RmsError) as e:
            s.set_lattice(lab.reshape(12, 12, 16))
        assert e.value.code == -4 and f"label 5 at voxel {first} " in str(e.value), str(e.value)
    # one labelled voxel is enough; labels Nc - 1 are accepted
    lab = np.zeros(n, dtype=np.uint8)
    lab[300] = 2
    s.set_lattice(lab.reshape(12, 12, 16))


def test_large_lattice_check_spans_the_threads():
    # above 32 MB the scan and the copy are split across host threads: a bad
    # label in the last range is still found, and the first one is reported
    shape = (64, 64, 16384 + 64)   # 67 MB: two ranges
    s = engine.Sim(None, shape=shape, dt=2e-4, tn=1000, npar=32, res=0.1, diffusivity=[0, 2.0],
                   t2=[80, 80], bval=[1.0], bvec=[[1, 0, 0]])
    lab = np.ones(shape, dtype=np.uint8)
    s.set_lattice(lab)
    flat = lab.reshape(-1)
    last = flat.size - 3
    flat[last] = 2
    with pytest.raises(engine.RmsError) as e:
        s.set_lattice(lab)
    assert f"label 2 at voxel {last} " in str(e.value)
    flat[1000] = 7
    with pytest.raises(engine.RmsError) as e:
        s.set_lattice(lab)
    assert "label 7 at voxel 1000 " in str(e.value)


def test_results_before_run_are_an_error():
    s = small_sim()
    with pytest.raises(engine.RmsError) as e:
        s.get("sig0")
    assert e.value.code == -7
    # no run and no reverse pass yet: no times either
    with pytest.raises(engine.RmsError) as e:
        s.timing()
    assert e.value.code == -7


@pytest.mark.parametrize("case", ["narrow_3comp", "pgse_3comp"])
def test_load_dir_reads_reference_inputs(case, tmp_path):
    d = unpack_golden(case, str(tmp_path), inputs_only=True)
    s = engine.Sim.from_dir(d)
    assert s.mode == ("pgse" if case.startswith("pgse") else "narrow")
    assert s.field_size("sig0") == 1000
    D = np.loadtxt(os.path.join(d, "diffusivity.txt"))
    assert np.array_equal(s.get("diffusivity"), D)


def test_load_dir_errors(tmp_path):
    d = unpack_golden("narrow_3comp", str(tmp_path / "a"), inputs_only=True)
    os.remove(os.path.join(d, "T2.txt"))
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d)
    assert e.value.code == -2
    d = unpack_golden("narrow_3comp", str(tmp_path / "b"), inputs_only=True)
    txt = open(os.path.join(d, "fiber.txt")).read().split()
    open(os.path.join(d, "fiber.txt"), "w").write(" ".join(txt[:-5]))
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d)
    assert e.value.code == -3
    # a narrow-pulse simParamInput.txt given to the PGSE reader: the reference
    # would read Nbvec as Nc (main_PGSE.cu:442); here it is an error
    d = unpack_golden("narrow_3comp", str(tmp_path / "c"), inputs_only=True)
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d, mode="pgse")
    assert e.value.code == -3


@pytest.mark.parametrize("fn,content,code", [
    ("diffusivity.txt", "0 abc 1.0", -3),        # a token that is not a number
    ("T2.txt", "80 nan 40", -3),
    ("bval.txt", "1 2 x 4 5 6", -3),
    ("fiber.txt", "junk", -3),
    ("simParamInput.txt", None, -4),             # NPar = -5
])
def test_corrupt_input_files_are_rejected(tmp_path, fn, content, code):
    d = unpack_golden("narrow_3comp", str(tmp_path), inputs_only=True)
    if content is None:
        vals = open(os.path.join(d, fn)).read().split()
        vals[2] = "-5"
        content = " ".join(vals)
    open(os.path.join(d, fn), "w").write(content)
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d)
    assert e.value.code == code, str(e.value)


def test_run_without_gpu_fails_loudly():
    pytest.importorskip("torch")
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = small_sim()
    with pytest.raises(engine.RmsError) as e:
        s.run(seed=1)
    assert e.value.code == -5


def test_binary_lattice_is_read_in_place_of_text(tmp_path):
    from rms_b200 import runio
    d = unpack_golden("narrow_3comp", str(tmp_path / "a"), inputs_only=True)
    vals = np.array(open(os.path.join(d, "fiber.txt")).read().split(), dtype=np.uint8)
    runio.write_lattice_binary(os.path.join(d, "fiber.bin"), vals)
    # fiber.bin wins: a broken fiber.txt beside it is not read
    open(os.path.join(d, "fiber.txt"), "w").write("0 0 0")
    engine.Sim.from_dir(d)
    # wrong size and labels >= Nc are refused
    vals[:-1].tofile(os.path.join(d, "fiber.bin"))
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d)
    assert e.value.code == -3
    bad = vals.copy()
    bad[7] = 200
    bad.tofile(os.path.join(d, "fiber.bin"))
    with pytest.raises(engine.RmsError) as e:
        engine.Sim.from_dir(d)
    assert e.value.code == -4


def test_write_inputs_binary_lattice(tmp_path):
    from rms_b200 import geometry, runio
    lab = geometry.axon_lattice(8, 8, 12, 0.1, seed=1, exterior=2)
    runio.write_inputs(str(tmp_path), lab, dt=2e-4, tn=1000, npar=10, res=0.1, diffusivity=[0, 2, 2],
                       t2=[80, 80, 60], bval=[1.0], bvec=[[1, 0, 0]], lattice="bin")
    assert not os.path.exists(os.path.join(tmp_path, "fiber.txt"))
    assert np.array_equal(np.fromfile(os.path.join(tmp_path, "fiber.bin"), dtype=np.uint8), lab.reshape(-1))
    engine.Sim.from_dir(str(tmp_path))


def test_combine_cumulants_matches_the_demo_formula():
    rng = np.random.default_rng(0)
    na, T, nd = 5, 40, 3
    f = rng.dirichlet(np.ones(na))
    Ds = rng.uniform(0.5, 2.0, (na, T, nd))
    Ks = rng.uniform(-0.5, 2.0, (na, T, nd))
    D, K = engine.combine_cumulants(f, Ds, Ks)
    # part1_demo4_analysis.m:88-90
    Dw = np.einsum("a,atd->td", f, Ds)
    Kw = 3 * (np.einsum("a,atd->td", f, Ds ** 2) - Dw ** 2) / Dw ** 2 + np.einsum("a,atd->td", f, Ds ** 2 * Ks) / Dw ** 2
    np.testing.assert_allclose(D, Dw, rtol=1e-14)
    np.testing.assert_allclose(K, Kw, rtol=1e-12)
    # one axon: D and K pass through
    D1, K1 = engine.combine_cumulants([1.0], Ds[:1], Ks[:1])
    np.testing.assert_allclose(D1, Ds[0], rtol=1e-15)
    np.testing.assert_allclose(K1, Ks[0], rtol=1e-12, atol=1e-14)


def test_reference_mat_files_are_read(tmp_path):
    # files in the reference's MAT layouts (fiber struct array, b-table)
    from scipy.io import savemat
    from rms_b200 import runio
    rng = np.random.default_rng(4)
    shapes = [rng.integers(0, 3, size=(6, 5, 4)).astype(np.uint8), rng.integers(0, 2, size=(3, 4, 7)).astype(np.uint8)]
    fiber = np.zeros((1, 2), dtype=[("shape", "O"), ("voxel_size", "O")])
    for j, sh in enumerate(shapes):
        fiber[0, j]["shape"] = sh
        fiber[0, j]["voxel_size"] = np.array([[0.1 * (j + 1)]])
    savemat(str(tmp_path / "fiber.mat"), {"fiber": fiber})
    got = runio.read_fiber_mat(str(tmp_path / "fiber.mat"))
    assert len(got) == 2
    for (lab, vs), sh, j in zip(got, shapes, range(2)):
        assert lab.dtype == np.uint8 and lab.flags.c_contiguous
        np.testing.assert_array_equal(lab, sh)
        assert vs == pytest.approx(0.1 * (j + 1))
    bvec = rng.normal(size=(9, 3))
    savemat(str(tmp_path / "bt.mat"), {"bval": np.linspace(0.2, 1.0, 9)[:, None], "bvec": bvec})
    bval, bv = runio.read_btable_mat(str(tmp_path / "bt.mat"))
    np.testing.assert_allclose(bval, np.linspace(0.2, 1.0, 9))
    np.testing.assert_allclose(bv, bvec)
    # a lattice read this way runs through the engine's set-up like fiber.txt
    s = engine.Sim(got[0][0], dt=2e-4, tn=1000, npar=4, res=got[0][1], diffusivity=[0, 2.0, 1.0],
                   t2=[80, 80, 40], bval=bval, bvec=bv)
    np.testing.assert_array_equal(s.get("bval"), bval)


def test_lattice_text_writer_matches_the_reference_format(tmp_path):
    # setupRMS.m:17-23 writes sprintf('%u ', ...) per label, i outer, k fastest
    import gzip
    from rms_b200 import runio
    v = np.arange(256, dtype=np.uint8)
    lab = np.concatenate([v, np.random.default_rng(5).integers(0, 256, size=4096 - 256)]).astype(np.uint8)
    runio.write_lattice(str(tmp_path / "f.txt"), lab.reshape(16, 16, 16))
    assert open(tmp_path / "f.txt", "rb").read() == "".join("%u " % x for x in lab).encode()
    # the golden run directories' fiber.txt, which the reference program read
    want = gzip.open(os.path.join(os.path.dirname(__file__), "golden", "narrow_3comp", "fiber.txt.gz")).read()
    runio.write_lattice(str(tmp_path / "g.txt"), np.array(want.split(), dtype=np.uint8).reshape(-1, 1, 1))
    assert open(tmp_path / "g.txt", "rb").read() == want
    runio.write_lattice(str(tmp_path / "e.txt"), np.zeros((0, 1, 1), dtype=np.uint8))
    assert open(tmp_path / "e.txt", "rb").read() == b""


def test_graph_refuses_closed_simulations():
    # Graph.run checks its simulations before the library sees the graph
    # (a stand-in graph object: capturing one needs a GPU)
    s = small_sim()
    g = engine.Graph.__new__(engine.Graph)
    g._h = engine.C.c_void_p(1)          # never reaches the library
    g.sims = [s]
    s.close()
    try:
        with pytest.raises(engine.RmsError) as e:
            g.run(1)
        assert e.value.code == -7
    finally:
        g._h = engine.C.c_void_p()
    with pytest.raises(engine.RmsError):
        g.run(1)


def test_sim_para_field_and_cli_flags():
    # sim_para.txt's values without a run (main.cu:606-609)
    s = small_sim()
    np.testing.assert_array_equal(s.get("sim_para"), [2e-4, 1000, 32, 0.1])
    # the CLI knows --metrics; without a GPU it still fails loudly, after parsing
    import subprocess
    r = subprocess.run([engine.CLI_PATH, "--metrics", "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2 and "--metrics" in r.stderr
