"""CPU-side checks of the product library: it loads without a GPU, exports every
entry point include/mgfvm.h declares, and its host logic (InputData parser, checks,
pattern generators, output writers) behaves like the reference.  No kernel runs."""
import ctypes as C
import filecmp
import os
import shutil

import numpy as np
import pytest

from conftest import GOLDEN, REPO


def test_library_exports_every_declared_symbol():
    from mgfvm import _lib
    L = _lib.lib()
    names = _lib.exported_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_parser_round_trip(tmp_path):
    from mgfvm import configs, read_case
    cfg = configs.small(32, 3, isolve=2, ig_obs=3, ig_inlt=2, ig_outlt=2, sc_obs=0.25,
                        obstacles=[(1, 2, 3, 4), (5, 5, 6, 7)], inlets=[(1, 3, 1.5, 0.1, 0.9)],
                        outlets=[(2, 4, 0.2, 0.0, 0.1), (1, 1, 0.3, 0.0, 0.0)])
    cfg.write(str(tmp_path))
    assert read_case(str(tmp_path)) == cfg


def test_parser_errors(tmp_path):
    from mgfvm import MgfvmError, configs, read_case
    from mgfvm._abi import EINVAL, EIO
    with pytest.raises(MgfvmError) as e:
        read_case(str(tmp_path))
    assert e.value.status == EIO
    configs.small().write(str(tmp_path))
    with open(tmp_path / "InputData") as f:
        lines = f.read().splitlines()
    lines[1] = "1.0 1.0 0.01"            # second line cut short; like fscanf in the
    (tmp_path / "InputData").write_text("\n".join(lines) + "\n")   # reference, values run on
    with pytest.raises(MgfvmError) as e:
        read_case(str(tmp_path))
    assert e.value.status == EINVAL and "failed reading" in str(e.value)
    configs.small().write(str(tmp_path))
    (tmp_path / "pattern.txt").write_text("2\n1 1 1 1\n2 2\n")
    with pytest.raises(MgfvmError) as e:
        read_case(str(tmp_path))
    assert e.value.status == EINVAL and "obstacle 1" in str(e.value)


@pytest.mark.parametrize("bad,status", [
    (dict(obstacles=[(1, 9, 1, 1)], ig_obs=3), "EOOB"),     # beyond the 8-cell level
    (dict(obstacles=[(0, 1, 1, 1)], ig_obs=3), "EOOB"),     # index 0 is the ghost layer
    (dict(ngrid=7), "EINVAL"),                               # 32 not divisible by 2^6
    (dict(isolve=3), "EINVAL"),
    (dict(ibc_xp=5), "EINVAL"),
    (dict(obstacles=[(1, 1, 1, 1)], ig_obs=4), "EINVAL"),   # ig_obs > ngrid
])
def test_validation_rejects(bad, status):
    from mgfvm import MgfvmError, configs, validate
    from mgfvm import _abi
    with pytest.raises(MgfvmError) as e:
        validate(configs.small(32, 3).replace(**bad))
    assert _abi.STATUS_NAMES[e.value.status] == status


def test_create_rejects_before_touching_a_device():
    """Bad input is reported as EINVAL even on a machine without a GPU."""
    from mgfvm import MgfvmError, Solver, configs
    with pytest.raises(MgfvmError) as e:
        Solver([configs.small(32, 3, isolve=1), configs.small(32, 3, isolve=2)])
    assert "smoothing schedule" in str(e.value)


def test_staggered_patterns():
    from mgfvm import patterns
    inline = patterns.staggered_grid(16, "full", 1, 1, variant=1)
    assert inline.shape == (16, 16)
    # inline lattice of 1x1 blocks with spacing 1: every other row and column
    assert abs(patterns.porosity(inline) - 0.75) < 0.02
    stag = patterns.staggered_grid(16, "quarter", 1, 1, variant=2)
    assert stag.shape == (64, 64)
    a = patterns.staggered_grid(16, "full", 1, 1, variant=5, seed=11)
    b = patterns.staggered_grid(16, "full", 1, 1, variant=5, seed=11)
    c = patterns.staggered_grid(16, "full", 1, 1, variant=5, seed=12)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    px = patterns.pixels(a)
    assert len(px) == int(a.sum()) and all(r[0] == r[1] and r[2] == r[3] for r in px)
    r, c_ = px[0][0] - 1, px[0][2] - 1
    assert a[r, c_] == 1


def test_random_patterns():
    from mgfvm import patterns
    g, rects = patterns.random_grid(16, 0.3, seed=5)
    assert abs(g.sum() / g.size - 0.3) < 0.08
    cover = np.zeros_like(g)
    for r1, r2, c1, c2 in rects:
        assert r2 - r1 == c2 - c1 and 0 <= r2 - r1 <= 2
        cover[r1 - 1:r2, c1 - 1:c2] += 1
    assert cover.max() == 1 and np.array_equal(cover, g)     # non-overlapping, exact cover
    g2, rects2 = patterns.random_grid(16, 0.3, seed=5)
    assert rects == rects2


def test_writers_byte_identical_to_reference(tmp_path, capfd, monkeypatch, oracle_built):
    """VTK and CSV written from the oracle's fields equal the reference binary's files."""
    from mgfvm import lib, read_case
    from mgfvm._lib import check
    from oracle import OracleCase
    d = os.path.join(GOLDEN, "cli")
    cfg = read_case(d)
    o = OracleCase(cfg)
    o.cycle(cfg.nvcycle)
    c, keep = cfg.to_c()
    npx, npy = o.dims(0)
    arrs = [np.ascontiguousarray(o.get(0, f)) for f in ("u", "v", "p", "sc")]
    rng = np.ascontiguousarray(o.obstacle_ranges(0), dtype=np.int32)
    dp = C.POINTER(C.c_double)
    monkeypatch.chdir(tmp_path)
    vtk = "vtk_acc.vtk"
    check(lib().mgfvm_write_vtk(vtk.encode(), C.byref(c), npx, npy, *[a.ctypes.data_as(dp) for a in arrs],
                                rng.ctypes.data_as(C.POINTER(C.c_int)), 0, None))
    e, _ = o.history()
    csv = "convergence.csv"
    check(lib().mgfvm_write_convergence(csv.encode(), np.ascontiguousarray(e).ctypes.data_as(dp),
                                        cfg.nvcycle - 1, cfg.nvcycle, 1))
    assert filecmp.cmp(vtk, os.path.join(d, "vtk_acc.vtk"), shallow=False)
    assert filecmp.cmp(csv, os.path.join(d, "convergence.csv"), shallow=False)
    out = capfd.readouterr().out.splitlines()
    ref = open(os.path.join(d, "stdout.txt")).read().splitlines()
    assert out == ref[-4:]


def test_sweep_driver_arguments(tmp_path):
    """The batch driver checks its arguments and inputs before it needs a GPU."""
    import subprocess
    sweep = os.path.join(REPO, "multigrid-fvm_b200", "bin", "mgfvm_sweep")
    r = subprocess.run([sweep, "--bogus"], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([sweep], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "pattern_*.txt" in r.stderr


def _read_pattern(path):
    lines = open(path).read().split("\n")
    n = int(lines[0])
    return [tuple(int(v) for v in l.split()) for l in lines[1:1 + n]]


def _read_pgm(path):
    tok = open(path).read().split()
    assert tok[0] == "P2" and tok[3] == "255"
    w, h = int(tok[1]), int(tok[2])
    return np.array([int(v) for v in tok[4:]], dtype=np.int32).reshape(h, w)


def test_pattern_generator_tool(tmp_path):
    """bin/mgfvm_patterns writes the reference generators' directory layout and file
    formats, with the seeded library generators' patterns."""
    import subprocess
    from mgfvm import patterns
    tool = os.path.join(REPO, "multigrid-fvm_b200", "bin", "mgfvm_patterns")
    r = subprocess.run([tool, "staggered", "16", "3", "1", "1", "2", "7"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    d = tmp_path / "n16_por_75.0_sx1_sy1_scale1x"
    for v in (1, 2, 3, 4):
        g = patterns.staggered_grid(16, "full", 1, 1, variant=v, seed=7)
        assert _read_pattern(d / f"pattern_{v}.txt") == patterns.pixels(g)
        assert np.array_equal(_read_pgm(d / f"pattern_{v}.pgm"), np.where(g == 1, 0, 255))
    r = subprocess.run([tool, "random", "20", "0.3", "2", "50", "30", "20", "5"], cwd=tmp_path,
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    d = tmp_path / "n_20" / "p_0.30"
    for p in (1, 2):
        g, rects = patterns.random_grid(20, 0.3, (50.0, 30.0, 20.0), seed=5 + p - 1)
        assert _read_pattern(d / f"pattern_{p}.txt") == rects
        assert np.array_equal(_read_pgm(d / f"pattern_{p}.pgm"), np.where(g == 1, 0, 255))
    assert subprocess.run([tool, "bogus"], cwd=tmp_path, capture_output=True, timeout=60).returncode == 2
