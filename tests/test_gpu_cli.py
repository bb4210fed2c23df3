"""The drop-in command-line solver against the reference binary's own outputs on the
same InputData / pattern.txt (fixtures in tests/golden/cli, made by the reference)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

pytestmark = pytest.mark.gpu

BIN = os.path.join(REPO, "multigrid-fvm_b200", "bin", "mgfvm")


def _err_lines(lines):
    return [float(l.split("=")[-1]) for l in lines if l.startswith("icycle")]


def test_cli_matches_reference_binary(tmp_path):
    src = os.path.join(GOLDEN, "cli")
    for f in ("InputData", "pattern.txt"):
        shutil.copy(os.path.join(src, f), tmp_path / f)
    res = subprocess.run([BIN], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    mine = res.stdout.splitlines()
    ref = open(os.path.join(src, "stdout.txt")).read().splitlines()
    assert len(mine) == len(ref)
    for a, b in zip(mine, ref):
        if a.startswith("simple solution took"):
            assert b.startswith("simple solution took")
        elif a.startswith("icycle"):
            assert a.split("=")[0] == b.split("=")[0]
        else:
            assert a == b
    # the per-cycle mass error is a parallel sum: equal to 1e-12, printed with %e
    np.testing.assert_allclose(_err_lines(mine), _err_lines(ref), rtol=1e-6)
    vtk = open(tmp_path / "vtk_acc.vtk").read()
    assert vtk == open(os.path.join(src, "vtk_acc.vtk")).read()
    csv_m = open(tmp_path / "convergence.csv").read().splitlines()
    csv_r = open(os.path.join(src, "convergence.csv")).read().splitlines()
    assert csv_m[0] == csv_r[0] and len(csv_m) == len(csv_r)
    np.testing.assert_allclose([float(l.split(",")[1]) for l in csv_m[1:]],
                               [float(l.split(",")[1]) for l in csv_r[1:]], rtol=1e-6)


SWEEP = os.path.join(REPO, "multigrid-fvm_b200", "bin", "mgfvm_sweep")


def test_sweep_matches_one_run_per_pattern(tmp_path):
    """The batch driver (run_patterns_and_save_vtk.sh's loop, all cases in one GPU
    context) writes the same files as the drop-in solver run once per (Re, pattern)
    in its own directory, as the shell loop runs the reference."""
    from mgfvm import configs
    base = configs.small(32, 3, isolve=2, ig_obs=3, sc_obs=0.0, nvcycle=40)
    pats = {"1": [(2, 3, 2, 2), (5, 6, 4, 6)], "12": [(1, 1, 7, 8)], "3": []}
    (tmp_path / "patterns").mkdir()
    base.write(str(tmp_path))
    for n, obs in pats.items():
        (tmp_path / "patterns" / f"pattern_{n}.txt").write_text(base.replace(obstacles=obs).pattern_text())
    res = subprocess.run([SWEEP, "--re", "10,20"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    for re in ("10", "20"):
        for n, obs in pats.items():
            d = tmp_path / f"single_{re}_{n}"
            base.replace(obstacles=obs, amuf=1.0 / float(re)).write(str(d))
            r = subprocess.run([BIN], cwd=d, capture_output=True, text=True, timeout=120)
            assert r.returncode == 0, r.stderr
            out = tmp_path / "solution" / f"Re_{re}"
            assert (out / "vtk_files" / f"vtk_{n}.vtk").read_text() == (d / "vtk_acc.vtk").read_text(), (re, n)
            assert (out / "convergence_files" / f"convergence_{n}.csv").read_text() == \
                (d / "convergence.csv").read_text(), (re, n)
