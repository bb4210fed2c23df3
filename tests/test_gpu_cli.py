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
