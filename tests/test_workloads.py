"""The benchmark workload's committed reference-format inputs (workloads/) are what
the seeded generators and the InputData writer produce today."""
import os
import sys

from conftest import REPO


def test_committed_workload_inputs_regenerate(tmp_path):
    sys.path.insert(0, os.path.join(REPO, "workloads"))
    import make_workloads
    make_workloads.main(str(tmp_path))
    for name in make_workloads.NAMES:
        for f in ("InputData", "pattern.txt"):
            with open(os.path.join(REPO, "workloads", name, f)) as a, open(tmp_path / name / f) as b:
                assert a.read() == b.read(), f"workloads/{name}/{f} differs from the generator's output"


def test_committed_workload_inputs_parse_back(tmp_path):
    """The C parser reads them back to the same cases (readInput :280-401)."""
    sys.path.insert(0, os.path.join(REPO, "workloads"))
    import make_workloads
    from mgfvm import read_case
    for name, cfg in make_workloads.cases().items():
        got = read_case(os.path.join(REPO, "workloads", name))
        assert got == cfg, name
