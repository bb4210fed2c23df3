"""TEST INFRASTRUCTURE ONLY: oracle error of a benchmark configuration's timed solves.

`python bench.py --workload W --parity-dump F.json` (on the GPU) writes, per case of the
workload, the number of V-cycles its solve ran, a SHA-256 of its final level-0 u, v, p,
sc (FP64) and the mixed-precision solve's relative L2 distance to those fields.  This
script (on any CPU) runs the C oracle on every case for the same cycles from the same
initial state, in parallel processes, and compares hashes: equal hashes mean the FP64
engine's fields are the oracle's bit for bit (relative L2 error 0), and then the mixed
form's distance to the FP64 fields is its distance to the oracle.

    python oracle/config_parity.py F.json [--procs N] [--out summary.json] [--cache C.json]
    python oracle/config_parity.py --precompute W --cycles N --cache C.json [--procs N]

The oracle's hashes can be computed ahead of the GPU run (--precompute: every case of
workload W after N cycles) and kept in a cache file that later comparisons reuse.

Cases whose solve turned non-finite (the reference build diverges on the same inputs)
are reported and excluded from the distributions.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _paths():
    for p in (REPO, HERE, os.path.join(REPO, "multigrid-fvm_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)


def _oracle_hash(args):
    """One case on the oracle: (sha256 of its level-0 u, v, p, sc after `cycles`, seconds)."""
    cfg_dict, prof, cycles = args
    _paths()
    import oracle
    from mgfvm.inputs import CaseConfig
    t = time.perf_counter()
    o = oracle.OracleCase(CaseConfig(**cfg_dict), None if prof is None else np.asarray(prof))
    o.cycle(cycles)
    h = hashlib.sha256(b"".join(np.ascontiguousarray(o.get(0, f)).tobytes() for f in ("u", "v", "p", "sc")))
    o.close()
    return h.hexdigest(), time.perf_counter() - t


def _oracle_hashes(workload, cycles, procs, cache_path, skip=()):
    """(sha256, seconds) of every case of `workload` after cycles[k] cycles, from the
    cache where it holds them; cases in `skip` get (None, 0)."""
    import dataclasses

    import bench
    cases, desc, profiles = bench.workload(workload)
    cache = {"workload": workload, "hashes": {}}
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        assert cache["workload"] == workload
    key = lambda k: f"{k}:{cycles[k]}"
    todo = [k for k in range(len(cases)) if key(k) not in cache["hashes"] and k not in skip]
    jobs = [(dataclasses.asdict(cases[k]), None if profiles is None else list(profiles[k]), cycles[k]) for k in todo]
    t0 = time.perf_counter()
    if jobs:
        with mp.get_context("spawn").Pool(procs) as pool:
            for k, r in zip(todo, pool.imap(_oracle_hash, jobs, chunksize=1)):
                cache["hashes"][key(k)] = list(r)
                if cache_path and len(cache["hashes"]) % 16 == 0:
                    with open(cache_path, "w") as f:
                        json.dump(cache, f)
    if cache_path:
        with open(cache_path, "w") as f:
            json.dump(cache, f)
    return ([(None, 0.0) if k in skip else tuple(cache["hashes"][key(k)]) for k in range(len(cases))], desc,
            time.perf_counter() - t0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("dump", nargs="?")
    ap.add_argument("--procs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--cache", default=None)
    ap.add_argument("--precompute", default=None, help="workload whose oracle hashes to compute into --cache")
    ap.add_argument("--cycles", type=int, default=2000)
    a = ap.parse_args()
    _paths()
    import bench
    if a.precompute:
        n = len(bench.workload(a.precompute)[0])
        _oracle_hashes(a.precompute, [a.cycles] * n, a.procs, a.cache)
        return
    with open(a.dump) as f:
        dump = json.load(f)
    rows = dump["cases"]
    res, desc, wall = _oracle_hashes(dump["workload"], [r["cycles"] for r in rows], a.procs, a.cache,
                                     skip={k for k, r in enumerate(rows) if r["diverged"]})
    assert len(rows) == len(res), "the dump and the workload disagree on the number of cases"
    ok = [k for k, r in enumerate(rows) if not r["diverged"]]
    same = [k for k in ok if res[k][0] == rows[k]["sha256"]]
    differ = [k for k in ok if res[k][0] != rows[k]["sha256"]]
    mixed = [rows[k]["mixed_rel_l2_vs_fp64"] for k in same if rows[k].get("mixed_rel_l2_vs_fp64") is not None]
    out = {
        "workload": desc, "cases": len(rows), "diverged": len(rows) - len(ok),
        "fp64_bit_identical_to_oracle": len(same), "fp64_differs_from_oracle": differ,
        "fp64_rel_l2_vs_oracle": 0.0 if not differ and same else None,
        "cycles": {"min": min(r["cycles"] for r in rows), "max": max(r["cycles"] for r in rows)},
        "oracle_cpu_seconds": round(sum(r[1] for r in res), 1), "oracle_wall_seconds": round(wall, 1),
        "procs": a.procs,
    }
    if mixed:
        m = np.array(mixed)
        out["mixed_rel_l2_vs_oracle"] = {
            "min": float(m.min()), "median": float(np.median(m)), "p90": float(np.percentile(m, 90)),
            "max": float(m.max()), "below_1e-6": int((m < 1e-6).sum()), "of": int(m.size)}
    print(json.dumps(out, indent=1))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
