"""Multi-GPU host path on CPU: two gloo ranks partition a batch of independent cases
(mgfvm.batching.shard), advance their shares (CPU oracle standing in for the device),
and gather per-case results; the union equals a single-rank run."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _cases():
    from mgfvm import configs
    return [configs.small(16, 2, isolve=1 + (k % 2), relxp=0.3 + 0.05 * k, nvcycle=3 + k) for k in range(7)]


def _run(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    repo = os.path.dirname(here)
    sys.path.insert(0, os.path.join(repo, "multigrid-fvm_b200"))
    sys.path.insert(0, os.path.join(repo, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from mgfvm.batching import shard
    from oracle import OracleCase
    cases = _cases()
    mine = shard(cases, world)[rank]
    res = {}
    for k in mine:
        o = OracleCase(cases[k])
        o.cycle(cases[k].nvcycle)
        res[k] = (o.history()[0].tolist(), float(o.get(0, "u").sum()))
    gathered = [None] * world
    dist.all_gather_object(gathered, res)
    if rank == 0:
        merged = {}
        for g in gathered:
            assert not set(g) & set(merged), "a case was solved on two ranks"
            merged.update(g)
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_partition_equals_single_rank(oracle_built):
    from mgfvm.batching import shard
    from oracle import OracleCase
    cases = _cases()
    parts = shard(cases, 2)
    assert sorted(parts[0] + parts[1]) == list(range(len(cases)))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(len(cases)))
    for k, cfg in enumerate(cases):
        o = OracleCase(cfg)
        o.cycle(cfg.nvcycle)
        assert merged[k][0] == o.history()[0].tolist()
        assert merged[k][1] == float(o.get(0, "u").sum())


def test_shard_balances_cost():
    from mgfvm import configs
    from mgfvm.batching import case_cost, shard
    cases = configs.c2(40, seed=9)
    parts = shard(cases, 4)
    loads = [sum(case_cost(cases[k]) for k in p) for p in parts]
    assert max(loads) / min(loads) < 1.3
