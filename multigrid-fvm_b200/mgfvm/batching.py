"""Spreading independent cases over GPUs (one process per GPU).

Cases never exchange data, so a multi-GPU run is a partition of the batch: each rank
builds one context for its share and no collective sits on the data path; only the
small per-case results (cycle counts, histories, level-0 fields) are gathered.
"""
from __future__ import annotations

from typing import List, Sequence

from .inputs import CaseConfig


def case_cost(cfg: CaseConfig) -> float:
    """Work of one solve: cells over all levels times the V-cycles it may run."""
    cells = sum((cfg.nfx >> ig) * (cfg.nfy >> ig) for ig in range(cfg.ngrid))
    return float(cells) * max(1, cfg.nvcycle)


def shard(cases: Sequence[CaseConfig], world: int) -> List[List[int]]:
    """Indices of the cases of each rank: longest-processing-time-first greedy
    partition on case_cost, so ranks finish close together."""
    order = sorted(range(len(cases)), key=lambda k: -case_cost(cases[k]))
    load = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += case_cost(cases[k])
    return [sorted(p) for p in parts]
