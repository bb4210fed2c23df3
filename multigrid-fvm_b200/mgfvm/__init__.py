"""mgfvm — B200 engine for the staggered-grid SIMPLE solver with FAS multigrid
V-cycles of akashu4295/Multigrid-FVM (Version-6-26-04.c).

    from mgfvm import CaseConfig, Solver
    with Solver([cfg_a, cfg_b]) as s:      # one batch, one GPU
        cycles = s.solve(max_cycles=5000, fp_tol=1e-10)
        u = s.field(0, 0, "u")

The compute path is libmgfvm.so (CUDA, sm_100a) behind the C ABI of include/mgfvm.h.
"""
from ._abi import FIELDS, OPS  # noqa: F401
from ._lib import MgfvmError, lib  # noqa: F401
from .inputs import CaseConfig, obstacle_ranges  # noqa: F401
from .solver import Solver, gradient, read_case, validate  # noqa: F401

__all__ = ["CaseConfig", "Solver", "gradient", "read_case", "validate", "MgfvmError", "FIELDS", "OPS",
           "obstacle_ranges", "lib"]
