"""Seeded obstacle patterns (wrappers of the C generators in csrc/host/patterns.c).

The reference's generators (create_patterns_staggered.c, create_patterns_random.c) are
interactive and seeded with time(NULL); these take every choice as an argument and a
64-bit seed, and return obstacle lists in the reference's pattern.txt row format.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Tuple

import numpy as np

from ._lib import check, lib

_ip = C.POINTER(C.c_int)

SHIFT_SCALE = {"quarter": 4, "half": 2, "full": 1}


def staggered_grid(n_base: int, shift: str = "full", spacing_x: int = 1, spacing_y: int = 1,
                   variant: int = 3, seed: int = 0) -> np.ndarray:
    """Occupancy grid of a staggered lattice (create_patterns_staggered.c:71-200):
    variant 1 inline, 2 staggered, >= 3 seeded random perturbations."""
    scale = SHIFT_SCALE[shift]
    dim = n_base * scale
    g = np.zeros(dim * dim, dtype=np.int32)
    check(lib().mgfvm_pattern_staggered(n_base, scale, spacing_x, spacing_y, variant,
                                        seed & 0xFFFFFFFFFFFFFFFF, g.ctypes.data_as(_ip)))
    return g.reshape(dim, dim)


def random_grid(n_grid: int, ratio: float, pct: Tuple[float, float, float] = (50.0, 30.0, 20.0),
                seed: int = 0) -> Tuple[np.ndarray, List[Tuple[int, int, int, int]]]:
    """Random non-overlapping square particles (create_patterns_random.c:18-181); returns the
    grid and the particle rectangles (r1, r2, c1, c2), 1-based."""
    g = np.zeros(n_grid * n_grid, dtype=np.int32)
    cap = n_grid * n_grid
    rects = np.zeros(4 * cap, dtype=np.int32)
    n = C.c_int()
    check(lib().mgfvm_pattern_random(n_grid, ratio, pct[0], pct[1], pct[2], seed & 0xFFFFFFFFFFFFFFFF,
                                     g.ctypes.data_as(_ip), rects.ctypes.data_as(_ip), cap, C.byref(n)))
    r = rects[:4 * n.value].reshape(-1, 4)
    return g.reshape(n_grid, n_grid), [tuple(int(v) for v in row) for row in r]


def pixels(grid: np.ndarray) -> List[Tuple[int, int, int, int]]:
    """One obstacle per occupied pixel, (r+1, r+1, c+1, c+1), row-major
    (create_patterns_staggered.c:47-54)."""
    dim = grid.shape[0]
    g = np.ascontiguousarray(grid, dtype=np.int32)
    n = C.c_int()
    check(lib().mgfvm_pattern_pixels(g.ctypes.data_as(_ip), dim, None, 0, C.byref(n)))
    out = np.zeros(4 * max(n.value, 1), dtype=np.int32)
    check(lib().mgfvm_pattern_pixels(g.ctypes.data_as(_ip), dim, out.ctypes.data_as(_ip), n.value, C.byref(n)))
    return [tuple(int(v) for v in out[4 * k:4 * k + 4]) for k in range(n.value)]


def porosity(grid: np.ndarray) -> float:
    return 1.0 - float(np.count_nonzero(grid)) / grid.size
