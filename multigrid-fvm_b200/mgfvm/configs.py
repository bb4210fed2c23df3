"""The benchmark workloads, as seeded synthetic cases.

  c0  plain channel, 64 x 64, ngrid 3, Jacobi, Re 100, no obstacles
  c1  obstacle flow, 256 x 256, ngrid 5, red-black Gauss-Seidel, Re 10 or 100, a
      staggered lattice of 1x1 blocks on a 16 x 16 base grid (spacing 1, porosity
      0.75) with seeded full-pixel random moves
  c2  a batch of independent cases of mixed size (64/128/256, coarsest level 8 x 8),
      random particles on a 16 x 16 base grid at porosity U[0.6, 0.9], Re in
      {10, 50, 100, 200}
  c3  1024 x 1024, ngrid 7, Re 200, staggered lattice on a 32 x 32 base with
      quarter-pixel moves (spacing 1: porosity 0.75; 0.7 is not reachable with an
      integer spacing)
  c4  cases at 256 x 256, ngrid 5, Re 100, random particles at porosity
      U[0.65, 0.85], per-face inlet profile 1 + 0.1 N(0, 1)

Every case uses the left boundary as the inlet (u = 1, v = 0, sc = 1 on every row,
InputData line 4), no-slip walls at the bottom and top, and the zero-gradient outflow
(ibc_xp = 4) on the right, with relxm 0.7, relxp 0.3, nswpm 2, nswpp 10, prsc 1.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

from . import patterns
from .inputs import CaseConfig


def _base(n: int, ngrid: int, re: float, isolve: int, nvcycle: int = 5000) -> CaseConfig:
    return CaseConfig(nfx=n, nfy=n, ngrid=ngrid, ig_obs=0, ibeg_obs=0, ig_inlt=0, ig_outlt=0,
                      nvcycle=nvcycle, nswpm=2, nswpp=10, isolve=isolve, omega=1.0,
                      convergence=1e-6, xl=1.0, yl=1.0, amuf=1.0 / re, prsc=1.0, relxm=0.7,
                      relxp=0.3, ibc_xm=1, ibc_xp=4, ibc_ym=1, ibc_yp=1,
                      bc_xm=(1.0, 0.0, 0.0, 1.0), bc_xp=(0.0, 0.0, 0.0, 0.0),
                      bc_ym=(0.0, 0.0, 0.0, 0.0), bc_yp=(0.0, 0.0, 0.0, 0.0),
                      guess=(0.0, 0.0, 0.0, 0.0), sc_obs=0.0)


def c0(isolve: int = 1) -> CaseConfig:
    """64 x 64 channel, ngrid 3, Jacobi, Re 100, nvcycle up to 2000."""
    return _base(64, 3, 100.0, isolve, nvcycle=2000)


def level_of(n: int, cells: int) -> int:
    """Index of the level of an n-cell grid that has `cells` cells per side."""
    lv = 0
    while (n >> lv) > cells:
        lv += 1
    if (n >> lv) != cells:
        raise ValueError(f"{n} is not {cells} * 2^k")
    return lv


def c1(re: float = 100.0, seed: int = 1, n: int = 256, ngrid: int = 5, isolve: int = 2,
       nvcycle: int = 2000) -> CaseConfig:
    """Staggered obstacle flow; obstacles defined on the 16-cell level (ig_obs = that
    level + 1)."""
    g = patterns.staggered_grid(16, "full", 1, 1, variant=3, seed=seed)
    cfg = _base(n, ngrid, re, isolve, nvcycle=nvcycle)
    ig16 = level_of(n, 16)
    if ig16 >= ngrid:
        raise ValueError("the 16-cell level must exist")
    return cfg.replace(ig_obs=ig16 + 1, obstacles=patterns.pixels(g))


def c1_pair(seed: int = 1) -> List[CaseConfig]:
    """The two Reynolds numbers of the obstacle-flow workload."""
    return [c1(10.0, seed), c1(100.0, seed)]


def c2(ncases: int = 512, seed: int = 2, sizes=(64, 128, 256), isolve: int = 2) -> List[CaseConfig]:
    rng = np.random.default_rng(seed)
    out = []
    for k in range(ncases):
        n = int(rng.choice(sizes))
        ngrid = level_of(n, 8) + 1
        poro = float(rng.uniform(0.6, 0.9))
        re = float(rng.choice([10.0, 50.0, 100.0, 200.0]))
        _, rects = patterns.random_grid(16, 1.0 - poro, seed=int(rng.integers(1 << 62)))
        cfg = _base(n, ngrid, re, isolve)
        out.append(cfg.replace(ig_obs=level_of(n, 16) + 1, obstacles=rects))
    return out


def c3(seed: int = 3, isolve: int = 2) -> CaseConfig:
    g = patterns.staggered_grid(32, "quarter", 1, 1, variant=3, seed=seed)
    cfg = _base(1024, 7, 200.0, isolve)
    return cfg.replace(ig_obs=level_of(1024, 128) + 1, obstacles=patterns.pixels(g))


def c4(ncases: int = 64, seed: int = 4, n: int = 256, isolve: int = 2
       ) -> Tuple[List[CaseConfig], List[np.ndarray]]:
    """Cases and their per-face inlet u profiles."""
    rng = np.random.default_rng(seed)
    cases, profiles = [], []
    for _ in range(ncases):
        poro = float(rng.uniform(0.65, 0.85))
        _, rects = patterns.random_grid(16, 1.0 - poro, seed=int(rng.integers(1 << 62)))
        cases.append(_base(n, 5, 100.0, isolve).replace(ig_obs=level_of(n, 16) + 1, obstacles=rects))
        profiles.append(1.0 + 0.1 * rng.standard_normal(n))
    return cases, profiles


def small(n: int = 32, ngrid: int = 3, isolve: int = 1, **kw) -> CaseConfig:
    """A small channel for tests."""
    return _base(n, ngrid, 100.0, isolve).replace(**kw)
