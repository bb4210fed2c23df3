"""Case configurations: the reference's InputData / pattern.txt pair as a Python object.

`CaseConfig` holds exactly the values readInput() and read_obstacle_data() read
(Version-6-26-04.c:280-401, :2367-2400; format in README.md:6-29).  It converts to
the C struct of include/mgfvm.h, and writes the two files in the reference's
layout so the same case can be run by the reference binary, by the command-line
tool of this package, or through the C ABI.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

from . import _abi


@dataclass
class CaseConfig:
    # InputData line 1
    nfx: int = 64
    nfy: int = 64
    ngrid: int = 3
    ig_obs: int = 0
    ibeg_obs: int = 0
    ig_inlt: int = 0
    ig_outlt: int = 0
    nvcycle: int = 2000
    nswpm: int = 2
    nswpp: int = 10
    isolve: int = 1
    omega: float = 1.0
    convergence: float = 1e-6
    # line 2
    xl: float = 1.0
    yl: float = 1.0
    amuf: float = 0.01
    prsc: float = 1.0
    relxm: float = 0.7
    relxp: float = 0.3
    # line 3
    ibc_xm: int = 1
    ibc_xp: int = 4
    ibc_ym: int = 1
    ibc_yp: int = 1
    # lines 4-7: (u, v, p, sc) on x-, x+, y-, y+
    bc_xm: Tuple[float, float, float, float] = (1.0, 0.0, 0.0, 1.0)
    bc_xp: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    bc_ym: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    bc_yp: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    # line 8
    guess: Tuple[float, float, float, float] = (0.0, 0.0, 0.0, 0.0)
    # line 9
    sc_obs: float = 0.0
    # discrete inlets / outlets: (jf, jl, u, v, sc)
    inlets: List[Tuple[int, int, float, float, float]] = field(default_factory=list)
    outlets: List[Tuple[int, int, float, float, float]] = field(default_factory=list)
    # pattern.txt rectangles (if, il, jf, jl), 1-based on level ig_obs-1
    obstacles: List[Tuple[int, int, int, int]] = field(default_factory=list)

    def replace(self, **kw) -> "CaseConfig":
        return dataclasses.replace(self, **kw)

    # ------------------------------------------------------------ geometry
    def level_dims(self, ig: int) -> Tuple[int, int]:
        """(npx, npy) of level ig (Version-6-26-04.c:408-411)."""
        return self.nfx // (1 << ig) + 2, self.nfy // (1 << ig) + 2

    # ------------------------------------------------------------ C struct
    def to_c(self) -> Tuple[_abi.Config, object]:
        """The C struct plus the object that keeps its obstacle array alive."""
        c = _abi.Config()
        for name in ("nfx", "nfy", "ngrid", "ig_obs", "ibeg_obs", "ig_inlt", "ig_outlt",
                     "nvcycle", "nswpm", "nswpp", "isolve", "omega", "convergence", "xl",
                     "yl", "amuf", "prsc", "relxm", "relxp", "ibc_xm", "ibc_xp", "ibc_ym",
                     "ibc_yp", "sc_obs"):
            setattr(c, name, getattr(self, name))
        for side in ("xm", "xp", "ym", "yp"):
            vals = getattr(self, "bc_" + side)
            for k, q in enumerate("uvp"):
                setattr(c, f"{q}_{side}", float(vals[k]))
            setattr(c, f"sc_{side}", float(vals[3]))
        c.u_guess, c.v_guess, c.p_guess, c.sc_guess = (float(x) for x in self.guess)
        if len(self.inlets) > _abi.MAX_PORTS or len(self.outlets) > _abi.MAX_PORTS:
            raise ValueError(f"at most {_abi.MAX_PORTS} inlets and outlets")
        c.ninlt = len(self.inlets)
        for k, (jf, jl, u, v, s) in enumerate(self.inlets):
            c.jfinlt[k], c.jlinlt[k], c.uinlt[k], c.vinlt[k], c.scinlt[k] = jf, jl, u, v, s
        c.noutlt = len(self.outlets)
        for k, (jf, jl, u, v, s) in enumerate(self.outlets):
            c.jfoutlt[k], c.jloutlt[k], c.uoutlt[k], c.voutlt[k], c.scoutlt[k] = jf, jl, u, v, s
        n = len(self.obstacles)
        arr = (C.c_int * max(4 * n, 4))()
        for k, rect in enumerate(self.obstacles):
            for t in range(4):
                arr[4 * k + t] = int(rect[t])
        c.nobs = n
        c.obs = C.cast(arr, C.POINTER(C.c_int))
        c.dpdxm = 0.0
        c.dpdym = 0.0
        return c, arr

    @staticmethod
    def from_c(c: _abi.Config) -> "CaseConfig":
        kw = {}
        for name in ("nfx", "nfy", "ngrid", "ig_obs", "ibeg_obs", "ig_inlt", "ig_outlt",
                     "nvcycle", "nswpm", "nswpp", "isolve", "omega", "convergence", "xl",
                     "yl", "amuf", "prsc", "relxm", "relxp", "ibc_xm", "ibc_xp", "ibc_ym",
                     "ibc_yp", "sc_obs"):
            kw[name] = getattr(c, name)
        for side in ("xm", "xp", "ym", "yp"):
            kw["bc_" + side] = tuple(getattr(c, f"{q}_{side}") for q in ("u", "v", "p", "sc"))
        kw["guess"] = (c.u_guess, c.v_guess, c.p_guess, c.sc_guess)
        kw["inlets"] = [(c.jfinlt[k], c.jlinlt[k], c.uinlt[k], c.vinlt[k], c.scinlt[k])
                        for k in range(c.ninlt)]
        kw["outlets"] = [(c.jfoutlt[k], c.jloutlt[k], c.uoutlt[k], c.voutlt[k], c.scoutlt[k])
                         for k in range(c.noutlt)]
        kw["obstacles"] = [tuple(c.obs[4 * k + t] for t in range(4)) for k in range(c.nobs)]
        return CaseConfig(**kw)

    # ------------------------------------------------------------ files
    def inputdata_text(self) -> str:
        """InputData in the reference's line layout (README.md:6-29)."""
        g = lambda x: repr(float(x))
        lines = [
            f"{self.nfx} {self.nfy} {self.ngrid} {self.ig_obs} {self.ibeg_obs} {self.ig_inlt} "
            f"{self.ig_outlt} {self.nvcycle} {self.nswpm} {self.nswpp} {self.isolve} "
            f"{g(self.omega)} {g(self.convergence)}",
            " ".join(g(x) for x in (self.xl, self.yl, self.amuf, self.prsc, self.relxm, self.relxp)),
            f"{self.ibc_xm} {self.ibc_xp} {self.ibc_ym} {self.ibc_yp}",
            " ".join(g(x) for x in self.bc_xm),
            " ".join(g(x) for x in self.bc_xp),
            " ".join(g(x) for x in self.bc_ym),
            " ".join(g(x) for x in self.bc_yp),
            " ".join(g(x) for x in self.guess),
            g(self.sc_obs),
            str(len(self.inlets)),
        ]
        lines += [f"{jf} {jl} {g(u)} {g(v)} {g(s)}" for jf, jl, u, v, s in self.inlets]
        lines.append(str(len(self.outlets)))
        lines += [f"{jf} {jl} {g(u)} {g(v)} {g(s)}" for jf, jl, u, v, s in self.outlets]
        return "\n".join(lines) + "\n"

    def pattern_text(self) -> str:
        """pattern.txt: the count, then one `if il jf jl` line per obstacle (:2375-2385)."""
        rows = [str(len(self.obstacles))]
        rows += [" ".join(str(int(x)) for x in r) for r in self.obstacles]
        return "\n".join(rows) + "\n"

    def write(self, directory: str) -> Tuple[str, str]:
        """Write InputData and pattern.txt into `directory`; returns their paths."""
        os.makedirs(directory, exist_ok=True)
        pin = os.path.join(directory, "InputData")
        ppat = os.path.join(directory, "pattern.txt")
        with open(pin, "w") as f:
            f.write(self.inputdata_text())
        with open(ppat, "w") as f:
            f.write(self.pattern_text())
        return pin, ppat


def obstacle_ranges(cfg: CaseConfig, ig: int) -> List[Tuple[int, int, int, int]]:
    """Obstacle index ranges of level ig (AllocateMemorySoA, Version-6-26-04.c:468-478);
    levels at or above ig_obs take the empty range (1, 0, 1, 0)."""
    out = []
    for (i0, i1, j0, j1) in cfg.obstacles:
        if ig < cfg.ig_obs:
            fac = 1 << (cfg.ig_obs - 1 - ig)
            out.append(((i0 + cfg.ibeg_obs - 1) * fac + 1, (i1 + cfg.ibeg_obs) * fac,
                        (j0 - 1) * fac + 1, j1 * fac))
        else:
            out.append((1, 0, 1, 0))
    return out


def cases_share_schedule(cases: Sequence[CaseConfig]) -> bool:
    """Cases batched in one context must share the smoother and sweep counts."""
    first = cases[0]
    return all(c.isolve == first.isolve and c.nswpm == first.nswpm and c.nswpp == first.nswpp
               for c in cases)
