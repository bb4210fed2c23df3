"""Python interface of the engine: a batch of cases on one GPU.

It mirrors the reference program's workflow (Version-6-26-04.c:180-276): read
InputData and pattern.txt, build the levels, run V-cycles until the mass error is
below `convergence` (or the V-cycle reaches its fixed point), read the level-0
fields.  Every call goes through the C ABI of libmgfvm.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Iterable, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _abi
from ._lib import check, lib
from .inputs import CaseConfig

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def read_case(directory: str = ".", inputdata: str = "InputData",
              pattern: str = "pattern.txt", verbose: bool = False) -> CaseConfig:
    """Parse InputData + pattern.txt with the C parser (readInput :280-401)."""
    L = lib()
    c = _abi.Config()
    check(L.mgfvm_config_read(os.path.join(directory, inputdata).encode(),
                              os.path.join(directory, pattern).encode(), C.byref(c), int(verbose)))
    try:
        return CaseConfig.from_c(c)
    finally:
        L.mgfvm_config_release(C.byref(c))


def validate(cfg: CaseConfig) -> None:
    c, keep = cfg.to_c()
    check(lib().mgfvm_config_validate(C.byref(c)))
    del keep


class Solver:
    """`ncases` independent cases advanced together on one GPU (an mgfvm_ctx)."""

    def __init__(self, cases: Union[CaseConfig, Sequence[CaseConfig]], device: int = 0,
                 precision: str = "fp64", tail_level: int = -1, use_graph: bool = True,
                 sync_every: int = 64, tangent: bool = False):
        if isinstance(cases, CaseConfig):
            cases = [cases]
        self.cases: List[CaseConfig] = list(cases)
        L = lib()
        arr = (_abi.Config * len(self.cases))()
        self._keep = []
        for k, cfg in enumerate(self.cases):
            c, keep = cfg.to_c()
            arr[k] = c
            self._keep.append(keep)
        opt = _abi.Options()
        L.mgfvm_options_default(C.byref(opt))
        opt.device = device
        opt.precision = {"fp64": _abi.PREC_FP64, "mixed": _abi.PREC_MIXED}[precision]
        opt.tail_level = tail_level
        opt.use_graph = int(use_graph)
        opt.sync_every = sync_every
        opt.tangent = int(tangent)
        h = C.c_void_p()
        check(L.mgfvm_create(arr, len(self.cases), C.byref(opt), C.byref(h)))
        self._h = h
        self._lib = L
        self.device = device
        self._opt_tangent = bool(tangent)

    # ------------------------------------------------------------ lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mgfvm_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ geometry
    @property
    def ncases(self) -> int:
        return len(self.cases)

    def levels(self, case: int = 0) -> int:
        n = C.c_int()
        check(self._lib.mgfvm_num_levels(self._h, case, C.byref(n)))
        return n.value

    def dims(self, case: int, level: int) -> Tuple[int, int]:
        a, b = C.c_int(), C.c_int()
        check(self._lib.mgfvm_level_dims(self._h, case, level, C.byref(a), C.byref(b)))
        return a.value, b.value

    # ------------------------------------------------------------ running
    def reset(self) -> None:
        check(self._lib.mgfvm_reset(self._h))

    def set_inlet_profile(self, case: int, u: Iterable[float]) -> None:
        a = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        check(self._lib.mgfvm_set_inlet_profile(self._h, case, a.ctypes.data_as(_dp), a.size))

    def cycle(self, n: int = 1) -> None:
        check(self._lib.mgfvm_cycle(self._h, n))

    def solve(self, max_cycles: int, fp_tol: float = 0.0, allow_nonfinite: bool = False) -> np.ndarray:
        """Cycles each case ran.  A case whose mass error turns NaN/Inf stops there;
        the call then fails with ENONFINITE unless `allow_nonfinite` (see `diverged`)."""
        out = np.zeros(self.ncases, dtype=np.int32)
        st = self._lib.mgfvm_solve(self._h, max_cycles, fp_tol, out.ctypes.data_as(_ip))
        if not (allow_nonfinite and st == _abi.ENONFINITE):
            check(st)
        return out

    def diverged(self) -> List[int]:
        """Cases whose last recorded mass error is NaN/Inf."""
        bad = []
        for k in range(self.ncases):
            e, _ = self.history(k)
            if e.size and not np.isfinite(e[-1]):
                bad.append(k)
        return bad

    def op(self, name: Union[str, int], level: int) -> None:
        op = _abi.OP[name] if isinstance(name, str) else name
        check(self._lib.mgfvm_op(self._h, op, level))

    # ------------------------------------------------------------ data
    def field(self, case: int, level: int, name: Union[str, int]) -> np.ndarray:
        npx, npy = self.dims(case, level)
        f = _abi.FIELD[name] if isinstance(name, str) else name
        out = np.empty(npx * npy, dtype=np.float64)
        check(self._lib.mgfvm_get_field(self._h, case, level, f, out.ctypes.data_as(_dp)))
        return out.reshape(npy, npx)

    def set_field(self, case: int, level: int, name: Union[str, int], arr) -> None:
        f = _abi.FIELD[name] if isinstance(name, str) else name
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        npx, npy = self.dims(case, level)
        if a.size != npx * npy:
            raise ValueError(f"expected {npx * npy} values, got {a.size}")
        check(self._lib.mgfvm_set_field(self._h, case, level, f, a.ctypes.data_as(_dp)))

    def tag(self, case: int, level: int) -> np.ndarray:
        npx, npy = self.dims(case, level)
        out = np.empty(npx * npy, dtype=np.int32)
        check(self._lib.mgfvm_get_tag(self._h, case, level, out.ctypes.data_as(_ip)))
        return out.reshape(npy, npx)

    def obstacle_ranges(self, case: int, level: int) -> np.ndarray:
        n = len(self.cases[case].obstacles)
        out = np.zeros(max(4 * n, 4), dtype=np.int32)
        check(self._lib.mgfvm_get_obstacle_ranges(self._h, case, level, out.ctypes.data_as(_ip)))
        return out[:4 * n].reshape(-1, 4)

    def history(self, case: int = 0) -> Tuple[np.ndarray, np.ndarray]:
        n = C.c_int()
        check(self._lib.mgfvm_history(self._h, case, None, None, 0, C.byref(n)))
        e = np.zeros(max(n.value, 1))
        d = np.zeros(max(n.value, 1))
        check(self._lib.mgfvm_history(self._h, case, e.ctypes.data_as(_dp), d.ctypes.data_as(_dp),
                                      n.value, C.byref(n)))
        return e[:n.value], d[:n.value]

    @property
    def kernel_launches(self) -> int:
        n = C.c_longlong()
        check(self._lib.mgfvm_kernel_launches(self._h, C.byref(n)))
        return n.value

    @property
    def last_elapsed_ms(self) -> float:
        v = C.c_double()
        check(self._lib.mgfvm_last_elapsed_ms(self._h, C.byref(v)))
        return v.value

    def time_op(self, name: Union[str, int], level: int, reps: int = 10) -> Tuple[float, int]:
        """(milliseconds, kernel launches) of `reps` back-to-back runs of one op, timed with
        CUDA events on the context stream."""
        op = _abi.OP[name] if isinstance(name, str) else name
        ms, n = C.c_double(), C.c_int()
        check(self._lib.mgfvm_time_op(self._h, op, level, reps, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    KERNELS = ["fluxes", "asm", "mass_coefp", "update", "pfix", "bound", "smooth", "copy", "restv_fluxes",
               "restrict", "prol_corr", "prol_apply", "tail", "endcycle", "prol_apply_end", "smooth_mixed", "pfix_bound", "pp_level",
               "tail_tan", "level_visit", "smooth_tma", "band_visit", "coarse_cycle"]

    def profile_cycle(self):
        """One directly-launched V-cycle with an event after every kernel: a list of
        (kernel name, level, milliseconds)."""
        cap = 4096
        ms = np.zeros(cap)
        kid = np.zeros(cap, dtype=np.int32)
        lvl = np.zeros(cap, dtype=np.int32)
        n = C.c_int()
        check(self._lib.mgfvm_profile_cycle(self._h, ms.ctypes.data_as(_dp), kid.ctypes.data_as(_ip),
                                            lvl.ctypes.data_as(_ip), cap, C.byref(n)))
        return [(self.KERNELS[kid[k]], int(lvl[k]), float(ms[k])) for k in range(min(n.value, cap))]

    def field_view(self, case: int, level: int, name: str):
        """A torch float64 CUDA tensor (npy, npx) sharing the engine's memory of one
        array (no copy).  Valid while the solver is open; order work on it with the
        context stream (`stream`), e.g. by running torch work on
        torch.cuda.ExternalStream(solver.stream)."""
        import torch
        ptr, nx, ny = C.c_void_p(), C.c_int(), C.c_int()
        check(self._lib.mgfvm_field_device_ptr(self._h, case, level, _abi.FIELD[name], C.byref(ptr),
                                                C.byref(nx), C.byref(ny)))

        class _View:
            __cuda_array_interface__ = {"shape": (ny.value, nx.value), "typestr": "<f8",
                                        "data": (ptr.value, False), "version": 2, "strides": None}
        t = torch.as_tensor(_View(), device=torch.device("cuda", self.device))
        return t

    @property
    def tuning(self) -> dict:
        """Per-level schedule choices {smooth_units, smooth_threads, asm_slices,
        restrict_slices} (lists of MAX_LEVELS ints, 0 = default)."""
        t = _abi.Tuning()
        check(self._lib.mgfvm_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **per_level) -> None:
        """Replace schedule choices, e.g. set_tuning(smooth_units={0: 4}, asm_slices={1: 1});
        unspecified levels keep their values.  Scalar fields (tma_first_wait) take an int."""
        t = _abi.Tuning()
        check(self._lib.mgfvm_get_tuning(self._h, C.byref(t)))
        for key, vals in per_level.items():
            if isinstance(vals, (int, np.integer)):
                setattr(t, key, int(vals))
                continue
            arr = getattr(t, key)
            for lv, v in (vals.items() if isinstance(vals, dict) else enumerate(vals)):
                arr[lv] = int(v)
        check(self._lib.mgfvm_set_tuning(self._h, C.byref(t)))

    def autotune(self, cycles: int = 5) -> Tuple[float, float, dict]:
        """Time candidate schedules on this batch and keep the fastest; the batch's state
        is unchanged.  Returns (ms per cycle before, after, chosen tuning)."""
        t = _abi.Tuning()
        a, b = C.c_double(), C.c_double()
        check(self._lib.mgfvm_autotune(self._h, cycles, C.byref(t), C.byref(a), C.byref(b)))
        return a.value, b.value, t.as_dict()

    # ------------------------------------------------------------ derivatives
    def set_direction(self, case: int, kind: str, index: int = 0) -> None:
        """Tangent contexts: differentiate case `case` along `kind` ("inlet" face
        `index`, "amuf", "prsc"); the case restarts from its initial state."""
        check(self._lib.mgfvm_set_direction(self._h, case, _abi.DIR[kind], index))

    def tangent(self, case: int, level: int, name: Union[str, int]) -> np.ndarray:
        """Derivative of a field along the case's direction (npy, npx)."""
        npx, npy = self.dims(case, level)
        f = _abi.FIELD[name] if isinstance(name, str) else name
        out = np.empty(npx * npy, dtype=np.float64)
        check(self._lib.mgfvm_get_tangent(self._h, case, level, f, out.ctypes.data_as(_dp)))
        return out.reshape(npy, npx)

    def objective(self, case: int = 0) -> Tuple[float, Optional[float]]:
        """(J, dJ): the pressure drop plus mean outlet scalar of the level-0 state
        (mgfvm_objective) and, in a tangent context, its derivative."""
        j = C.c_double()
        d = C.c_double()
        tan = bool(self._opt_tangent)
        check(self._lib.mgfvm_objective(self._h, case, C.byref(j), C.byref(d) if tan else None))
        return j.value, (d.value if tan else None)

    def adjoint(self, cycles: int) -> None:
        """Reverse mode (mgfvm_adjoint): every case restarts from its initial state, runs
        `cycles` V-cycles, and the transposed cycles carry the adjoint of J back to the
        inputs.  Read the result with adjoint_gradient(case)."""
        check(self._lib.mgfvm_adjoint(self._h, int(cycles)))

    def adjoint_gradient(self, case: int = 0, allow_nonfinite: bool = False) -> Tuple[float, np.ndarray, float, float]:
        """(J, dJ/dinlet (nfy values), dJ/damuf, dJ/dprsc) of the last adjoint run.  A case
        that turned non-finite raises ENONFINITE unless `allow_nonfinite` (its gradient is
        then NaN)."""
        g_in = np.zeros(int(self.cases[case].nfy))
        j, ga, gp = C.c_double(), C.c_double(), C.c_double()
        st = self._lib.mgfvm_adjoint_gradient(self._h, case, C.byref(j), g_in.ctypes.data_as(_dp), C.byref(ga),
                                              C.byref(gp))
        if not (allow_nonfinite and st == _abi.ENONFINITE):
            check(st)
        return j.value, g_in, ga.value, gp.value

    @property
    def transfer_bytes(self) -> Tuple[int, int]:
        """(host->device, device->host) bytes copied by this context so far."""
        a, b = C.c_longlong(), C.c_longlong()
        check(self._lib.mgfvm_transfer_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(self._lib.mgfvm_stream(self._h, C.byref(s)))
        return s.value or 0


def gradient(cfg: CaseConfig, inlet_u=None, cycles: int = 100, device: int = 0):
    """J after `cycles` V-cycles from cfg's initial state (with the per-face inlet
    profile `inlet_u`, or none) and its exact derivatives with respect to every inlet
    face (nfy values), amuf and prsc: one batched tangent run (mgfvm_gradient).
    Returns (J, dJ_dinlet, dJ_damuf, dJ_dprsc)."""
    c, keep = cfg.to_c()
    prof = np.ascontiguousarray(np.zeros(0) if inlet_u is None else np.asarray(inlet_u, dtype=np.float64))
    nf = int(cfg.nfy)
    g_in = np.zeros(nf)
    j, ga, gp = C.c_double(), C.c_double(), C.c_double()
    check(lib().mgfvm_gradient(C.byref(c), prof.ctypes.data_as(_dp) if prof.size else None, int(prof.size),
                               int(cycles), int(device), C.byref(j), g_in.ctypes.data_as(_dp), C.byref(ga),
                               C.byref(gp)))
    del keep
    return j.value, g_in, ga.value, gp.value
