"""TEST INFRASTRUCTURE ONLY: Python access to the CPU checkers of the CUDA engine.

  OracleCase    the C restatement of the reference V-cycle (oracle/liboracle.so)
  RefCase       the unmodified reference Version-6-26-04.c compiled with gcc through
                oracle/ref_harness.c (oracle/_ref/libmgref.so); present only where the
                reference source was available when it was built

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module.  The product path (multigrid-fvm_b200/mgfvm) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "multigrid-fvm_b200"))
from mgfvm import _abi  # noqa: E402
from mgfvm.inputs import CaseConfig  # noqa: E402

ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmgref.so")
REF_BIN = os.path.join(HERE, "_ref", "ref_solver")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/ when the environment variable MGFVM_REF_DIR names
    the directory holding the reference's Version-6-26-04.c)."""
    ref = os.environ.get("MGFVM_REF_DIR")
    out = subprocess.run(["make", "-C", HERE, "all"] + ([f"REF_DIR={ref}"] if ref else []),
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_olib = None


def _oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = C.CDLL(ORACLE_SO)
        lib.orc_create.argtypes = [C.POINTER(_abi.Config), _dp, C.c_int, C.POINTER(C.c_void_p)]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_ngrid.argtypes = [C.c_void_p]
        lib.orc_dims.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
        lib.orc_get.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        lib.orc_set.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        lib.orc_get_tag.argtypes = [C.c_void_p, C.c_int, _ip]
        lib.orc_get_obstacle_ranges.argtypes = [C.c_void_p, C.c_int, _ip]
        lib.orc_cycle.argtypes = [C.c_void_p]
        lib.orc_solve.argtypes = [C.c_void_p, C.c_int, C.c_double]
        lib.orc_history.argtypes = [C.c_void_p, _dp, _dp, C.c_int]
        lib.orc_op.argtypes = [C.c_void_p, C.c_int, C.c_int]
        lib.orc_last_err.argtypes = [C.c_void_p]
        lib.orc_last_err.restype = C.c_double
        _olib = lib
    return _olib


class OracleCase:
    """One case run by the C restatement (mgfvm_oracle.c)."""

    def __init__(self, cfg: CaseConfig, inlet_u=None):
        self.lib = _oracle_lib()
        self.cfg = cfg
        c, self._keep = cfg.to_c()
        h = C.c_void_p()
        prof = None
        n = 0
        if inlet_u is not None:
            prof = np.ascontiguousarray(inlet_u, dtype=np.float64)
            n = prof.size
        rc = self.lib.orc_create(C.byref(c), prof.ctypes.data_as(_dp) if prof is not None else None,
                                 n, C.byref(h))
        if rc != 0:
            raise RuntimeError(f"orc_create failed with status {rc}")
        self.h = h

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ngrid(self):
        return self.lib.orc_ngrid(self.h)

    def dims(self, level):
        a, b = C.c_int(), C.c_int()
        self.lib.orc_dims(self.h, level, C.byref(a), C.byref(b))
        return a.value, b.value

    def get(self, level, field):
        npx, npy = self.dims(level)
        out = np.empty(npx * npy, dtype=np.float64)
        f = _abi.FIELD[field] if isinstance(field, str) else field
        self.lib.orc_get(self.h, level, f, out.ctypes.data_as(_dp))
        return out.reshape(npy, npx)

    def set(self, level, field, arr):
        f = _abi.FIELD[field] if isinstance(field, str) else field
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        self.lib.orc_set(self.h, level, f, a.ctypes.data_as(_dp))

    def tag(self, level):
        npx, npy = self.dims(level)
        out = np.empty(npx * npy, dtype=np.int32)
        self.lib.orc_get_tag(self.h, level, out.ctypes.data_as(_ip))
        return out.reshape(npy, npx)

    def obstacle_ranges(self, level):
        out = np.zeros(max(4 * len(self.cfg.obstacles), 4), dtype=np.int32)
        self.lib.orc_get_obstacle_ranges(self.h, level, out.ctypes.data_as(_ip))
        return out[:4 * len(self.cfg.obstacles)].reshape(-1, 4)

    def cycle(self, n=1):
        for _ in range(n):
            self.lib.orc_cycle(self.h)

    def solve(self, max_cycles, fp_tol):
        return self.lib.orc_solve(self.h, max_cycles, fp_tol)

    def op(self, name, level):
        op = _abi.OP[name] if isinstance(name, str) else name
        rc = self.lib.orc_op(self.h, op, level)
        if rc != 0:
            raise RuntimeError(f"orc_op({name}, {level}) -> {rc}")

    def last_err(self):
        """Mass error of the last masserror call (any level)."""
        return self.lib.orc_last_err(self.h)

    def history(self):
        n = self.lib.orc_history(self.h, None, None, 0)
        e = np.empty(max(n, 1))
        d = np.empty(max(n, 1))
        self.lib.orc_history(self.h, e.ctypes.data_as(_dp), d.ctypes.data_as(_dp), n)
        return e[:n], d[:n]


# ---------------------------------------------------------------- reference
_rlib = None


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ref_lib():
    global _rlib
    if _rlib is None:
        lib = C.CDLL(REF_SO)
        lib.ref_load.argtypes = [C.c_char_p, _dp, C.c_int]
        lib.ref_get.argtypes = [C.c_int, C.c_int, _dp]
        lib.ref_set.argtypes = [C.c_int, C.c_int, _dp]
        lib.ref_get_tag.argtypes = [C.c_int, _ip]
        lib.ref_get_obstacle_ranges.argtypes = [C.c_int, _ip]
        lib.ref_cycle.argtypes = [C.c_int]
        lib.ref_history.argtypes = [_dp, C.c_int]
        lib.ref_op.argtypes = [C.c_int, C.c_int, C.c_int]
        lib.ref_last_err.argtypes = [C.c_int]
        lib.ref_last_err.restype = C.c_double
        lib.ref_time_cycles.argtypes = [C.c_int, C.c_int]
        lib.ref_time_cycles.restype = C.c_double
        lib.ref_get_config.argtypes = [_ip, _dp, _ip, _ip, _dp]
        lib.ref_verbose.argtypes = [C.c_int]
        _rlib = lib
    return _rlib


class RefCase:
    """The reference itself (one case at a time: its state is process-global)."""

    def __init__(self, cfg: CaseConfig, inlet_u=None, workdir=None):
        """cfg = None: `workdir` already holds the case's InputData and pattern.txt."""
        self.lib = _ref_lib()
        self.cfg = cfg
        self._tmp = None
        if workdir is None:
            self._tmp = tempfile.TemporaryDirectory()
            workdir = self._tmp.name
        if cfg is not None:
            cfg.write(workdir)
        prof, n = None, 0
        if inlet_u is not None:
            prof = np.ascontiguousarray(inlet_u, dtype=np.float64)
            n = prof.size
        rc = self.lib.ref_load(workdir.encode(), prof.ctypes.data_as(_dp) if prof is not None else None, n)
        if rc != 0:
            raise RuntimeError(f"reference readInput failed ({rc})")
        self.icyc = 0

    def dims(self, level):
        return self.lib.ref_npx(level), self.lib.ref_npy(level)

    @property
    def ngrid(self):
        return self.lib.ref_ngrid()

    def get(self, level, field):
        npx, npy = self.dims(level)
        out = np.empty(npx * npy, dtype=np.float64)
        f = _abi.FIELD[field] if isinstance(field, str) else field
        self.lib.ref_get(level, f, out.ctypes.data_as(_dp))
        return out.reshape(npy, npx)

    def set(self, level, field, arr):
        f = _abi.FIELD[field] if isinstance(field, str) else field
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        self.lib.ref_set(level, f, a.ctypes.data_as(_dp))

    def tag(self, level):
        npx, npy = self.dims(level)
        out = np.empty(npx * npy, dtype=np.int32)
        self.lib.ref_get_tag(level, out.ctypes.data_as(_ip))
        return out.reshape(npy, npx)

    def obstacle_ranges(self, level):
        n = len(self.cfg.obstacles)
        out = np.zeros(max(4 * n, 4), dtype=np.int32)
        self.lib.ref_get_obstacle_ranges(level, out.ctypes.data_as(_ip))
        return out[:4 * n].reshape(-1, 4)

    def cycle(self, n=1):
        for _ in range(n):
            self.lib.ref_cycle(self.icyc)
            self.icyc += 1

    def op(self, name, level, slot=0):
        op = _abi.OP[name] if isinstance(name, str) else name
        rc = self.lib.ref_op(op, level, slot)
        if rc != 0:
            raise RuntimeError(f"ref_op({name}, {level}) -> {rc}")

    def history(self):
        n = self.lib.ref_history(None, 0)
        e = np.empty(max(n, 1))
        self.lib.ref_history(e.ctypes.data_as(_dp), n)
        return e[:n]

    def time_cycles(self, n):
        t = self.lib.ref_time_cycles(self.icyc, n)
        self.icyc += n
        return t
