"""The raw-pointer entry points (caller-owned device memory) against the oracle:
mgfvm_jacobi_f64 (solver, Version-6-26-04.c:1231-1296), mgfvm_rbgs_f64 (solvergs,
:1297-1351) and mgfvm_masserror_f64 (masserror, :1096-1125).  Device buffers come
from torch; the calls go through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from conftest import assert_bitexact

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _p(t):
    return C.c_void_p(t.data_ptr())


def _equation_state(cfg, op, cycles=2):
    """Coefficients, right-hand side and the field before/after one oracle solve_* call."""
    from oracle import OracleCase
    o = OracleCase(cfg)
    o.cycle(cycles)
    o.op("fluxes", 0)
    if op == "solve_v":
        o.op("solve_u", 0)
    fld = {"solve_u": "u", "solve_v": "v"}[op]
    before = o.get(0, fld).copy()
    o.op(op, 0)
    coefs = {k: o.get(0, k) for k in ("aw", "ae", "as", "an", "ap", "su")}
    return o, fld, before, coefs, o.get(0, fld)


@pytest.mark.parametrize("isolve,op", [(1, "solve_u"), (1, "solve_v"), (2, "solve_u"), (2, "solve_v")])
def test_raw_smoothers_match_oracle(isolve, op, oracle_built):
    import torch
    from mgfvm import configs, lib
    from mgfvm._lib import check
    cfg = configs.small(32, 3, isolve=isolve, nswpm=3, ig_obs=3, obstacles=[(2, 3, 3, 3), (6, 6, 5, 6)])
    o, fld, before, coefs, after = _equation_state(cfg, op)
    npx, npy = o.dims(0)
    nx, ny = (npx - 2, npy - 1) if op == "solve_u" else (npx - 1, npy - 2)
    d = {k: _dev(v) for k, v in coefs.items()}
    phi = _dev(before)
    if isolve == 1:
        scratch = torch.zeros_like(phi)
        check(lib().mgfvm_jacobi_f64(_p(d["aw"]), _p(d["ae"]), _p(d["as"]), _p(d["an"]), _p(d["ap"]),
                                     _p(d["su"]), _p(phi), _p(scratch), npx, npy, nx, ny, cfg.nswpm, None))
    else:
        check(lib().mgfvm_rbgs_f64(_p(d["aw"]), _p(d["ae"]), _p(d["as"]), _p(d["an"]), _p(d["ap"]),
                                   _p(d["su"]), _p(phi), npx, npy, nx, ny, cfg.nswpm, None))
    torch.cuda.synchronize()
    assert_bitexact(phi.cpu().numpy(), after, f"{fld} after {cfg.nswpm} sweeps")


def test_raw_masserror_matches_oracle(oracle_built):
    import torch
    from mgfvm import configs, lib
    from mgfvm._lib import check
    from oracle import OracleCase
    cfg = configs.small(48, 3, isolve=2, ig_obs=3, obstacles=[(2, 3, 3, 3)])
    o = OracleCase(cfg)
    o.cycle(3)
    u, v, ax, ay = (o.get(0, k) for k in ("u", "v", "areax", "areay"))
    o.op("solve_pp", 0)
    npx, npy = o.dims(0)
    tu, tv, tax, tay = (_dev(a) for a in (u, v, ax, ay))
    su = torch.zeros_like(tu)
    pp = torch.full_like(tu, 7.0)
    err = torch.zeros(1, dtype=torch.float64, device="cuda")
    n = lib().mgfvm_masserror_scratch_doubles(npx, npy)
    partials = torch.zeros(n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        check(lib().mgfvm_masserror_f64(_p(tu), _p(tv), _p(tax), _p(tay), _p(su), _p(pp), npx, npy,
                                        _p(err), _p(partials), None))
        torch.cuda.synchronize()
        np.testing.assert_allclose(err.item(), o.last_err(), rtol=1e-12)
        assert_bitexact(su.cpu().numpy()[1:-1, 1:-1], o.get(0, "su")[1:-1, 1:-1], "su = -div")
        assert np.all(pp.cpu().numpy()[1:-1, 1:-1] == 0.0)


def test_raw_rejects_bad_extent():
    from mgfvm import lib
    from mgfvm._abi import EINVAL
    rc = lib().mgfvm_rbgs_f64(*([C.c_void_p(0)] * 7), 10, 10, 20, 5, 2, None)
    assert rc == EINVAL


def test_division_by_reciprocal_matches_ieee():
    """The smoothers divide by a reciprocal taken once per cell plus two Markstein
    correction steps; the result must carry the bits of the IEEE division on raw bit
    patterns (every exponent, zeros, subnormals, Inf, NaN) and smoother-like values."""
    from mgfvm._lib import lib
    L = lib()
    bad = C.c_longlong(-1)
    for seed in (1, 2, 3):
        assert L.mgfvm_check_division(0, 1 << 27, seed, C.byref(bad)) == 0
        assert bad.value == 0


def test_field_views_share_engine_memory(oracle_built):
    """mgfvm_field_device_ptr / Solver.field_view: a torch tensor over the engine's own
    array, no copy: it reads what the engine computed, and what is written through it
    is what the next cycles start from."""
    import torch
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cfg = configs.small(32, 3, isolve=2)
    s = Solver(cfg)
    s.cycle(2)
    u = s.field_view(0, 0, "u")
    assert u.shape == (34, 34) and u.dtype == torch.float64 and u.is_cuda
    np.testing.assert_array_equal(u.cpu().numpy(), s.field(0, 0, "u"))
    o = OracleCase(cfg)
    o.cycle(2)
    sc = o.get(0, "sc") * 0.5
    o.set(0, "sc", sc)
    stream = torch.cuda.ExternalStream(s.stream)
    with torch.cuda.stream(stream):
        s.field_view(0, 0, "sc").copy_(torch.from_numpy(sc).cuda())
    stream.synchronize()
    s.cycle(2)
    o.cycle(2)
    for f in ("u", "v", "p", "sc"):
        assert_bitexact(s.field(0, 0, f), o.get(0, f), f"after writing sc through the view: {f}")
    s.close()
