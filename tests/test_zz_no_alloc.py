"""mgfvm_masserror_f64_noalloc: the mass residual for callers that cannot allocate
device memory (their device memory belongs to another runtime, or they must stay out
of the CUDA allocator).  Its reduction scratch is a fixed static device array inside
the library, so it must give what mgfvm_masserror_f64 gives with a caller-allocated
buffer, call after call, and refuse levels larger than that array serves.

This file is collected last so a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _level(n, seed):
    """Level-0 u, v and face areas of an n x n case after a few oracle V-cycles."""
    from mgfvm import configs
    from oracle import OracleCase
    o = OracleCase(configs.small(n, 3, isolve=2, ig_obs=3, obstacles=[(2, 3, 3, 3)], relxp=0.3 + 0.1 * seed))
    o.cycle(2 + seed)
    return o.dims(0), [o.get(0, f) for f in ("u", "v", "areax", "areay")]


def _call(fn, dims, fields, with_partials):
    import torch
    npx, npy = dims
    u, v, ax, ay = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in fields)
    su = torch.zeros_like(u)
    pp = torch.full_like(u, 3.0)
    err = torch.zeros(1, dtype=torch.float64, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    if with_partials:
        from mgfvm import lib
        part = torch.zeros(lib().mgfvm_masserror_scratch_doubles(npx, npy), dtype=torch.float64, device="cuda")
        rc = fn(p(u), p(v), p(ax), p(ay), p(su), p(pp), npx, npy, p(err), p(part), None)
    else:
        rc = fn(p(u), p(v), p(ax), p(ay), p(su), p(pp), npx, npy, p(err), None)
    torch.cuda.synchronize()
    return rc, err.item(), su.cpu().numpy(), pp.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice(oracle_built):
    from mgfvm import lib
    from mgfvm._abi import OK
    L = lib()
    fn = L.mgfvm_masserror_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    # a large level, then a smaller one: the second call reuses scratch the first left behind
    for n, seed in ((96, 0), (48, 1)):
        dims, fields = _level(n, seed)
        rc0, e0, su0, pp0 = _call(L.mgfvm_masserror_f64, dims, fields, True)
        rc1, e1, su1, pp1 = _call(fn, dims, fields, False)
        assert rc0 == OK and rc1 == OK
        np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(su1, su0)
        np.testing.assert_array_equal(pp1, pp0)


def test_noalloc_rejects_levels_beyond_its_scratch():
    import torch
    from mgfvm import lib
    from mgfvm._abi import EINVAL
    L = lib()
    fn = L.mgfvm_masserror_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = fn(p, p, p, p, p, p, 1030, 1030, p, None)       # 1028^2 interior cells > 2^20
    assert rc == EINVAL
    assert b"exceed" in L.mgfvm_last_error()
