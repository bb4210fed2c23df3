"""mgfvm_masserror_f64_noalloc: the mass residual for callers that cannot allocate
device memory (their device memory belongs to another runtime, or they must stay out
of the CUDA allocator).  Its reduction scratch is a fixed static device array inside
the library, so it must give what mgfvm_masserror_f64 gives with a caller-allocated
buffer, and what the oracle's masserror gives, call after call; it must take no
device memory; and it must refuse levels larger than that array serves while serving
the largest level it admits.

This file is collected last so a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NOALLOC_MAX_SIDE = 1026     # (npx-2)*(npy-2) = 1024^2 = 2^20 interior cells, the largest admitted


def _noalloc_fn():
    from mgfvm import lib
    fn = lib().mgfvm_masserror_f64_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p] * 6 + [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return fn


def _level(n, seed):
    """Level-0 u, v and face areas of an n x n case after a few oracle V-cycles, and the
    oracle's own masserror of that state (its sum |div| and su = -div)."""
    from mgfvm import configs
    from oracle import OracleCase
    o = OracleCase(configs.small(n, 3, isolve=2, ig_obs=3, obstacles=[(2, 3, 3, 3)], relxp=0.3 + 0.1 * seed))
    o.cycle(2 + seed)
    dims = o.dims(0)
    fields = [o.get(0, f) for f in ("u", "v", "areax", "areay")]
    # solve_pp starts with masserror (:1096-1125); no p' Dirichlet rows here, so coefp
    # leaves su = -div as masserror wrote it
    o.op("solve_pp", 0)
    ref = (o.last_err(), o.get(0, "su"))
    o.close()
    return dims, fields, ref


class _Buffers:
    """Device inputs and outputs of one call, allocated up front so the calls
    themselves can be checked for taking device memory."""

    def __init__(self, dims, fields):
        import torch
        from mgfvm import lib
        self.dims = dims
        npx, npy = dims
        self.u, self.v, self.ax, self.ay = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in fields)
        self.su = torch.zeros_like(self.u)
        self.pp = torch.full_like(self.u, 3.0)
        self.err = torch.zeros(1, dtype=torch.float64, device="cuda")
        self.part = torch.zeros(lib().mgfvm_masserror_scratch_doubles(npx, npy), dtype=torch.float64,
                                device="cuda")
        torch.cuda.synchronize()

    def call(self, noalloc):
        import torch
        from mgfvm import lib
        p = lambda t: C.c_void_p(t.data_ptr())
        npx, npy = self.dims
        self.su.zero_()
        self.pp.fill_(3.0)
        self.err.zero_()
        torch.cuda.synchronize()
        if noalloc:
            rc = _noalloc_fn()(p(self.u), p(self.v), p(self.ax), p(self.ay), p(self.su), p(self.pp), npx, npy,
                               p(self.err), None)
        else:
            rc = lib().mgfvm_masserror_f64(p(self.u), p(self.v), p(self.ax), p(self.ay), p(self.su), p(self.pp),
                                           npx, npy, p(self.err), p(self.part), None)
        torch.cuda.synchronize()
        return rc, self.err.item(), self.su.cpu().numpy(), self.pp.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_and_oracle_twice(oracle_built):
    from mgfvm._abi import OK
    # a large level, then a smaller one: the second call reuses scratch the first left behind
    for n, seed in ((96, 0), (48, 1)):
        dims, fields, (err_ref, su_ref) = _level(n, seed)
        b = _Buffers(dims, fields)
        rc0, e0, su0, pp0 = b.call(noalloc=False)
        rc1, e1, su1, pp1 = b.call(noalloc=True)
        assert rc0 == OK and rc1 == OK
        np.testing.assert_allclose(e1, e0, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(su1, su0)
        np.testing.assert_array_equal(pp1, pp0)
        # against the oracle: su bit for bit on the interior, the sum (a different
        # but fixed summation order) to 1e-12 relative, pp = 0 on the interior
        np.testing.assert_array_equal(su1[1:-1, 1:-1], su_ref[1:-1, 1:-1])
        np.testing.assert_allclose(e1, err_ref, rtol=1e-12, atol=0)
        assert not pp1[1:-1, 1:-1].any()


def test_noalloc_takes_no_device_memory(oracle_built):
    import torch
    from mgfvm._abi import OK
    dims, fields, _ = _level(64, 0)
    b = _Buffers(dims, fields)
    assert b.call(noalloc=True)[0] == OK      # first call on the device: module load, symbol lookup
    free0, _ = torch.cuda.mem_get_info()
    used0 = torch.cuda.memory_allocated()
    for _ in range(3):
        assert b.call(noalloc=True)[0] == OK
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed by {free0 - free1} bytes across the calls"
    assert torch.cuda.memory_allocated() == used0


def test_noalloc_largest_admitted_level_then_smaller():
    """1024 x 1024 interior cells put the last block's partial sums and the completion
    counter at the very end of the static array."""
    from mgfvm._abi import OK
    rng = np.random.default_rng(7)
    npx = npy = NOALLOC_MAX_SIDE
    fields = [rng.standard_normal((npy, npx)), rng.standard_normal((npy, npx)),
              rng.uniform(0.5, 1.5, (npy, npx)), rng.uniform(0.5, 1.5, (npy, npx))]
    big = _Buffers((npx, npy), fields)
    rc0, e0, su0, pp0 = big.call(noalloc=False)
    rc1, e1, su1, pp1 = big.call(noalloc=True)
    assert rc0 == OK and rc1 == OK
    assert e1 == e0                       # same kernel, same block count, same summation order
    np.testing.assert_array_equal(su1, su0)
    np.testing.assert_array_equal(pp1, pp0)
    del big
    small = [rng.standard_normal((40, 40)), rng.standard_normal((40, 40)),
             rng.uniform(0.5, 1.5, (40, 40)), rng.uniform(0.5, 1.5, (40, 40))]
    b = _Buffers((40, 40), small)
    rc0, e0, su0, _ = b.call(noalloc=False)
    rc1, e1, su1, _ = b.call(noalloc=True)
    assert rc0 == OK and rc1 == OK
    assert e1 == e0
    np.testing.assert_array_equal(su1, su0)


def test_noalloc_rejects_levels_beyond_its_scratch():
    import torch
    from mgfvm import lib
    from mgfvm._abi import EINVAL
    fn = _noalloc_fn()
    t = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = C.c_void_p(t.data_ptr())
    rc = fn(p, p, p, p, p, p, 1030, 1030, p, None)       # 1028^2 interior cells > 2^20
    assert rc == EINVAL
    assert b"exceed" in lib().mgfvm_last_error()
    rc = fn(p, p, p, p, p, p, NOALLOC_MAX_SIDE + 1, NOALLOC_MAX_SIDE, p, None)   # one row past the limit
    assert rc == EINVAL
