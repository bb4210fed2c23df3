"""Pin the CPU oracle against fixtures produced by the reference itself
(tests/golden/make_golden.py: the unmodified Version-6-26-04.c compiled with gcc).
Bit-exact: every array after init and after 3 V-cycles, and the mass-error history."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, assert_bitexact

INIT_FIELDS = ["u", "v", "p", "sc", "spu", "spv", "spsc", "areax", "areay", "apu", "apv"]
CYCLE_FIELDS = ["u", "v", "p", "pp", "sc", "resu", "resv", "ressc", "apu", "apv"]
NAMES = ["c0_jacobi", "obs_gs_touch", "obs_below_coarsest", "ports", "bc_mix", "odd_sweeps", "rect_grid"]


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_fixtures(name, oracle_built):
    from cases import small_cases
    from oracle import OracleCase
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    o = OracleCase(small_cases()[name])
    for ig in range(o.ngrid):
        assert_bitexact(o.tag(ig), g[f"init_tag_{ig}"], f"tag {ig}")
        assert_bitexact(o.obstacle_ranges(ig), g[f"ranges_{ig}"], f"ranges {ig}")
        for f in INIT_FIELDS:
            assert_bitexact(o.get(ig, f), g[f"init_{f}_{ig}"], f"init {f} {ig}")
    o.cycle(3)
    for ig in range(o.ngrid):
        for f in CYCLE_FIELDS:
            assert_bitexact(o.get(ig, f), g[f"cyc_{f}_{ig}"], f"3 cycles {f} {ig}")
    e, _ = o.history()
    assert_bitexact(e, g["err"], "mass-error history")


def test_oracle_fixed_point_fixture(oracle_built):
    """2000 Gauss-Seidel V-cycles of the 64x64 channel: the V-cycle fixed point."""
    from mgfvm import configs
    from oracle import OracleCase
    g = np.load(os.path.join(GOLDEN, "c0gs_fixed.npz"))
    o = OracleCase(configs.c0(2))
    o.cycle(2000)
    for f in ("u", "v", "p", "sc"):
        assert_bitexact(o.get(0, f), g[f], f)
    e, d = o.history()
    assert_bitexact(e, g["err"], "history")
    assert d[-1] < 1e-12          # at its fixed point


def test_oracle_planted_mistake_is_caught(oracle_built):
    """The fixture comparison fails when the oracle state is perturbed by one ulp."""
    from cases import small_cases
    from oracle import OracleCase
    g = np.load(os.path.join(GOLDEN, "obs_gs_touch.npz"))
    o = OracleCase(small_cases()["obs_gs_touch"])
    o.cycle(3)
    u = o.get(0, "u")
    u[5, 5] = np.nextafter(u[5, 5], np.inf)
    with pytest.raises(AssertionError):
        assert_bitexact(u, g["cyc_u_0"], "planted")
