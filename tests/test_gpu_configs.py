"""Parity at the sizes and shapes of the benchmark configurations (seeded synthetic
inputs): the engine against the CPU oracle, bit for bit, after a few V-cycles.

  obstacle flow   256 x 256, ngrid 5, staggered lattice, Re 10 and 100
  mixed batch     cases of 64, 128 and 256 cells (ngrid 4/5/6, coarsest 8 x 8),
                  random particles, Re in {10, 50, 100, 200}, in one context
  large grid      1024 x 1024, ngrid 7, quarter-pixel staggered lattice (ig_obs 4)
  inlet profiles  256 x 256 random-particle cases with per-face inlet u
"""
import numpy as np
import pytest

from conftest import assert_bitexact

pytestmark = pytest.mark.gpu

FIELDS = ["u", "v", "p", "pp", "sc", "resu", "resv", "ressc", "apu", "apv"]


def _check(s, k, o, cycles, what, levels=(0, 1)):
    for ig in levels:
        for f in FIELDS:
            assert_bitexact(s.field(k, ig, f), o.get(ig, f), f"{what} after {cycles} cycles, level {ig} {f}")
    np.testing.assert_allclose(s.history(k)[0], o.history()[0], rtol=1e-12, atol=0)


@pytest.mark.parametrize("band,coarse", [(2, 2), (1, 0)])
def test_obstacle_flow_pair(band, coarse, oracle_built):
    """Levels 1 and 2 (130^2 and 66^2 padded) by band visits (a cluster of 8 and of 2
    CTAs per case; band 2) and by the tile smoothers (band 1, the default for two cases);
    levels 3 and 4 with the transfers into and out of them in one cluster launch
    (coarse 2) and by their separate launches (coarse 0, the default)."""
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cases = configs.c1_pair(seed=1)
    s = Solver(cases)
    s.set_tuning(band_visit=[band] * 5, coarse_cluster=coarse)
    # the first cycle launched kernel by kernel (profile_cycle), two more from the graph
    kinds = {k for k, _, _ in s.profile_cycle()}
    assert ("band_visit" in kinds) == (band == 2)
    assert ("coarse_cycle" in kinds) == (coarse == 2)
    s.cycle(2)
    for k, cfg in enumerate(cases):
        o = OracleCase(cfg)
        o.cycle(3)
        _check(s, k, o, 3, f"obstacle flow case {k}", levels=range(cfg.ngrid))


def test_obstacle_flow_pair_long_run(oracle_built):
    """The benchmark's solve, shortened to 250 V-cycles: the autotuned schedule and the
    chunked solve with the reference's stop rule, then every level-0 field against the
    oracle's 250 cycles, bit for bit (the converged-field error of the benchmark is 0)."""
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cases = configs.c1_pair(seed=1)
    n = 250
    with Solver(cases, sync_every=64) as s:
        s.autotune(2)
        ran = s.solve(n, 0.0)
        assert list(ran) == [n, n]
        for k, cfg in enumerate(cases):
            o = OracleCase(cfg)
            o.cycle(n)
            for f in ("u", "v", "p", "pp", "sc"):
                assert_bitexact(s.field(k, 0, f), o.get(0, f), f"obstacle flow case {k} after {n} cycles, {f}")
            np.testing.assert_allclose(s.history(k)[0], o.history()[0], rtol=1e-12, atol=0)
            o.close()


@pytest.mark.parametrize("band", [0, 2])
def test_mixed_size_batch(band, oracle_built):
    """Cases of three sizes share every launch.  With band 2, band visits run levels 0-2
    where they fit, shaped for the largest case, so smaller cases leave bands empty
    (the default takes none for this batch: too few cases, and of several sizes)."""
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cases = configs.c2(9, seed=2)
    assert {c.nfx for c in cases} == {64, 128, 256}
    s = Solver(cases)
    s.set_tuning(band_visit=[band] * 6)
    s.cycle(2)
    for k, cfg in enumerate(cases):
        o = OracleCase(cfg)
        o.cycle(2)
        _check(s, k, o, 2, f"batch case {k} ({cfg.nfx}^2)", levels=range(cfg.ngrid))


def test_large_grid(oracle_built):
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cfg = configs.c3(seed=3)
    assert cfg.nfx == 1024 and cfg.ngrid == 7
    s = Solver(cfg)
    o = OracleCase(cfg)
    s.cycle(2)
    o.cycle(2)
    _check(s, 0, o, 2, "1024^2", levels=(0, 1, 6))


def test_inlet_profiles(oracle_built):
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cases, profiles = configs.c4(3, seed=4)
    s = Solver(cases)
    for k, pr in enumerate(profiles):
        s.set_inlet_profile(k, pr)
    s.cycle(3)
    for k, (cfg, pr) in enumerate(zip(cases, profiles)):
        o = OracleCase(cfg, pr)
        o.cycle(3)
        _check(s, k, o, 3, f"profile case {k}")


def test_divergence_as_the_reference(oracle_built):
    """A random-particle case on which the reference's iteration blows up (case 34 of
    the adjoint configuration, seed 4: max |u| ~1e7 after cycle 2, NaN in cycle 3 in the
    reference build): the engine follows it bit for bit while the values are finite,
    goes non-finite in the same cycle, stops that case there in a solve, and keeps
    solving the other cases of the batch."""
    from mgfvm import MgfvmError, Solver, configs
    from oracle import OracleCase
    cases, profs = configs.c4(64, seed=4)
    pick = [33, 34]
    o = OracleCase(cases[34], profs[34])
    s = Solver([cases[k] for k in pick])
    for c, k in enumerate(pick):
        s.set_inlet_profile(c, profs[k])
    s.cycle(2)
    o.cycle(2)
    _check(s, 1, o, 2, "diverging case", levels=range(cases[34].ngrid))
    assert np.abs(s.field(1, 0, "u")).max() > 1e6
    s.cycle(1)
    o.cycle(1)
    assert not np.isfinite(s.history(1)[0][-1]) and not np.isfinite(o.history()[0][-1])
    s.reset()
    with pytest.raises(MgfvmError):
        s.solve(10)
    s.reset()
    ran = s.solve(10, allow_nonfinite=True)
    assert list(ran) == [10, 3] and s.diverged() == [1]
    s.close()
