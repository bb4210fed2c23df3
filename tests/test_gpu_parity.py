"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

The FP64 engine is compiled without FMA contraction and applies every reference
operation in the reference's order, so the bar is bit-exact equality of every state
array after every routine and every cycle; only the mass-error sums (parallel,
fixed-order reductions) are compared with a 1e-12 relative tolerance.
"""
import numpy as np
import pytest

from cases import small_cases
from conftest import assert_bitexact, interior, rel_l2

pytestmark = pytest.mark.gpu

STATE = ["u", "v", "p", "pp", "sc", "su", "resu", "resv", "ressc", "apu", "apv", "cx", "cy", "c"]
# the arrays an equation's assembly writes on that equation's domain only; outside it
# they hold stale values that no routine reads (the engine keeps one set per equation,
# the reference one shared set)
COEF = ["aw", "ae", "as", "an", "ap", "su"]
OP_STATE = [f for f in STATE if f != "su"]
ERR_RTOL = 1e-12


def _pair(cfg, **kw):
    from mgfvm import Solver
    from oracle import OracleCase
    return Solver(cfg, **kw), OracleCase(cfg)


def _domain(a, op):
    """The cells a routine writes its coefficients on (solve_u :701, solve_v :710,
    solve_pprime :725, solve_sc :735); elsewhere they are stale and never read."""
    if op == "solve_u":
        return a[1:-1, 1:-2]
    if op == "solve_v":
        return a[1:-2, 1:-1]
    return interior(a)


def _compare(s, o, fields, levels=None, case=0, what="", op=""):
    for ig in range(o.ngrid) if levels is None else levels:
        for f in fields:
            a, b = s.field(case, ig, f), o.get(ig, f)
            if f in COEF:
                a, b = _domain(a, op), _domain(b, op)
            assert_bitexact(a, b, f"{what} level {ig} {f}")


@pytest.mark.parametrize("name", list(small_cases()))
def test_initial_state_bitexact(name, oracle_built):
    cfg = small_cases()[name]
    s, o = _pair(cfg)
    for ig in range(o.ngrid):
        assert_bitexact(s.tag(0, ig), o.tag(ig), f"tag level {ig}")
        for f in ["u", "v", "p", "pp", "sc", "apu", "apv", "spu", "spv", "spsc", "areax", "areay", "su",
                  "resu", "resv", "ressc", "cx", "cy"]:
            assert_bitexact(s.field(0, ig, f), o.get(ig, f), f"init level {ig} {f}")
        assert_bitexact(s.obstacle_ranges(0, ig), o.obstacle_ranges(ig), f"ranges level {ig}")
    s.close()


@pytest.mark.parametrize("name", ["c0_jacobi", "obs_gs_touch", "ports", "bc_mix", "odd_sweeps"])
def test_single_ops_bitexact(name, oracle_built):
    """Every routine of a V-cycle on its own, in cycle order, compared after each."""
    cfg = small_cases()[name]
    s, o = _pair(cfg)
    s.cycle(2)
    o.cycle(2)
    ng = o.ngrid
    seq = []
    for ig in range(ng):
        seq += [("fluxes", ig), ("solve_u", ig), ("solve_v", ig), ("solve_pp", ig), ("pbound", ig),
                ("outflow", ig), ("solve_sc", ig)]
        if ig < ng - 1:
            seq.append(("restrict", ig))
    for ig in range(ng - 2, -1, -1):
        seq.append(("prolong", ig))
    for op, ig in seq:
        s.op(op, ig)
        o.op(op, ig)
        fields = OP_STATE + (COEF if op.startswith("solve") else [])
        lv = [ig, ig + 1] if op in ("restrict", "prolong") else [ig]
        _compare(s, o, fields, lv, what=f"after {op}({ig})", op=op)


@pytest.mark.parametrize("name", list(small_cases()))
@pytest.mark.parametrize("tail", [-1, 0, 99])
def test_cycles_bitexact(name, tail, oracle_built):
    cfg = small_cases()[name]
    s, o = _pair(cfg, tail_level=tail)
    for n in (1, 2, 7):
        s.cycle(n)
        o.cycle(n)
        _compare(s, o, STATE, what=f"tail {tail} after +{n} cycles")
    es, _ = s.history(0)
    eo, _ = o.history()
    assert len(es) == len(eo) == 10
    np.testing.assert_allclose(es, eo, rtol=ERR_RTOL, atol=0)
    s.close()


def test_direct_launch_equals_graph(oracle_built):
    from mgfvm import Solver
    cfg = small_cases()["obs_gs_touch"]
    a, b = Solver(cfg, use_graph=True), Solver(cfg, use_graph=False)
    a.cycle(5)
    b.cycle(5)
    for f in STATE:
        for ig in range(cfg.ngrid):
            assert_bitexact(a.field(0, ig, f), b.field(0, ig, f), f"{f} level {ig}")


def test_heterogeneous_batch(oracle_built):
    """Cases of different sizes, levels, physics and obstacles advance together and each
    matches its own oracle."""
    from mgfvm import Solver
    from oracle import OracleCase
    sc = small_cases()
    names = ["c0_gs", "obs_gs_touch", "obs_below_coarsest", "bc_mix", "rect_grid"]
    cfgs = [sc[n] for n in names]
    s = Solver(cfgs)
    orcs = [OracleCase(c) for c in cfgs]
    s.cycle(4)
    for k, o in enumerate(orcs):
        o.cycle(4)
        _compare(s, o, STATE, case=k, what=names[k])
        np.testing.assert_allclose(s.history(k)[0], o.history()[0], rtol=ERR_RTOL)


def test_reset_and_inlet_profile(oracle_built):
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cfg = configs.small(32, 3, isolve=2)
    prof = 1.0 + 0.1 * np.random.default_rng(7).standard_normal(32)
    s = Solver([cfg, cfg])
    s.cycle(3)
    s.set_inlet_profile(1, prof)      # resets case 1 only
    o0, o1 = OracleCase(cfg), OracleCase(cfg, prof)
    o0.cycle(3)
    _compare(s, o0, STATE, case=0, what="case 0 kept")
    _compare(s, o1, ["u", "v", "p", "sc"], case=1, what="case 1 reset with profile")
    s.cycle(3)
    o0.cycle(3)
    o1.cycle(3)
    _compare(s, o0, STATE, case=0, what="case 0")
    _compare(s, o1, STATE, case=1, what="case 1")
    s.reset()
    o2 = OracleCase(cfg)
    _compare(s, o2, ["u", "v", "p", "sc"], case=0, what="after reset")


def test_solve_stops_like_oracle(oracle_built):
    """Fixed-point stop rule: same cycle count and the same converged fields."""
    from mgfvm import Solver, configs
    from oracle import OracleCase
    cfg = configs.small(32, 3, isolve=2)
    s = Solver(cfg, sync_every=16)
    o = OracleCase(cfg)
    n_gpu = int(s.solve(3000, fp_tol=1e-9)[0])
    n_cpu = o.solve(3000, 1e-9)
    assert abs(n_gpu - n_cpu) <= 1, (n_gpu, n_cpu)
    if n_gpu == n_cpu:
        _compare(s, o, ["u", "v", "p", "sc"], levels=[0], what="converged")
    else:
        for f in ["u", "v", "sc"]:
            assert rel_l2(s.field(0, 0, f), o.get(0, f)) < 1e-6
    _, d = s.history(0)
    _, dd = o.history()
    np.testing.assert_allclose(d[1:n_gpu], dd[1:n_gpu], rtol=1e-6, atol=1e-14)


def test_reference_stop_rule(oracle_built):
    """convergence above the first mass error stops after one cycle (:247-248)."""
    from mgfvm import Solver, configs
    cfg = configs.small(32, 3, convergence=1e9)
    s = Solver(cfg)
    assert int(s.solve(50)[0]) == 1


TUNINGS = [
    {"smooth_units": [1, 3, 2], "smooth_threads": [512, 1024, 512], "asm_slices": [1, 3, 1],
     "restrict_slices": [3, 1, 3]},
    {"smooth_units": [7, 5, 0], "smooth_threads": [1024, 512, 0], "asm_slices": [3, 1, 3],
     "restrict_slices": [1, 3, 1]},
    {"smooth_units": [16, 12, 20], "smooth_threads": [1024, 512, 1024]},
    {"smooth_units": [3, 7, 5], "smooth_threads": [256, 256, 256]},
    {"update_pfix": [1, 1, 1], "odd_chunks": [1, 1, 1], "pp_level": [1, 1, 1], "prol_fused": [1, 1, 1]},
    {"smooth_units": [5, 3, 7], "odd_chunks": [2, 2, 2]},
    {"smooth_tma": [2, 2, 2]},
    {"smooth_tma": [2, 2, 2], "smooth_units": [3, 5, 7], "smooth_threads": [512, 256, 1024]},
    {"smooth_tma": [2, 2, 2], "smooth_units": [7, 1, 4], "smooth_threads": [256, 512, 512], "odd_chunks": [1, 1, 1]},
    {"coarse_kernel": [0, 0, 2]},
    {"coarse_kernel": [0, 2, 2], "smooth_units": [4, 0, 0]},
    {"pdl": 1},
    {"pdl": 1, "smooth_tma": [2, 2, 2], "coarse_kernel": [0, 0, 2]},
    {"band_visit": [2, 2, 2]},
    {"band_visit": [2, 2, 2], "pdl": 1},
    {"band_visit": [2, 2, 2], "update_pfix": [1, 1, 1], "coarse_kernel": [0, 0, 2]},
    {"coarse_cluster": 2},
    {"coarse_cluster": 2, "pdl": 1, "smooth_units": [3, 5, 7]},
    {"coarse_cluster": 2, "update_pfix": [1, 1, 1], "odd_chunks": [1, 1, 1]},
    {"coarse_cluster": 2, "band_visit": [2, 2, 2], "pdl": 1},
]


@pytest.mark.parametrize("name", ["c0_jacobi", "c0_gs", "obs64_gs", "obs64_odd_jacobi"])
@pytest.mark.parametrize("k", range(len(TUNINGS)))
def test_schedule_choices_bitexact(name, k, oracle_built):
    """Every schedule choice (units per smoother launch, smoother CTA size, assembly and
    restriction slices, band visits) gives the oracle's bits.  The 64-cell cases smooth
    level 0 in tiles unless the tuning asks for band visits (a cluster of two CTAs per
    case runs the whole level-0 visit, the mass error included)."""
    from mgfvm import configs
    cfg = dict(small_cases(),
               obs64_gs=configs.small(64, 3, isolve=2, ig_obs=3, sc_obs=0.2,
                                      obstacles=[(2, 3, 2, 2), (5, 6, 4, 6), (1, 1, 7, 8)]),
               obs64_odd_jacobi=configs.small(64, 3, isolve=1, nswpm=3, nswpp=9, ig_obs=3,
                                              obstacles=[(3, 4, 3, 5)]))[name]
    s, o = _pair(cfg)
    s.set_tuning(**{"band_visit": [1, 1, 1], **TUNINGS[k]})
    for n in (1, 3):
        s.cycle(n)
        o.cycle(n)
        _compare(s, o, STATE, what=f"tuning {k} after +{n} cycles")
    s.close()


def test_autotune_keeps_state(oracle_built):
    """The autotuner times candidates on the live batch and restores it: the next cycles
    continue exactly where they would have."""
    cfg = small_cases()["c0_gs"]
    s, o = _pair(cfg)
    s.cycle(2)
    o.cycle(2)
    before, after, chosen = s.autotune(2)
    assert before > 0 and 0 < after <= before
    assert set(chosen) == {"smooth_units", "smooth_threads", "asm_slices", "restrict_slices", "update_pfix", "odd_chunks", "pp_level",
                           "smooth_tma", "coarse_kernel", "prol_fused", "tma_first_wait", "pdl", "band_visit",
                           "coarse_cluster"}
    _compare(s, o, STATE, what="after autotune")
    s.cycle(3)
    o.cycle(3)
    _compare(s, o, STATE, what="after autotune +3 cycles")
    es, _ = s.history(0)
    assert len(es) == 5
    np.testing.assert_allclose(es, o.history()[0], rtol=ERR_RTOL, atol=0)


@pytest.mark.parametrize("kw", [dict(n=32, ngrid=1, isolve=2), dict(n=32, ngrid=1, isolve=1),
                                dict(n=8, ngrid=2, isolve=2), dict(n=16, ngrid=4, isolve=1)])
def test_edge_sizes_bitexact(kw, oracle_built):
    """One level (no multigrid), a tiny grid, and a coarsest level of 2 x 2 cells."""
    from mgfvm import configs
    n, ng, iso = kw["n"], kw["ngrid"], kw["isolve"]
    cfg = configs.small(n, ng, isolve=iso)
    s, o = _pair(cfg)
    for c in (1, 4):
        s.cycle(c)
        o.cycle(c)
        _compare(s, o, STATE, what=f"n={n} ngrid={ng} after +{c} cycles")
    s.close()


def test_zero_cycles_and_mixed_depth_batch(oracle_built):
    """solve(0) runs nothing; a batch whose cases have different level counts, where
    the shallow case stops early under the reference rule, keeps the deep one going."""
    from mgfvm import Solver, configs
    from oracle import OracleCase
    deep = configs.small(32, 3, isolve=2)
    shallow = configs.small(16, 2, isolve=2, convergence=1e30)   # stops after one cycle
    s = Solver([deep, shallow])
    assert list(s.solve(0, 0.0)) == [0, 0]
    ran = s.solve(5, 0.0)
    assert list(ran) == [5, 1]
    od, osh = OracleCase(deep), OracleCase(shallow)
    od.cycle(5)
    osh.cycle(1)
    _compare(s, od, STATE, case=0, what="deep case")
    _compare(s, osh, STATE, case=1, what="shallow case")
    s.close()


def test_tma_wait_timeout_fails_the_call_and_reset_recovers(oracle_built):
    """A TMA-staged smoother CTA whose first wait for its loads gives up (here at once:
    tma_first_wait = -1, a wait with no polls) records the stall, lets its copies land
    in a second wait at the full bound and leaves; the call fails with ETIMEOUT.  After
    mgfvm_reset, with the default wait, the context runs the oracle's cycles again."""
    from mgfvm import MgfvmError, configs
    from mgfvm._abi import ETIMEOUT
    cfg = configs.small(64, 3, isolve=2, ig_obs=3, sc_obs=0.2, obstacles=[(2, 3, 2, 2), (5, 6, 4, 6)])
    s, o = _pair(cfg)
    s.set_tuning(smooth_tma=[2, 2, 2], smooth_units=[3, 3, 3], tma_first_wait=-1)
    with pytest.raises(MgfvmError) as ei:
        s.cycle(1)
    assert ei.value.status == ETIMEOUT
    assert "every case" in str(ei.value)
    s.set_tuning(tma_first_wait=0)
    s.reset()
    s.cycle(2)
    o.cycle(2)
    _compare(s, o, STATE, what="after a timed-out call, reset and 2 cycles")
    s.close()
