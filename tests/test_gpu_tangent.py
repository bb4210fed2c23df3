"""Forward-mode derivatives of the V-cycle (tangent contexts, mgfvm_gradient and the
torch.autograd wrapper) against the CPU oracle.

The value half of a tangent run applies the same FP64 operations as a plain run, so
its state must be bit-identical to the oracle's.  The derivative half is checked
against central differences of the oracle's own V-cycles (h = 1e-6 relative, the
same number of cycles): the north-star bar is 1e-4 relative on dJ; the derivatives
are exact up to the difference quotient's own error, so the tests also hold every
field's derivative to 1e-5 of its largest magnitude.
"""
import dataclasses

import numpy as np
import pytest

from cases import small_cases
from conftest import assert_bitexact

pytestmark = pytest.mark.gpu

DJ_RTOL = 1e-4      # dJ vs the oracle's central difference
FIELD_RTOL = 1e-5   # field derivatives vs the oracle's central difference, relative to their max
H = 1e-6
STATE = ["u", "v", "p", "pp", "sc", "resu", "resv", "ressc", "apu", "apv", "cx", "cy"]


def j_of(p, sc):
    """The objective of mgfvm_objective from level-0 arrays (npy, npx)."""
    rows = slice(1, p.shape[0] - 1)
    ny = p.shape[0] - 2
    return (p[rows, 1].sum() / ny - p[rows, -2].sum() / ny) + sc[rows, -1].sum() / ny


def oracle_state(cfg, prof, cycles):
    from oracle import OracleCase
    o = OracleCase(cfg, prof)
    o.cycle(cycles)
    out = {f: o.get(0, f) for f in ["u", "v", "p", "sc"]}
    o.close()
    return out


def oracle_fd(cfg, prof, cycles, kind, index=0):
    """Central difference of the oracle's level-0 u, v, p, sc and J along a direction."""
    if kind == "inlet":
        base = np.ones(cfg.nfy) if prof is None else np.asarray(prof, dtype=np.float64)
        h = H * max(1.0, abs(base[index]))
        pp_, pm_ = base.copy(), base.copy()
        pp_[index] += h
        pm_[index] -= h
        sp, sm = oracle_state(cfg, pp_, cycles), oracle_state(cfg, pm_, cycles)
    else:
        v0 = getattr(cfg, kind)
        h = H * abs(v0)
        sp = oracle_state(dataclasses.replace(cfg, **{kind: v0 + h}), prof, cycles)
        sm = oracle_state(dataclasses.replace(cfg, **{kind: v0 - h}), prof, cycles)
    d = {f: (sp[f] - sm[f]) / (2 * h) for f in sp}
    dj = (j_of(sp["p"], sp["sc"]) - j_of(sm["p"], sm["sc"])) / (2 * h)
    return d, dj


CASES = {
    "channel_gs": lambda: small_cases()["c0_gs"].replace(nfx=32, nfy=32),
    "obs_jacobi": lambda: small_cases()["obs_jacobi"],
    "obs_gs_touch": lambda: small_cases()["obs_gs_touch"],
    "odd_sweeps": lambda: small_cases()["odd_sweeps"],
    "ports": lambda: small_cases()["ports"],
    "bc_mix": lambda: small_cases()["bc_mix"],
    "obs_below_coarsest": lambda: small_cases()["obs_below_coarsest"],
}
# a derivative the iteration does not see (an inlet face overwritten by a periodic copy,
# or blocked): both sides are zero to rounding
DJ_ATOL = 1e-12
DIRECTIONS = [("inlet", 0), ("inlet", 9), ("inlet", 31), ("amuf", 0), ("prsc", 0)]


def _profile(cfg, seed=3):
    rng = np.random.default_rng(seed)
    return 1.0 + 0.1 * rng.standard_normal(cfg.nfy)


def _tangent_solver(cfg, prof, dirs):
    from mgfvm import Solver
    s = Solver([cfg] * len(dirs), tangent=True)
    for c, (kind, idx) in enumerate(dirs):
        s.set_inlet_profile(c, prof)
        s.set_direction(c, kind, idx)
    return s


@pytest.mark.parametrize("name", list(CASES))
def test_tangent_values_bitexact(name, oracle_built):
    """The value half of a tangent run is the oracle's state, bit for bit."""
    from oracle import OracleCase
    cfg = CASES[name]()
    prof = _profile(cfg)
    s = _tangent_solver(cfg, prof, [("amuf", 0), ("inlet", 4)])
    o = OracleCase(cfg, prof)
    for n in (1, 3):
        s.cycle(n)
        o.cycle(n)
        for c in range(2):
            for ig in range(o.ngrid):
                for f in STATE:
                    assert_bitexact(s.field(c, ig, f), o.get(ig, f), f"case {c} after +{n} level {ig} {f}")
    es, _ = s.history(0)
    eo, _ = o.history()
    np.testing.assert_allclose(es, eo, rtol=1e-12, atol=0)
    s.close()


@pytest.mark.parametrize("name", list(CASES))
def test_tangent_matches_oracle_differences(name, oracle_built):
    """d(state after n cycles)/d(parameter) and dJ agree with central differences of
    the oracle's n cycles for inlet faces, amuf and prsc."""
    cfg = CASES[name]()
    prof = _profile(cfg)
    cycles = 4
    dirs = [(k, i) for k, i in DIRECTIONS if k != "inlet" or i < cfg.nfy]
    s = _tangent_solver(cfg, prof, dirs)
    s.cycle(cycles)
    worst = 0.0
    for c, (kind, idx) in enumerate(dirs):
        d, dj_fd = oracle_fd(cfg, prof, cycles, kind, idx)
        for f in ["u", "v", "p", "sc"]:
            t = s.tangent(c, 0, f)
            scale = max(np.abs(t).max(), np.abs(d[f]).max())
            if scale <= DJ_ATOL:
                continue
            err = np.abs(t - d[f]).max() / scale
            assert err <= FIELD_RTOL, f"{kind}[{idx}] d{f}: max error {err:.2e} of its max {scale:.3e}"
        j, dj = s.objective(c)
        assert j == pytest.approx(j_of(*(oracle_state(cfg, prof, cycles)[f] for f in ("p", "sc"))), rel=1e-13)
        if abs(dj_fd) <= DJ_ATOL:
            assert abs(dj) <= DJ_ATOL, f"{kind}[{idx}]: dJ {dj:.3e} where the central difference is {dj_fd:.3e}"
            continue
        rel = abs(dj - dj_fd) / abs(dj_fd)
        worst = max(worst, rel)
        assert rel <= DJ_RTOL, f"{kind}[{idx}]: dJ {dj:.12e} vs central difference {dj_fd:.12e} ({rel:.2e})"
    s.close()
    print(f"{name}: worst dJ relative error vs the oracle's central differences {worst:.2e}")


def test_gradient_batch_and_autograd(oracle_built):
    """mgfvm_gradient (every inlet face, amuf, prsc in one batch) equals the one-case
    tangent runs, and the torch.autograd wrapper passes those derivatives back."""
    import torch

    import mgfvm
    from mgfvm.autograd import objective
    cfg = CASES["obs_gs_touch"]()
    prof = _profile(cfg)
    cycles = 3
    j, g_in, g_amuf, g_prsc = mgfvm.gradient(cfg, prof, cycles)
    assert g_in.shape == (cfg.nfy,)
    k = int(np.argmax(np.abs(g_in)))       # the face J depends on most after these cycles
    probe = [("inlet", 0), ("inlet", k), ("amuf", 0), ("prsc", 0)]
    s = _tangent_solver(cfg, prof, probe)
    s.cycle(cycles)
    want = [g_in[0], g_in[k], g_amuf, g_prsc]
    for c in range(len(probe)):
        jc, djc = s.objective(c)
        assert jc == j
        assert djc == want[c]
    s.close()
    _, dj_fd = oracle_fd(cfg, prof, cycles, "inlet", k)
    assert abs(g_in[k] - dj_fd) <= DJ_RTOL * abs(dj_fd)

    x = torch.tensor(prof, dtype=torch.float64, requires_grad=True)
    a = torch.tensor(cfg.amuf, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(cfg.prsc, dtype=torch.float64, requires_grad=True)
    out = objective(x, a, b, cfg, cycles)
    assert out.item() == j
    (2.0 * out).backward()
    np.testing.assert_array_equal(x.grad.numpy(), 2.0 * g_in)
    assert a.grad.item() == 2.0 * g_amuf and b.grad.item() == 2.0 * g_prsc


def test_tangent_context_refuses_state_edits(oracle_built):
    """Calls that would change the state without its derivatives fail in a tangent context."""
    from mgfvm import MgfvmError, Solver
    cfg = CASES["obs_jacobi"]()
    s = Solver(cfg, tangent=True)
    with pytest.raises(MgfvmError):
        s.op("solve_u", 0)
    with pytest.raises(MgfvmError):
        s.set_field(0, 0, "u", np.zeros(s.dims(0, 0)[::-1]))
    with pytest.raises(MgfvmError):
        s.set_direction(0, "inlet", cfg.nfy)
    s.close()
    with pytest.raises(MgfvmError):
        Solver(cfg, tangent=True, precision="mixed")


def test_gradient_in_batches_and_mixed_cases(oracle_built, monkeypatch):
    """The gradient is the same whether its directions run in one batch or in batches of
    five (MGFVM_GRADIENT_BATCH), and a tangent context may hold cases of different sizes
    and obstacles, each differentiated as on its own."""
    import mgfvm
    cfg = CASES["obs_jacobi"]()
    prof = _profile(cfg)
    whole = mgfvm.gradient(cfg, prof, 2)
    monkeypatch.setenv("MGFVM_GRADIENT_BATCH", "5")
    parts = mgfvm.gradient(cfg, prof, 2)
    assert whole[0] == parts[0] and whole[2] == parts[2] and whole[3] == parts[3]
    np.testing.assert_array_equal(whole[1], parts[1])

    from mgfvm import Solver
    other = small_cases()["c0_jacobi"].replace(nfx=64, nfy=32, xl=2.0)
    prof2 = _profile(other, seed=5)
    s = Solver([cfg, other], tangent=True)
    s.set_inlet_profile(0, prof)
    s.set_inlet_profile(1, prof2)
    s.set_direction(0, "amuf")
    s.set_direction(1, "inlet", 7)
    s.cycle(3)
    for c, (cc, pr, kind, idx) in enumerate([(cfg, prof, "amuf", 0), (other, prof2, "inlet", 7)]):
        _, dj_fd = oracle_fd(cc, pr, 3, kind, idx)
        _, dj = s.objective(c)
        assert abs(dj - dj_fd) <= DJ_RTOL * abs(dj_fd), f"case {c}: {dj} vs {dj_fd}"
    s.close()
