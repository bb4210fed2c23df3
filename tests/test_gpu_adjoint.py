"""Reverse-mode derivatives (mgfvm_adjoint) against the forward mode and the oracle.

The adjoint applies the transpose of the Jacobian the tangent kernel applies, phase
by phase, over the same cycles; the two gradients of J are therefore the same
numbers up to rounding (the tangent sums the chain rule forwards, the adjoint
backwards, with atomics), held here to 1e-10 of the gradient's largest entry.
Against the oracle's central differences (h = 1e-6) the bar is the north star's
1e-4 relative.
"""
import numpy as np
import pytest

from cases import small_cases
from conftest import assert_bitexact

pytestmark = pytest.mark.gpu

ADJ_RTOL = 1e-10


def _forward_mode(cfg, prof, cycles):
    from mgfvm import gradient
    return gradient(cfg, prof, cycles)


def _adjoint(cases, profiles, cycles):
    from mgfvm import Solver
    with Solver(cases) as s:
        for k, pr in enumerate(profiles):
            if pr is not None:
                s.set_inlet_profile(k, pr)
        s.adjoint(cycles)
        return [s.adjoint_gradient(k) for k in range(len(cases))]


def _close(adj, fwd, what):
    ja, ga, aa, pa = adj
    jf, gf, af, pf = fwd
    assert ja == jf, f"{what}: J {ja!r} vs {jf!r}"
    full_a = np.concatenate([ga, [aa, pa]])
    full_f = np.concatenate([gf, [af, pf]])
    scale = max(np.abs(full_f).max(), 1e-300)
    err = np.abs(full_a - full_f).max() / scale
    assert err <= ADJ_RTOL, f"{what}: adjoint vs forward mode {err:.3e} (largest |dJ| {scale:.3e})"


@pytest.mark.parametrize("name", [k for k in small_cases() if k != "bc_mix"])
def test_adjoint_equals_forward_mode(name, oracle_built):
    cfg = small_cases()[name]
    rng = np.random.default_rng(11)
    prof = 1.0 + 0.1 * rng.standard_normal(cfg.nfy)
    for cycles in (1, 4):
        adj = _adjoint([cfg], [prof], cycles)[0]
        _close(adj, _forward_mode(cfg, prof, cycles), f"{name}, {cycles} cycles")


def test_adjoint_batch_of_different_cases(oracle_built):
    """One context, cases of different sizes, depths, smoothers' obstacle sets and inlet
    profiles: every case's gradient is its own."""
    sc = small_cases()
    cases = [sc["obs_gs_touch"], sc["obs_below_coarsest"], sc["rect_grid"], sc["obs_gs_touch"]]
    rng = np.random.default_rng(5)
    profs = [1.0 + 0.1 * rng.standard_normal(c.nfy) for c in cases]
    profs[3] = None
    adj = _adjoint(cases, profs, 3)
    for k, (cfg, pr) in enumerate(zip(cases, profs)):
        _close(adj[k], _forward_mode(cfg, pr, 3), f"batch case {k}")


def test_adjoint_leaves_the_state_after_the_cycles(oracle_built):
    from mgfvm import Solver
    from oracle import OracleCase
    cfg = small_cases()["obs_gs_touch"]
    with Solver(cfg) as s:
        s.cycle(2)                       # the adjoint starts from the initial state regardless
        s.adjoint(5)
        o = OracleCase(cfg)
        o.cycle(5)
        for ig in range(cfg.ngrid):
            for f in ("u", "v", "p", "sc"):
                assert_bitexact(s.field(0, ig, f), o.get(ig, f), f"after the adjoint, level {ig} {f}")
        np.testing.assert_allclose(s.history(0)[0], o.history()[0], rtol=1e-12, atol=0)
        s.cycle(2)                       # and the context carries on from there
        o.cycle(2)
        assert_bitexact(s.field(0, 0, "u"), o.get(0, "u"), "2 cycles after the adjoint")


def test_adjoint_against_central_differences(oracle_built):
    """A 64 x 64 random-particle case with an inlet profile, 6 cycles: dJ/d(inlet face),
    dJ/damuf and dJ/dprsc against the oracle's central differences."""
    from mgfvm import configs
    from test_gpu_tangent import oracle_fd
    cases, profs = configs.c4(1, seed=9, n=64)
    cfg, prof = cases[0], profs[0]
    cycles = 6
    j, g_in, g_a, g_p = _adjoint([cfg], [prof], cycles)[0]
    k = int(np.argmax(np.abs(g_in)))
    for kind, idx, got in (("inlet", k, g_in[k]), ("amuf", 0, g_a), ("prsc", 0, g_p)):
        _, fd = oracle_fd(cfg, prof, cycles, kind, idx)
        assert abs(got - fd) <= 1e-4 * abs(fd), f"dJ/d{kind}[{idx}] {got:.12e} vs central difference {fd:.12e}"


def test_adjoint_refuses_periodic_boundaries():
    from mgfvm import MgfvmError, Solver
    from mgfvm._abi import EUNSUPPORTED
    with Solver(small_cases()["bc_mix"]) as s:
        with pytest.raises(MgfvmError) as ei:
            s.adjoint(2)
        assert ei.value.status == EUNSUPPORTED


def test_objective_batch_through_autograd(oracle_built):
    """objective_batch: J of every case, and backward() hands each case's adjoint
    gradient scaled by the incoming gradient."""
    import torch

    from mgfvm import configs
    from mgfvm.autograd import objective_batch
    cases, profs = configs.c4(3, seed=21, n=32)
    cases = [c.replace(nvcycle=10) for c in cases]
    cycles = 3
    x = torch.tensor(np.stack(profs), dtype=torch.float64, requires_grad=True)
    a = torch.tensor([c.amuf for c in cases], dtype=torch.float64, requires_grad=True)
    b = torch.tensor([c.prsc for c in cases], dtype=torch.float64, requires_grad=True)
    out = objective_batch(x, a, b, cases, cycles)
    w = torch.tensor([1.0, -2.0, 0.5], dtype=torch.float64)
    (w * out).sum().backward()
    for k, (cfg, pr) in enumerate(zip(cases, profs)):
        jf, gf, af, pf = _forward_mode(cfg, pr, cycles)
        assert out[k].item() == jf
        scale = max(np.abs(gf).max(), abs(af), abs(pf))
        assert np.abs(x.grad[k].numpy() - w[k].item() * gf).max() <= ADJ_RTOL * abs(w[k].item()) * scale
        assert abs(a.grad[k].item() - w[k].item() * af) <= ADJ_RTOL * abs(w[k].item()) * scale
        assert abs(b.grad[k].item() - w[k].item() * pf) <= ADJ_RTOL * abs(w[k].item()) * scale


@pytest.mark.parametrize("cluster", ["1", "2", "8"])
def test_adjoint_cluster_sizes(cluster, monkeypatch, oracle_built):
    """The CTAs a case's adjoint cycle runs on (a cluster of 1, 2 or 8) only change the
    order in which contributions land."""
    monkeypatch.setenv("MGFVM_ADJOINT_CLUSTER", cluster)
    cfg = small_cases()["obs_gs_touch"]
    prof = 1.0 + 0.05 * np.sin(np.arange(cfg.nfy))
    _close(_adjoint([cfg], [prof], 3)[0], _forward_mode(cfg, prof, 3), f"cluster {cluster}")


def test_adjoint_with_a_diverging_case_in_the_batch(oracle_built):
    """A case whose iteration turns non-finite (the reference's does on the same input)
    gets no gradient; the other cases of its batch are unaffected."""
    from mgfvm import MgfvmError, Solver, configs
    from mgfvm._abi import ENONFINITE
    cases, profs = configs.c4(26, seed=4)
    pair = [cases[0], cases[25]]
    cycles = 10
    with Solver(pair) as s:
        s.set_inlet_profile(0, profs[0])
        s.set_inlet_profile(1, profs[25])
        s.adjoint(cycles)
        with pytest.raises(MgfvmError) as ei:
            s.adjoint_gradient(1)
        assert ei.value.status == ENONFINITE
        assert np.isnan(s.adjoint_gradient(1, allow_nonfinite=True)[2])
        good = s.adjoint_gradient(0)
    _close(good, _forward_mode(cases[0], profs[0], cycles), "the finite case beside a diverging one")


@pytest.mark.parametrize("name", ["obs_gs_touch", "obs_below_coarsest", "ports", "odd_sweeps", "rect_grid"])
def test_closed_form_transposes_equal_the_probed_ones(name, monkeypatch, oracle_built):
    """The phases transposed in closed form (the red-black half-sweep; the assemblies,
    fine residuals and FAS defects with their hybrid-scheme coefficients) give what
    transposing them by dual-number probes gives, to rounding."""
    cfg = small_cases()[name]
    prof = 1.0 + 0.05 * np.cos(np.arange(cfg.nfy))
    closed = _adjoint([cfg], [prof], 3)[0]
    monkeypatch.setenv("MGFVM_ADJOINT_GENERIC", "1")
    probed = _adjoint([cfg], [prof], 3)[0]
    a = np.concatenate([closed[1], closed[2:]])
    b = np.concatenate([probed[1], probed[2:]])
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
