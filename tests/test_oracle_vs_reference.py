"""The CPU oracle against the live reference build (oracle/_ref), on seeded random
configurations.  Runs only where the reference was compiled (this is how the oracle
was pinned); the committed fixtures of test_oracle_golden.py cover the rest."""
import numpy as np
import pytest

from conftest import assert_bitexact, interior

oracle = pytest.importorskip("oracle")

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="reference build (oracle/_ref) not present")

FIELDS = ["u", "v", "p", "pp", "sc", "su", "resu", "resv", "ressc", "apu", "apv", "cx", "cy", "rs", "c"]


def random_case(seed):
    from mgfvm import configs
    rng = np.random.default_rng(seed)
    n = int(rng.choice([16, 32]))
    ngrid = int(rng.integers(2, 4))
    ig_obs = int(rng.integers(1, ngrid + 1))
    span = n >> (ig_obs - 1)
    obs = []
    for _ in range(int(rng.integers(0, 6))):
        i0 = int(rng.integers(1, span + 1)); j0 = int(rng.integers(1, span + 1))
        obs.append((i0, min(span, i0 + int(rng.integers(0, 2))), j0, min(span, j0 + int(rng.integers(0, 2)))))
    kw = dict(isolve=int(rng.integers(1, 3)), nswpm=int(rng.integers(1, 4)), nswpp=int(rng.integers(1, 12)),
              relxm=float(rng.uniform(0.5, 0.9)), relxp=float(rng.uniform(0.2, 0.9)),
              amuf=float(rng.choice([0.1, 0.01, 0.005])), prsc=float(rng.choice([1.0, 0.7])),
              ig_obs=ig_obs if obs else 0, obstacles=obs, sc_obs=float(rng.uniform(0, 1)),
              ibc_xp=int(rng.choice([1, 2, 4])), ibc_xm=int(rng.choice([1, 2, 3])),
              ibc_ym=int(rng.choice([1, 3])), ibc_yp=int(rng.choice([1, 2])),
              guess=tuple(float(x) for x in rng.uniform(-0.2, 0.2, 4)))
    return configs.small(n, ngrid, **kw)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_equals_reference_random(seed, oracle_built):
    cfg = random_case(seed)
    o = oracle.OracleCase(cfg)
    r = oracle.RefCase(cfg)
    for n in (1, 3):
        o.cycle(n)
        r.cycle(n)
        for ig in range(cfg.ngrid):
            for f in FIELDS:
                assert_bitexact(o.get(ig, f), r.get(ig, f), f"seed {seed} level {ig} {f}")
            for f in ("aw", "ae", "as", "an", "ap"):
                assert_bitexact(interior(o.get(ig, f)), interior(r.get(ig, f)), f"seed {seed} level {ig} {f}")
    assert_bitexact(o.history()[0], r.history(), "history")


def test_parser_matches_reference_globals(tmp_path):
    """mgfvm_config_read reads the same values readInput() leaves in the reference globals."""
    import ctypes as C
    from mgfvm import read_case
    cfg = random_case(3).replace(inlets=[(1, 2, 0.5, 0.1, 0.3)], outlets=[(2, 3, 0.1, 0.0, 0.2)], ig_inlt=1, ig_outlt=1)
    cfg.write(str(tmp_path))
    mine = read_case(str(tmp_path))
    oracle.RefCase(cfg, workdir=str(tmp_path))
    L = oracle._ref_lib()
    iv = (C.c_int * 18)(); dv = (C.c_double * 29)()
    obs = (C.c_int * (4 * max(1, len(cfg.obstacles))))()
    pi = (C.c_int * 40)(); pd = (C.c_double * 60)()
    L.ref_get_config(iv, dv, obs, pi, pd)
    ints = [mine.nfx, mine.nfy, mine.ngrid, mine.ig_obs, mine.ibeg_obs, mine.ig_inlt, mine.ig_outlt,
            mine.nvcycle, mine.nswpm, mine.nswpp, mine.isolve, mine.ibc_xm, mine.ibc_xp, mine.ibc_ym,
            mine.ibc_yp, len(mine.obstacles), len(mine.inlets), len(mine.outlets)]
    assert list(iv) == ints
    dbl = [mine.omega, mine.convergence, mine.xl, mine.yl, mine.amuf, mine.prsc, mine.relxm, mine.relxp,
           *mine.bc_xm, *mine.bc_xp, *mine.bc_ym, *mine.bc_yp, *mine.guess, mine.sc_obs]
    assert list(dv) == dbl
    assert [tuple(obs[4 * k:4 * k + 4]) for k in range(len(cfg.obstacles))] == list(mine.obstacles)
    assert (pi[0], pi[1]) == mine.inlets[0][:2] and (pi[2], pi[3]) == mine.outlets[0][:2]
    assert tuple(pd[0:3]) == mine.inlets[0][2:] and tuple(pd[3:6]) == mine.outlets[0][2:]
