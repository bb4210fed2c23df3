"""Small cases shared by the parity tests: every InputData feature the V-cycle reads,
at sizes the CPU oracle finishes in well under a second per cycle."""
from mgfvm import configs

# touching, overlapping and edge-hugging obstacles: exercises the pressure-copy
# gather with hazards and multi-addition obstacle-face codes
TOUCHING = [(2, 3, 2, 2), (4, 4, 2, 3), (4, 5, 4, 4), (6, 6, 6, 6), (6, 6, 7, 7), (7, 7, 6, 6),
            (1, 1, 5, 6), (8, 8, 1, 1), (3, 3, 8, 8), (3, 4, 8, 8)]


def small_cases():
    s = configs.small
    return {
        "c0_jacobi": configs.c0(1),
        "c0_gs": configs.c0(2),
        "obs_jacobi": s(32, 3, isolve=1, ig_obs=3, sc_obs=0.3,
                        obstacles=[(2, 2, 2, 2), (5, 6, 3, 4), (7, 7, 6, 7)]),
        "obs_gs_touch": s(32, 3, isolve=2, ig_obs=3, sc_obs=0.25, obstacles=TOUCHING),
        "obs_below_coarsest": s(32, 4, isolve=2, ig_obs=3, sc_obs=0.5,
                                obstacles=[(1, 2, 1, 1), (3, 3, 2, 3)]),
        "ports": s(32, 3, isolve=1, ig_inlt=3, ig_outlt=3, bc_xm=(0.0, 0.0, 0.0, 0.0),
                   inlets=[(1, 4, 1.0, 0.0, 1.0), (3, 6, 0.5, 0.1, 0.2)],
                   outlets=[(2, 7, 0.2, 0.0, 0.0)]),
        "bc_mix": s(32, 3, isolve=2, ibc_xm=3, ibc_ym=3, ibc_xp=2, ibc_yp=2),
        "odd_sweeps": s(32, 3, isolve=1, nswpm=3, nswpp=7, relxp=0.7, guess=(0.1, 0.0, 0.2, 0.3)),
        "rect_grid": s(32, 2, isolve=2, nfx=64, nfy=16, xl=4.0, yl=1.0, ig_obs=2,
                       obstacles=[(3, 4, 2, 3), (10, 10, 5, 6)]),
    }
