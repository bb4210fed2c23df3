"""Regenerate the golden fixtures of tests/golden/ from the reference itself.

Runs only where the reference source exists (it builds oracle/_ref from
Version-6-26-04.c with oracle/Makefile; MGFVM_REF_DIR names its directory):

    MGFVM_REF_DIR=<reference checkout> python tests/golden/make_golden.py

Writes, per case,
  <name>.npz     initial state (masks, areas, boundary values) of every level, the
                 state after 3 V-cycles and the per-cycle mass-error history, all from
                 the unmodified reference compiled with gcc (oracle/ref_harness.c);
  c0gs_fixed.npz the level-0 u, v, p, sc of the 64x64 Gauss-Seidel channel after 2000
                 V-cycles (its V-cycle fixed point) and the 2000 mass errors;
  cli/           InputData, pattern.txt and the reference binary's stdout,
                 vtk_acc.vtk and convergence.csv for a 16x16 obstacle case.
The parity tests compare the C oracle (and, through it, the CUDA engine) with these.
"""
import os
import shutil
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "multigrid-fvm_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "tests"))

INIT_FIELDS = ["u", "v", "p", "sc", "spu", "spv", "spsc", "areax", "areay", "apu", "apv"]
CYCLE_FIELDS = ["u", "v", "p", "pp", "sc", "resu", "resv", "ressc", "apu", "apv"]
NCYC = 3


def golden_cases():
    from cases import small_cases
    sc = small_cases()
    keep = ["c0_jacobi", "obs_gs_touch", "obs_below_coarsest", "ports", "bc_mix", "odd_sweeps", "rect_grid"]
    return {k: sc[k] for k in keep}


def dump_case(name, cfg):
    import oracle
    r = oracle.RefCase(cfg)
    out = {}
    for ig in range(r.ngrid):
        out[f"init_tag_{ig}"] = r.tag(ig)
        out[f"ranges_{ig}"] = r.obstacle_ranges(ig)
        for f in INIT_FIELDS:
            out[f"init_{f}_{ig}"] = r.get(ig, f)
    r.cycle(NCYC)
    for ig in range(r.ngrid):
        for f in CYCLE_FIELDS:
            out[f"cyc_{f}_{ig}"] = r.get(ig, f)
    out["err"] = r.history()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


def dump_fixed_point():
    import oracle
    from mgfvm import configs
    r = oracle.RefCase(configs.c0(2))
    r.cycle(2000)
    np.savez_compressed(os.path.join(HERE, "c0gs_fixed.npz"), err=r.history(),
                        **{f: r.get(0, f) for f in ("u", "v", "p", "sc")})


def cli_case():
    from mgfvm import configs
    return configs.small(16, 3, isolve=2, nvcycle=6, ig_obs=3, sc_obs=0.2,
                         obstacles=[(1, 1, 2, 2), (2, 3, 3, 3)])


def dump_cli():
    import oracle
    d = os.path.join(HERE, "cli")
    if os.path.isdir(d):
        shutil.rmtree(d)
    os.makedirs(d)
    cli_case().write(d)
    res = subprocess.run([oracle.REF_BIN], cwd=d, capture_output=True, text=True, check=True)
    with open(os.path.join(d, "stdout.txt"), "w") as f:
        f.write(res.stdout)


def main():
    import oracle
    oracle.build()
    if not oracle.ref_available():
        raise SystemExit("reference build missing: the reference source is needed to regenerate goldens")
    for name, cfg in golden_cases().items():
        dump_case(name, cfg)
        print("wrote", name)
    dump_fixed_point()
    print("wrote c0gs_fixed")
    dump_cli()
    print("wrote cli/")


if __name__ == "__main__":
    main()
