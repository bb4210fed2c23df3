"""Benchmark: converged solves/s of the SIMPLE + FAS multigrid V-cycle on B200.

Workload (default, N=1): the obstacle-flow configuration — 256 x 256 cells, ngrid 5,
red-black Gauss-Seidel, a seeded staggered lattice of blocks on a 16 x 16 base grid
(porosity 0.75), both Reynolds numbers 10 and 100 solved together.  A step is one
solve of those cases from the initial guess through the public API, as the reference
program runs it: reset (device init + rest_geom) and V-cycles until the level-0 mass
error falls below `convergence` or nvcycle (2000) cycles have run.  FP64 throughout,
bit-identical to the reference's arithmetic.  The schedule (launch shapes only) is
autotuned on the workload before timing.  The line also carries the V-cycle rate of a
64-case batch of such cases against one case alone (`batched`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1|c0|c2] [--no-autotune] [--batch N]

Multi-GPU: one process per GPU (torchrun); every rank solves its own copy of the
workload (independent cases, no data-path collective: weak scaling); time is the max
over ranks of device time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "multigrid-fvm_b200"))

FP_TOL = 0.0            # stop rule of a solve: the reference's own (mass error or nvcycle)
# V-cycles each workload case needs to converge (FP_TOL, FP64).  The FP64 engine is
# bit-identical to the reference per cycle, so these counts are the reference's own;
# the CPU arm uses them to turn its timed sample of cycles into solves/s.  Re-derived
# by every GPU run of this script (reported as cycles_per_solve).
CYCLES_TO_CONVERGE = {"c1": [2000, 2000], "c0": [2000], "c2": None}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------- workloads
WORKLOAD_DIRS = {"c1": [os.path.join(REPO, "workloads", n) for n in ("obstacle256_re10", "obstacle256_re100")]}
WORKLOAD_DESC = {"c1": "obstacle flow 256x256 ngrid 5 RBGS Re {10,100} (2 cases)"}


def workload_config(desc, n_cases, nvcycle, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": desc, "cases_per_gpu": n_cases,
            "stop_rule": "reference: mass error < convergence or nvcycle V-cycles",
            "nvcycle": nvcycle, "l2": "flushed between steps (256 MiB write)",
            "parallelism": f"independent cases, {world} rank(s)"}


def workload(name):
    """(cases, description, per-case inlet u profiles or None)."""
    from mgfvm import configs
    if name == "c1":   # the cases of WORKLOAD_DIRS["c1"] (tests/test_workloads.py)
        return configs.c1_pair(seed=1), WORKLOAD_DESC["c1"], None
    if name == "c0":
        return [configs.c0(1)], "channel 64x64 ngrid 3 Jacobi Re 100", None
    if name == "c2":
        return configs.c2(512, seed=2), "512 mixed-size obstacle cases 64/128/256, coarsest 8x8", None
    if name == "c3":
        return [configs.c3(seed=3)], "1024x1024 ngrid 7 quarter-pixel staggered lattice Re 200", None
    if name == "c4":
        cases, prof = configs.c4(64, seed=4)
        return cases, "64 cases 256x256 ngrid 5 Re 100 random particles, per-face inlet u", prof
    raise SystemExit(f"unknown workload {name}")


def cell_sweeps_per_cycle(cfg):
    """(3 nswpm + nswpp) x sum over levels of visits x interior cells (visits: 1 for
    the finest and coarsest level, 2 otherwise)."""
    tot = 0
    for ig in range(cfg.ngrid):
        cells = (cfg.nfx >> ig) * (cfg.nfy >> ig)
        visits = 1 if ig in (0, cfg.ngrid - 1) else 2
        tot += visits * cells
    return (3 * cfg.nswpm + cfg.nswpp) * tot


def cycle_bytes(cfg):
    """Algorithmic bytes of one V-cycle of a case, from the per-routine FP64 word counts
    of the reference's loops: per cell and level visit 85 words of assembly (fluxes,
    coefficient assembly, masserror/coefp, update) plus 8 per cell-sweep of smoothing
    (3 nswpm + nswpp sweeps); per fine cell of each transfer 100 words of restriction
    and 24 of prolongation."""
    words = 0
    for ig in range(cfg.ngrid):
        cells = (cfg.nfx >> ig) * (cfg.nfy >> ig)
        visits = 1 if ig in (0, cfg.ngrid - 1) else 2
        words += visits * cells * (85 + 8 * (3 * cfg.nswpm + cfg.nswpp))
        if ig < cfg.ngrid - 1:
            words += cells * (100 + 24)
    return 8 * words


def load_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# DRAM bytes (read + write) per k_smooth launch of the p' smoothing on level 0, from ncu
# captures (profiles/k_smooth_obstacle256.md): the 2-case workload of
# `python bench.py --profile-cycles 1`, and the 64-case batch of the `batched` entry.
ROOFLINE_TRAFFIC = {"c1": 7475712, "c1x64": 266211072}


def smoother_roofline(solver, cases, traffic=None, reps=20):
    """Roofline entry of k_smooth: the p' smoothing of level 0 (nswpp red-black sweeps,
    split into launches of up to 10 half-sweeps each), timed with CUDA events on the
    context stream.  Algorithmic bytes: 64 B per cell-sweep (6 coefficients + phi read
    + phi write, FP64) x nswpp x interior cells, per launch."""
    solver.time_op("smooth_pp", 0, 2)
    kms, klaunch = solver.time_op("smooth_pp", 0, reps)
    per_launch_ms = kms / klaunch
    bytes_per_op = sum(64 * c.nswpp * c.nfx * c.nfy for c in cases)
    algo_bytes = bytes_per_op * reps / klaunch
    peaks = load_peaks()
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = algo_bytes / (per_launch_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "kernel": "k_smooth (shared-memory tile smoother, p' equation, level 0)",
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "per_launch_us": round(per_launch_ms * 1e3, 3), "launches_per_op": klaunch // reps,
            "algorithmic_bytes_per_launch": int(algo_bytes)}


def batched_rate(nb, device, tune, cycles_per_solve, ncyc=40):
    """V-cycle rate of `nb` obstacle-flow cases (256x256, ngrid 5, RBGS, Re alternating
    10/100, seeded staggered lattices) in one context, against one case alone; solves/s
    follow from the cycles one solve runs (the reference's stop rule does not fire on
    these cases within nvcycle, so every solve runs nvcycle cycles)."""
    from mgfvm import Solver, configs
    out = {}
    for label, n in (("one_case", 1), ("batch", nb)):
        cases = [configs.c1(10.0 if k % 2 == 0 else 100.0, seed=k + 1) for k in range(n)]
        with Solver(cases, device=device, sync_every=64) as s:
            if tune:
                s.autotune(3)
            s.cycle(3)
            s.cycle(ncyc)
            ms = s.last_elapsed_ms / ncyc
            gbs = sum(cycle_bytes(c) for c in cases) / (ms / 1e3) / 1e9
            peaks = load_peaks()
            peak = peaks.get("hbm_gbs", 6650.0)
            out[label] = {"cases": n, "ms_per_cycle": round(ms, 4),
                          "case_cycles_per_s": round(n / (ms / 1e3), 1),
                          "solves_per_s": round(n / (ms / 1e3) / max(cycles_per_solve), 4),
                          "cycle_roofline": {"bound": "hbm", "algorithmic_bytes_per_case_cycle": cycle_bytes(cases[0]),
                                             "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                                             "frac": round(gbs / peak, 4),
                                             "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}}
            if n > 1:   # level-0 fields of the batch exceed L2: the smoother against HBM
                out[label]["smoother_roofline"] = smoother_roofline(s, cases, ROOFLINE_TRAFFIC.get(f"c1x{n}"))
    out["speedup_per_case"] = round(out["batch"]["case_cycles_per_s"] / out["one_case"]["case_cycles_per_s"], 2)
    out["note"] = (f"{ncyc} graph-replayed V-cycles timed with CUDA events after 3 warm-up cycles; "
                   f"solves/s = case-cycles/s / {max(cycles_per_solve)} cycles per solve")
    return out


def gradient_rate(device, cycles=4, check=True):
    """Forward-mode gradient of J (mgfvm_objective) for the first adjoint-configuration
    case (256 x 256, seeded random obstacles, Re 100, per-face inlet profile): one
    tangent context of nfy + 2 cases (every inlet face, amuf, prsc), timed per
    V-cycle; two of its derivatives checked against central differences (h = 1e-6)
    of the CPU oracle's V-cycles."""
    from mgfvm import Solver, configs
    cases, profs = configs.c4(1, seed=4)
    cfg, prof = cases[0], profs[0]
    dirs = [("inlet", k) for k in range(cfg.nfy)] + [("amuf", 0), ("prsc", 0)]
    s = Solver([cfg] * len(dirs), device=device, tangent=True)
    for c, (kind, idx) in enumerate(dirs):
        s.set_inlet_profile(c, prof)
        s.set_direction(c, kind, idx)
    s.cycle(1)                                  # untimed warm-up cycle
    s.cycle(cycles)
    ms = s.last_elapsed_ms / cycles
    total = 1 + cycles
    dj = np.array([s.objective(c)[1] for c in range(len(dirs))])
    s.close()
    out = {"config": "adjoint configuration case 0: 256x256, ngrid 5, seeded random obstacles, Re 100, "
                     "inlet profile 1 + 0.1 N(0,1)",
           "method": "forward mode (tangent-linear, dual numbers), one batch of all directions",
           "directions": len(dirs), "ms_per_cycle": round(ms, 3),
           "direction_cycles_per_s": round(len(dirs) / (ms / 1e3), 1)}
    if check:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import dataclasses
        import oracle

        def j_after(c, pr):
            o = oracle.OracleCase(c, pr)
            o.cycle(total)
            p, sc = o.get(0, "p"), o.get(0, "sc")
            o.close()
            ny = p.shape[0] - 2
            return (p[1:-1, 1].sum() / ny - p[1:-1, -2].sum() / ny) + sc[1:-1, -1].sum() / ny

        k = int(np.argmax(np.abs(dj[:cfg.nfy])))
        h = 1e-6 * abs(prof[k])
        pp, pm = prof.copy(), prof.copy()
        pp[k] += h
        pm[k] -= h
        fd_in = (j_after(cfg, pp) - j_after(cfg, pm)) / (2 * h)
        ha = 1e-6 * cfg.amuf
        fd_a = (j_after(dataclasses.replace(cfg, amuf=cfg.amuf + ha), prof)
                - j_after(dataclasses.replace(cfg, amuf=cfg.amuf - ha), prof)) / (2 * ha)
        out["check"] = {"cycles": total, "inlet_face": k,
                        "rel_err_inlet": abs(dj[k] - fd_in) / abs(fd_in),
                        "rel_err_amuf": abs(dj[cfg.nfy] - fd_a) / abs(fd_a),
                        "bar": 1e-4}
    return out


def adjoint_rate(device, ncases=64, cycles=10, check=True):
    """Reverse-mode gradients of the adjoint configuration (ncases cases of 256 x 256,
    seeded random obstacles, Re 100, per-face inlet profiles): one mgfvm_adjoint run of
    the whole batch over `cycles` V-cycles (forward run with checkpoints, re-runs, and
    the taped cycle + transpose per cycle), against a plain forward run of the same
    cycles; case 0's gradient checked against the forward mode (all nfy + 2 directions)
    and one inlet face against the oracle's central difference."""
    from mgfvm import Solver, configs, gradient
    cases, profs = configs.c4(ncases, seed=4)
    with Solver(cases, device=device, sync_every=64) as s:
        for k, pr in enumerate(profs):
            s.set_inlet_profile(k, pr)
        s.cycle(cycles)
        fwd_ms = s.last_elapsed_ms / cycles
        s.adjoint(2)                                   # warm-up
        s.adjoint(cycles)
        adj_ms = s.last_elapsed_ms
        res = [s.adjoint_gradient(k, allow_nonfinite=True) for k in range(ncases)]
        res0 = res[0]
        diverged = [k for k, r in enumerate(res) if not np.isfinite(r[2])]
    out = {"config": f"adjoint configuration: {ncases} cases 256x256, ngrid 5, seeded random obstacles, Re 100, "
                     f"inlet profile 1 + 0.1 N(0,1)",
           "method": "reverse mode: taped V-cycle and its phase-by-phase transpose, checkpoints every ~sqrt(n) "
                     "cycles",
           "cycles": cycles, "gradients": ncases, "directions_per_gradient": cases[0].nfy + 2,
           "ms_total": round(adj_ms, 3), "ms_per_cycle": round(adj_ms / cycles, 3),
           "forward_ms_per_cycle": round(fwd_ms, 3),
           "cost_vs_forward_cycles": round(adj_ms / cycles / fwd_ms, 2),
           "diverged_cases": diverged,
           "note": "a gradient over n cycles costs cost_vs_forward_cycles x the plain batch's n cycles"}
    if check:
        j, g_in, g_a, g_p = res0
        jf, gf, af, pf = gradient(cases[0], profs[0], cycles, device)
        full_a, full_f = np.concatenate([g_in, [g_a, g_p]]), np.concatenate([gf, [af, pf]])
        out["check_vs_forward_mode"] = float(np.abs(full_a - full_f).max() / np.abs(full_f).max())
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        import oracle

        def j_after(pr):
            o = oracle.OracleCase(cases[0], pr)
            o.cycle(cycles)
            p, sc = o.get(0, "p"), o.get(0, "sc")
            o.close()
            ny = p.shape[0] - 2
            return (p[1:-1, 1].sum() / ny - p[1:-1, -2].sum() / ny) + sc[1:-1, -1].sum() / ny

        k = int(np.argmax(np.abs(g_in)))
        h = 1e-6 * abs(profs[0][k])
        pp, pm = profs[0].copy(), profs[0].copy()
        pp[k] += h
        pm[k] -= h
        fd = (j_after(pp) - j_after(pm)) / (2 * h)
        out["check_vs_oracle_central_difference"] = {"inlet_face": k, "rel_err": abs(g_in[k] - fd) / abs(fd),
                                                     "bar": 1e-4}
    return out


def mixed_solve(cases, device, ref_solver, tune, profiles=None):
    """One solve of the workload with MGFVM_PREC_MIXED (FP32 correction smoothing
    against FP64 residuals), timed like a bench step, and the relative L2 distance of
    its final fields to the FP64 solve's (`ref_solver` holds the FP64 result; p
    compared mean-free over the interior, its level being arbitrary).  Also returns
    the mixed solve's level-0 fields (for the comparison with the CPU oracle)."""
    import torch
    from mgfvm import Solver
    with Solver(cases, device=device, precision="mixed", sync_every=64) as s:
        for k, pr in enumerate(profiles or []):
            s.set_inlet_profile(k, pr)
        if tune:
            s.autotune(3)
        s.solve(20, FP_TOL, allow_nonfinite=True)
        s.reset()
        torch.cuda.synchronize()
        s.solve(max(c.nvcycle for c in cases), FP_TOL, allow_nonfinite=True)
        ms = s.last_elapsed_ms
        bad = set(s.diverged()) | set(ref_solver.diverged())
        fields = [{f: s.field(k, 0, f) for f in ("u", "v", "p", "sc")} for k in range(len(cases))]
        per_case = [None if k in bad else
                    field_errors(fields[k], {f: ref_solver.field(k, 0, f) for f in ("u", "v", "p", "sc")})
                    for k in range(len(cases))]
        err = max([e for e in per_case if e is not None], default=0.0)
    return {"value": round((len(cases) - len(bad)) / (ms / 1e3), 4), "unit": "solves/s", "ms_per_step": round(ms, 3),
            "rel_l2_vs_fp64_solve": err, "diverged": len(bad),
            "form": "levels smoothed in tiles keep FP32 smoother operands (aw, ae, as, an, 1/ap and the FP64 "
                    "residual, stored by the FP64 assembly) and iterate an FP32 correction; p' in FP32; "
                    "transfers, defects, norms and the one-CTA levels FP64"}, fields, bad, per_case


# --------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"mgfvm_bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # let nvidia-smi finish its start-up (NVML initialisation) before the timed
            # region opens: its first sample marks it as running
            for _ in range(100):
                if os.path.getsize(self.path) > 0 or self.proc.poll() is not None:
                    break
                time.sleep(0.05)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9:
                    rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------- CPU side
def _cpu_case(src):
    """The reference build (or the oracle port where the reference build is absent) on
    one case: `src` is a directory holding InputData + pattern.txt (read by the
    reference itself) or a CaseConfig as a dict."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "multigrid-fvm_b200"))
    import oracle
    from mgfvm.inputs import CaseConfig
    if oracle.ref_available():
        if isinstance(src, str):
            return "reference", oracle.RefCase(None, workdir=src)
        return "reference", oracle.RefCase(CaseConfig(**src))
    if isinstance(src, str):
        from mgfvm import read_case
        return "port", oracle.OracleCase(read_case(src))
    return "port", oracle.OracleCase(CaseConfig(**src))


def _ref_worker(args):
    """One process: time `ncyc` V-cycles of one case on the CPU."""
    src, ncyc, warm = args
    kind, r = _cpu_case(src)
    if kind == "reference":
        r.time_cycles(warm)
        return kind, r.time_cycles(ncyc) / ncyc
    r.cycle(warm)
    t = time.perf_counter()
    r.cycle(ncyc)
    return kind, (time.perf_counter() - t) / ncyc


def _warm_worker(src):
    """Loads the CPU implementation in a pool process (nothing is timed)."""
    _cpu_case(src)
    return 0


def _ref_solve_worker(args):
    """One process: `ncyc` V-cycles of one case on the CPU from its initial state (the
    solve a GPU step ran); returns the level-0 u, v, p, sc and the seconds taken."""
    src, ncyc = args
    kind, r = _cpu_case(src)
    t = time.perf_counter()
    r.cycle(ncyc)
    sec = time.perf_counter() - t
    return kind, sec, {f: r.get(0, f) for f in ("u", "v", "p", "sc")}


def field_errors(got, ref):
    """Relative L2 distance of one case's level-0 fields: u, v, sc over the whole array,
    p over the interior with its mean removed (its level is arbitrary); the max."""
    err = 0.0
    for f in ("u", "v", "sc"):
        a, b = got[f], ref[f]
        err = max(err, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))
    a, b = got["p"][1:-1, 1:-1], ref["p"][1:-1, 1:-1]
    a, b = a - a.mean(), b - b.mean()
    return max(err, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))


def cpu_sample(cases, cycles_to_converge, ncyc, procs):
    """solves/s of the CPU implementation on `procs` host processes (one case each,
    round-robin over the workload's cases), from the mean time per V-cycle."""
    import dataclasses
    import multiprocessing as mp
    srcs = cases if isinstance(cases[0], str) else [dataclasses.asdict(c) for c in cases]
    jobs = [(srcs[k % len(srcs)], ncyc, 2) for k in range(procs)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, jobs)
    wall = time.perf_counter() - t0
    kind = res[0][0]
    # mean time of one solve of the workload's cases on one core
    per_case = []
    for k, (_, tcyc) in enumerate(res):
        per_case.append(tcyc * cycles_to_converge[k % len(cases)])
    t_solve_one_core = float(np.mean(per_case))
    return procs / t_solve_one_core, kind, wall, float(np.mean([r[1] for r in res]))


def run_reference_arm(a, rank, world):
    if rank != 0:
        return
    # the reference reads the workload's own InputData/pattern.txt directories; nothing
    # of this package's native code is loaded
    if a.workload in WORKLOAD_DIRS:
        cases, nvcycle, desc = WORKLOAD_DIRS[a.workload], [2000, 2000], WORKLOAD_DESC[a.workload]
    else:
        cs, desc, _ = workload(a.workload)
        cases, nvcycle = cs, [c.nvcycle for c in cs]
    ctc = CYCLES_TO_CONVERGE.get(a.workload)
    if ctc is None:
        print(json.dumps({"impl": "reference", "unavailable": f"no converged cycle counts for {a.workload}"}))
        return
    procs = max(1, min(os.cpu_count() or 1, 64))
    ncyc = {"c1": 30, "c0": 400}.get(a.workload, 20)
    vals = []
    for s in range(a.warmup + a.steps):
        v, kind, wall, tcyc = cpu_sample(cases, ctc, ncyc, procs)
        if s >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    sample = (f"{ncyc} V-cycles per process after 2 warm-up cycles, {procs} processes (one case each, "
              f"round-robin over the workload's cases); solves/s = processes / (mean time per V-cycle x "
              f"V-cycles to converge {ctc})")
    line = {
        "impl": "reference", "metric": "converged solves/s", "value": value, "unit": "solves/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded obstacle patterns)",
        "config": workload_config(desc, len(cases), nvcycle, world),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# --------------------------------------------------------------- GPU side
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c0", "c2", "c3", "c4"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tail", type=int, default=-1, help="first level of the one-CTA coarse kernel (-1 auto)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's default schedule")
    ap.add_argument("--batch", type=int, default=64,
                    help="cases of the batched obstacle-flow measurement (0: skip it)")
    ap.add_argument("--no-gradient", action="store_true", help="skip the gradient measurements")
    ap.add_argument("--parity-dump", default=None,
                    help="write per-case hashes of the timed solve's final level-0 fields, the cycles each case "
                         "ran and the mixed form's distance to them to this JSON file (oracle/config_parity.py "
                         "compares them with the oracle)")
    ap.add_argument("--profile-cycles", type=int, default=0,
                    help="only run 3 warm-up V-cycles then this many V-cycles of the workload "
                         "(for ncu launch lists) and exit")
    ap.add_argument("--profile-tangent", type=int, default=0,
                    help="only run this many tangent V-cycles of a small gradient batch (64x64 channel, "
                         "all 66 directions) after 2 warm-up cycles, inside the NVTX range 'profile', and exit")
    ap.add_argument("--profile-adjoint", type=int, default=0,
                    help="only run the reverse mode over this many V-cycles of one adjoint-configuration case "
                         "(256x256) after a 1-cycle warm-up, the timed run inside the NVTX range 'profile', and exit")
    ap.add_argument("--profile-batch-smoother", choices=["plain", "tma", "band"], default=None,
                    help="only run one V-cycle of the 64-case obstacle-flow batch (levels 0-2 smoothed by "
                         "512-thread tiles of 6 units, per-thread or TMA-staged loads; 'band': the default "
                         "schedule, levels 1-2 by band visits) after 3 warm-up cycles, inside the NVTX range "
                         "'profile', and exit")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        run_reference_arm(a, rank, world)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    from mgfvm import Solver
    if a.profile_adjoint:
        from mgfvm import configs
        cases, profs = configs.c4(1, seed=4)
        with Solver(cases, device=local) as s:
            s.set_inlet_profile(0, profs[0])
            s.adjoint(1)
            torch.cuda.nvtx.range_push("profile")
            s.adjoint(a.profile_adjoint)
            torch.cuda.nvtx.range_pop()
            log(f"adjoint: {s.last_elapsed_ms / a.profile_adjoint:.3f} ms per cycle (one case)")
        return
    if a.profile_batch_smoother:
        from mgfvm import configs
        cases = [configs.c1(10.0 if k % 2 == 0 else 100.0, seed=k + 1) for k in range(64)]
        t = 2 if a.profile_batch_smoother == "tma" else 1
        with Solver(cases, device=local) as s:
            if a.profile_batch_smoother != "band":
                s.set_tuning(smooth_units={0: 6, 1: 6, 2: 6}, smooth_threads={0: 512, 1: 512, 2: 512},
                             smooth_tma={0: t, 1: t, 2: t}, band_visit=[1] * 5)
            s.cycle(3)
            torch.cuda.nvtx.range_push("profile")
            s.cycle(1)
            torch.cuda.nvtx.range_pop()
            s.cycle(10)
            log(f"batch smoother {a.profile_batch_smoother}: {s.last_elapsed_ms / 10:.3f} ms per V-cycle")
        return
    if a.profile_tangent:
        from mgfvm import configs
        cfg = configs.c0(2)
        dirs = [("inlet", k) for k in range(cfg.nfy)] + [("amuf", 0), ("prsc", 0)]
        with Solver([cfg] * len(dirs), device=local, tangent=True) as t:
            for c, (kind, idx) in enumerate(dirs):
                t.set_direction(c, kind, idx)
            t.cycle(2)
            torch.cuda.nvtx.range_push("profile")
            t.cycle(a.profile_tangent)
            torch.cuda.nvtx.range_pop()
            log(f"tangent: {len(dirs)} directions, {t.last_elapsed_ms / a.profile_tangent:.3f} ms per V-cycle")
        return
    cases, desc, profiles = workload(a.workload)
    n_cases = len(cases)
    solver = Solver(cases, device=local, sync_every=64, tail_level=a.tail)
    for k, pr in enumerate(profiles or []):
        solver.set_inlet_profile(k, pr)
    tuned = None
    if not a.no_autotune:
        t_before, t_after, tuned = solver.autotune(20)
        log(f"autotune: {t_before * 1e3:.1f} -> {t_after * 1e3:.1f} us per cycle")
    if a.profile_cycles:
        solver.cycle(3)
        n0 = solver.kernel_launches
        torch.cuda.nvtx.range_push("profile")     # ncu --nvtx --nvtx-include profile/
        solver.cycle(a.profile_cycles)
        torch.cuda.nvtx.range_pop()
        nprof = solver.kernel_launches - n0
        solver.cycle(20)
        log(f"20 cycles: {solver.last_elapsed_ms / 20:.3f} ms per cycle (tail {a.tail})")
        log(f"profile: {n0} launches before, {nprof} in {a.profile_cycles} cycle(s)")
        prof = [solver.profile_cycle() for _ in range(3)][-1]
        tot = sum(p[2] for p in prof)
        agg = {}
        for name, lv, t in prof:
            k = f"{name}@{lv}"
            c, v = agg.get(k, (0, 0.0))
            agg[k] = (c + 1, v + t)
        log(f"live per-launch profile (events between direct launches), cycle {tot * 1e3:.1f} us:")
        for k, (c, v) in sorted(agg.items(), key=lambda kv: -kv[1][1]):
            log(f"  {k:22s} x{c:3d} {v * 1e3:9.1f} us  {100 * v / tot:5.1f}%  avg {v / c * 1e3:7.2f} us")
        solver.close()
        return
    stream = torch.cuda.ExternalStream(solver.stream, device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        solver.reset()
        return solver.solve(max(c.nvcycle for c in cases), FP_TOL, allow_nonfinite=True)

    # Parity of the timed result: the CPU runs every case of the workload for the cycles
    # its GPU solve runs, from the same initial state, in background processes (one per
    # case) while the GPU part runs; its final fields are the oracle of the solve.  The
    # processes start (and finish their imports) before the warm-up steps, so that no
    # interpreter start-up competes with the host thread that drives the timed steps.
    parity_jobs = parity_pool = srcs = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline and n_cases <= 8 and not profiles:
        # (per-face inlet profiles are not expressible as reference input files)
        import dataclasses
        import multiprocessing as mp
        srcs = WORKLOAD_DIRS.get(a.workload) or [dataclasses.asdict(c) for c in cases]
        parity_pool = mp.get_context("spawn").Pool(n_cases)
        parity_pool.map(_warm_worker, srcs)
    for _ in range(a.warmup):
        cyc = step()
    # cases on which the reference's own iteration turns NaN/Inf stop at that cycle and
    # are not counted as solves (the reference's stop test never fires on NaN)
    diverged = solver.diverged()
    if parity_pool is not None:
        parity_t0 = time.perf_counter()
        parity_jobs = parity_pool.map_async(_ref_solve_worker, [(srcs[k], int(cyc[k])) for k in range(n_cases)])
    launches0 = solver.kernel_launches
    cycles = []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record(stream)
        solve_ms = []
        for _ in range(a.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)          # L2 flush between steps (256 MiB write)
            cycles.append(step())
            solve_ms.append(solver.last_elapsed_ms)
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    log(f"timed steps: {ms / max(1, a.steps):.1f} ms each; the solves inside them "
        + ", ".join(f"{t:.1f}" for t in solve_ms) + " ms (device, first to last chunk)")
    launches = solver.kernel_launches - launches0
    # the timed solve's final level-0 fields (later measurements change the state)
    gpu_fields = [{f: solver.field(k, 0, f) for f in ("u", "v", "p", "sc")} for k in range(n_cases)] \
        if parity_jobs is not None else None
    gpu_hashes = None
    if a.parity_dump:
        import hashlib
        gpu_hashes = [hashlib.sha256(b"".join(np.ascontiguousarray(solver.field(k, 0, f)).tobytes()
                                              for f in ("u", "v", "p", "sc"))).hexdigest() for k in range(n_cases)]
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    total_solves = (n_cases - len(diverged)) * a.steps * world
    value = total_solves / (ms / 1e3)
    cyc_arr = np.array(cycles)
    cycles_per_solve = [int(x) for x in cyc_arr[-1]]
    sweeps = sum(cell_sweeps_per_cycle(c) * int(n) for c, n in zip(cases, cycles_per_solve))
    cell_sweeps_per_s = sweeps * a.steps * world / (ms / 1e3)

    # ---- dominant kernel: the shared-memory tile smoother on level 0, p' equation (live)
    roofline = smoother_roofline(solver, cases, ROOFLINE_TRAFFIC.get(a.workload))

    # ---- end to end through the public API with host buffers
    e2e = None
    if rank == 0 or True:
        def e2e_step():
            t = [time.perf_counter()]
            with Solver(cases, device=local) as s2:
                t.append(time.perf_counter())
                for k, pr in enumerate(profiles or []):
                    s2.set_inlet_profile(k, pr)
                if tuned:
                    s2.set_tuning(**tuned)
                t.append(time.perf_counter())
                s2.solve(max(c.nvcycle for c in cases), FP_TOL, allow_nonfinite=True)
                t.append(time.perf_counter())
                dev = s2.last_elapsed_ms
                for k in range(n_cases):
                    for f in ("u", "v", "p", "sc"):
                        s2.field(k, 0, f)
                t.append(time.perf_counter())
                b = s2.transfer_bytes
            t.append(time.perf_counter())
            d = np.diff(t) * 1e3
            log(f"e2e step: create {d[0]:.1f} ms, inputs+schedule {d[1]:.1f}, solve {d[2]:.1f} "
                f"(device {dev:.1f}), fields {d[3]:.1f}, release {d[4]:.1f}")
            return b

        e2e_step()                           # untimed warm-up step
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h2d = d2h = 0
        for _ in range(max(1, a.steps)):
            b = e2e_step()
            h2d += b[0]
            d2h += b[1]
        torch.cuda.synchronize()
        t_e2e = time.perf_counter() - t0
        e2e = {"value": (n_cases - len(diverged)) * max(1, a.steps) * world / t_e2e, "unit": "solves/s",
               "h2d_bytes_per_step": int(h2d / max(1, a.steps)), "d2h_bytes_per_step": int(d2h / max(1, a.steps))}
        if world > 1:
            t = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e["value"] = (n_cases - len(diverged)) * max(1, a.steps) * world / float(t.item())

    # ---- mixed precision: the same solve with FP32 correction smoothing
    mixed = mixed_fields = None
    mixed_bad = set()
    if world == 1:
        mixed, mixed_fields, mixed_bad, mixed_per_case = mixed_solve(cases, local, solver, tuned is not None,
                                                                      profiles)

    # ---- batched throughput: many obstacle-flow cases in one context
    batched = None
    if a.batch > 0 and a.workload == "c1":
        batched = batched_rate(a.batch, local, not a.no_autotune, cycles_per_solve)

    # ---- derivatives: a whole gradient of J by forward mode, one batch
    grad = adj = None
    if world == 1 and not a.no_gradient:
        grad = gradient_rate(local, check=not a.no_cpu_baseline)
        adj = adjoint_rate(local, check=not a.no_cpu_baseline)

    if a.parity_dump and rank == 0:
        dump = {"workload": a.workload, "cases": []}
        for k in range(n_cases):
            dump["cases"].append({"cycles": int(cycles_per_solve[k]), "diverged": k in diverged,
                                  "sha256": gpu_hashes[k],
                                  "mixed_rel_l2_vs_fp64": None if mixed_fields is None else mixed_per_case[k]})
        with open(a.parity_dump, "w") as f:
            json.dump(dump, f)

    # ---- parity of the timed solve against the CPU oracle's run of the same cycles
    parity = None
    if parity_jobs is not None:
        res = parity_jobs.get()
        parity_pool.close()
        parity_pool.join()
        wall = time.perf_counter() - parity_t0
        per_case, per_case_mixed = [], []
        for k, (kind, sec, ref) in enumerate(res):
            per_case.append(None if k in diverged else field_errors(gpu_fields[k], ref))
            if mixed_fields is not None:
                per_case_mixed.append(None if k in mixed_bad else field_errors(mixed_fields[k], ref))
        ok = [e for e in per_case if e is not None]
        okm = [e for e in per_case_mixed if e is not None]
        parity = {
            "oracle": f"{'the reference build (gcc -O3)' if res[0][0] == 'reference' else 'the oracle port'}: "
                      f"every case for the cycles its GPU solve ran {cycles_per_solve}, one host process per case "
                      f"({wall:.0f} s wall, longest case {max(r[1] for r in res):.0f} s)",
            "metric": "relative L2 of level-0 u, v, sc and mean-free interior p, max over fields",
            "fp64": {"max": max(ok) if ok else None, "per_case": per_case},
            "mixed": {"max": max(okm) if okm else None, "per_case": per_case_mixed} if mixed_fields else None,
            "bar": 1e-6,
        }

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        ctc = cycles_per_solve
        v, kind, wall, tcyc = cpu_sample(WORKLOAD_DIRS.get(a.workload) or cases, ctc,
                                         {"c1": 30, "c0": 400}.get(a.workload, 20),
                                         max(1, min(os.cpu_count() or 1, 64)))
        cpu = {"value": v, "unit": "solves/s", "cores": max(1, min(os.cpu_count() or 1, 64)), "kind": kind,
               "sample": f"V-cycles timed per host process ({wall:.1f} s wall), one case per process, "
                         f"extrapolated with the GPU's cycles-to-converge {ctc}"}

    if rank == 0:
        line = {
            "metric": "converged solves/s", "value": round(value, 4), "unit": "solves/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded obstacle patterns)",
            "config": workload_config(desc, n_cases, [c.nvcycle for c in cases], world),
            "cycles_per_solve": cycles_per_solve if n_cases <= 8 else
            {"min": int(min(cycles_per_solve)), "max": int(max(cycles_per_solve)),
             "mean": float(np.mean(cycles_per_solve))},
            "diverged": {"cases": len(diverged), "of": n_cases,
                         "note": "the mass error turned NaN/Inf (the reference build diverges on the same "
                                 "inputs); stopped at that cycle, not counted as solves"} if diverged else None,
            "cell_sweeps_per_s": cell_sweeps_per_s,
            "l2_rel_err_vs_oracle": parity,
            "roofline": roofline,
            "batched": batched,
            "mixed": mixed,
            "gradient": grad,
            "adjoint": adj,
            "schedule": {"autotuned": tuned is not None,
                         "tuning": {k: v[:max(c.ngrid for c in cases)] if isinstance(v, list) else v
                                    for k, v in tuned.items()} if tuned else None},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
