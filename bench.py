"""Benchmark of the ADMM solve loop on the 32x32x128 twisted-and-bent bar.

Workload: 786,432 tets / 140,481 vertices, E = 1e5 Pa, nu = 0.45, global
L-BFGS history 5, reweighting (and GPU refactorization) every 10 iterations,
FP64.  One step = one ADMM iteration (local step, global L-BFGS step with its
triangular solves, reweight check).

Metric: ADMM element-iterations per second (elements x iterations / seconds),
the throughput behind the time-to-energy-gap metric; `local_elems_per_s` adds
the local step alone.  Inputs are far larger than L2 (the element state is
~0.7 GB), so no L2 flush is needed between steps.  The same line carries the
learned/FP32 form on the same bar; the time to relative energy gap 1e-6 of the
solver forms on the 8x8x32 bar, on a 786,432-tet bar with a 180 deg twist (the
bent bar above keeps inverted elements and does not reach that gap) and on the
3,932,160-tet bar with a 720 deg twist (reweight every 20), plain FP64 against
learned/FP32; and 64 uneven bars solved as one batch and one by one.

The reference arm (--impl reference) runs the reference's own solver,
compiled from its sources with two documented one-line patches for the
settings above (history 5, reweight every 10: oracle/Makefile), on the same
bar and times the same kind of window (ten iterations hold one reweight and
refactorization, as any ten of ours do).  Both arms' `e2e` is a whole solve of
W + K iterations from host data, setup included.

Usage:  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
        [--precision fp64|mixed] [--parts main,learned,gap,e2e,batch]
For N > 1 launch with torchrun: every rank solves its own replica of the bar
(the path does not shard; replicas only, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to rel. energy gap 1e-6: learned/FP32 vs plain FP64 GPU; local elems/s"
UNIT = "elem-iter/s"
WORKLOAD = "bar 32x32x128 cubes x6 tets (786,432 tets, 140,481 verts), 360 deg twist + 90 deg bend, E=1e5 nu=0.45"
E_YOUNG, NU = 1e5, 0.45


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--parts", default="main,learned,gap,e2e,batch",
                   help="measurements to run after the main one (main is always run)")
    return p.parse_args()


# ---- clocks ----------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms during the
    timed region (one nvidia-smi process in loop mode, stopped afterwards)."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._p = None
        self._t = None

    def _read(self):
        for line in self._p.stdout:
            f = [x.strip() for x in line.strip().split(",")]
            if len(f) >= 7:
                self.samples.append(f)

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                        "--format=csv,noheader,nounits", "-lms", "100"],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)   # first sample before the timed work starts
        return self

    def __exit__(self, *a):
        if self._p:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._p.kill()
            self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and
                          s[3 + i].lower() in ("active", "1", "yes")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---- distributed plumbing ----------------------------------------------------------
def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def _all_reduce(pg, v: float, op) -> float:
    import torch
    # NCCL reduces device tensors; gloo (the CPU tests of this harness) host ones
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    pg.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(pg, v: float) -> float:
    """The slowest rank's time: every rank calls it at the same point."""
    return v if pg is None else _all_reduce(pg, v, pg.ReduceOp.MAX)


def sum_over_ranks(pg, v: float) -> float:
    """The units all ranks processed: every rank calls it at the same point."""
    return v if pg is None else _all_reduce(pg, v, pg.ReduceOp.SUM)


# ---- bytes / flops model (algorithmic, per launch) -----------------------------------
def local_step_bytes(ne: int, fp: int) -> int:
    """k_local per element: reads symF, U, Z (9 each, fp bytes), w2, vol (8), slast (3 fp);
    writes Z, U (9 each), slast (3), w2c (8)."""
    return ne * (fp * (9 + 9 + 9 + 3) + 16 + fp * (9 + 9 + 3) + 8)


def grad_step_bytes(ne: int, nf: int, fp: int) -> int:
    """k_grad per element: idx (16), Di (96), x of 4 vertices (96, mostly L2 hits; counted once per
    vertex: 24 nf), Z, U (9 fp each), w2, vol (16); writes symF (9 fp), sig (3 fp), gel (12 fp)."""
    return ne * (16 + 96 + fp * 18 + 16 + fp * 24) + 24 * nf


# ---- reference arm -------------------------------------------------------------------
# The reference refactors with Eigen's single-threaded SimplicialLDLT, about
# 200 s on the 786,432-tet bar; ten timed iterations hold exactly one of the
# every-10 refactorizations, the same share as any window of our arm.
REF_TIMED_ITERS = 10


def run_reference(args, rank):
    """The reference's own CPU solver on the same workload and settings as our
    arm: oracle/_ref/quasi_ref_m5, compiled from the reference's sources with
    the two documented one-line patches of oracle/Makefile (global L-BFGS
    history 5; reweight + refactorization every 10 iterations).  It times the
    ADMM iterations W..W+K-1 with K at most REF_TIMED_ITERS (one reweight and
    refactorization in every ten iterations, as in our arm's window) from its
    own accumulated_time_s (local + global + refactor, its MicroTimer)."""
    if rank != 0:
        return
    from oracle import pyoracle as po
    from wrapd_b200 import bars
    cores = os.cpu_count() or 1
    if not os.path.exists(po.QUASI_REF_M5):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/quasi_ref_m5 not built (no reference sources)"}))
        return
    bar = bars.bar_32x32x128_bent()
    W = max(0, args.warmup)
    K = max(1, min(args.steps, REF_TIMED_ITERS))
    with tempfile.TemporaryDirectory() as d:
        files = bars.write_bar(bar, d, "c1")
        t0 = time.perf_counter()
        r = po.run_quasi_ref(files, E_YOUNG, NU, W + K, threads=cores, extra=["-rw_every", "10"],
                             outdir=d + "/out", timeout=3000, binary=po.QUASI_REF_M5)
        wall = time.perf_counter() - t0
    acc = r["accumulated_time_s"]
    timed = float(acc[W + K] - acc[W])
    value = bar.n_tets * K / timed
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": 1, "steps": K,
        "steps_requested": args.steps,
        "warmup": W, "ms_per_step": 1000.0 * timed / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bar generator)",
        "config": {"workload": WORKLOAD, "solver": "reference quasi (Eigen SimplicialLDLT, OpenMP), L-BFGS history 5, "
                                                   "reweight+refactor every 10 iterations (patched build quasi_ref_m5)",
                   "timed": f"ADMM iterations {W}..{W + K - 1} from the reference's accumulated_time_s"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"the bent 32x32x128 bar, {W + K} ADMM iterations, iterations {W}..{W + K - 1} "
                                   f"timed; wall {wall:.1f} s for the whole run"},
        # e2e: the whole process (mesh files in, setup with AMD ordering and the
        # first factorizations, W + K iterations, files out), as our e2e leg is a
        # whole solve of W + K iterations from host buffers
        "e2e": {"value": bar.n_tets * (W + K) / wall, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "wall_s": wall,
                "includes": "quasi_ref process: load meshes + setup + W+K iterations + output files"},
    }
    print(json.dumps(line))


# ---- CPU baseline inside our arm -------------------------------------------------------
def cpu_baseline():
    """The reference on a bounded sample of the workload: a 32x32x16 slice of the bar
    (98,304 tets, same cross-section), 6 ADMM iterations, all host threads, the
    patched build with the benchmark's settings (no reweight falls in 6 iterations)."""
    from oracle import pyoracle as po
    from wrapd_b200 import bars
    cores = os.cpu_count() or 1
    bar = bars.make_bar(32, 32, 16, twist_deg=45.0, noise=0.01, seed=0)
    W, K = 1, 5
    with tempfile.TemporaryDirectory() as d:
        files = bars.write_bar(bar, d, "s")
        if os.path.exists(po.QUASI_REF_M5):
            r = po.run_quasi_ref(files, E_YOUNG, NU, W + K, threads=cores, extra=["-rw_every", "10"],
                                 outdir=d + "/out", timeout=600, binary=po.QUASI_REF_M5)
            acc = r["accumulated_time_s"]
            v = bar.n_tets * K / float(acc[W + K] - acc[W])
            return {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                    "sample": "32x32x16 slice of the bar (98,304 tets), iterations 1-5 of 6, history 5 "
                              "(quasi_ref_m5)"}
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU, max_iters=W + K)
    o.setup()
    o.iterate()
    t0 = time.perf_counter()
    for _ in range(K):
        o.iterate()
    v = bar.n_tets * K / (time.perf_counter() - t0)
    return {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "32x32x16 slice of the bar (98,304 tets), 5 iterations of the C oracle"}


# ---- time to energy gap --------------------------------------------------------------
FORMS = [
    ("plain_fp64", dict(precision="fp64", prox_mode=0)),        # the reference's method on the GPU
    ("fp64_newton", dict(precision="fp64", prox_mode=1)),
    ("fp32_newton", dict(precision="mixed", prox_mode=1)),
    ("learned_fp32", dict(precision="mixed", prox_mode=2)),     # network warm start, FP32 local step
]


# Iteration caps of the 3.9M-tet bar's runs (about 20 ms per FP64 iteration).
# With the 180 deg twist the runs converge (tol 1e-13) within the first cap.
# With the 720 deg twist and reweighting every 20 iterations (the configuration
# as specified) neither form reaches a 1e-6 gap in thousands of iterations:
# elements stay inverted while the bar unwinds (120 flips after 2,000 FP64
# iterations, the energy still falling by percents per hundred iterations), so
# that configuration is measured per iteration over the second cap.
GAP_ITERS_64x64x160 = 1500
PROGRESS_ITERS_64x64x160 = 300


def gap_time(objectives, acc_time_s, e_star, gap=1e-6):
    """Solver time (local + global + refactor, device events) at the first
    iterate from which (E_k - E*) / |E*| stays <= gap; None if never."""
    g = (np.asarray(objectives) - e_star) / abs(e_star)
    bad = np.nonzero(g > gap)[0]
    k = 0 if bad.size == 0 else int(bad[-1]) + 1
    if k >= len(g):
        return None, None
    return float(acc_time_s[k]), k


def time_to_gap(bar, label, device, base, e_star_iters=20000, gap=1e-6, forms=None):
    """E* = lowest energy of a long plain-FP64 run (tol 1e-13); then each form
    to convergence at tol 1e-13, reporting its time to the gap, iterations and
    the final positions' error against the plain FP64 run (which matches the
    FP64 oracle to 1e-8 in the parity tests)."""
    forms = FORMS if forms is None else [f for f in FORMS if f[0] in forms]
    from wrapd_b200 import prox_net
    from wrapd_b200.solver import Solver

    def run(kw):
        s = Solver(**dict(base, **kw, device=device))
        s.add_tetmesh(bar.rest, bar.init, bar.tets)
        s.set_pins(bar.pins)
        if kw.get("prox_mode") == 2:
            s.set_prox_net(prox_net.load_default())
        s.initialize()
        X = s.solve()
        d = s.algorithm_data()
        s.close()
        return X, d

    Xr, dr = run(dict(FORMS[0][1], tol=1e-13, max_iters=e_star_iters))
    e_star = float(dr.objectives.min())
    out = {"workload": label, "gap": gap, "e_star": e_star, "e_star_run_iters": int(len(dr.objectives) - 1),
           "time_source": "solver accumulated_time_s (CUDA events: local + global + refactor)", "forms": {}}
    for name, kw in forms:
        X, d = (Xr, dr) if name == "plain_fp64" else run(dict(kw, tol=1e-13, max_iters=e_star_iters))
        t, k = gap_time(d.objectives, d.accumulated_time_s, e_star, gap)
        out["forms"][name] = {
            "seconds_to_gap": t, "iterations_to_gap": k, "iterations_run": int(len(d.objectives) - 1),
            "final_rel_gap": float((d.objectives[-1] - e_star) / abs(e_star)),
            "x_err_vs_plain_fp64": float(np.abs(X - Xr).max() / np.abs(Xr).max()),
            "mean_prox_iters": float(np.mean(d.prox_iters)) if len(d.prox_iters) else None,
        }
    p0 = out["forms"]["plain_fp64"]["seconds_to_gap"]
    pl = out["forms"]["learned_fp32"]["seconds_to_gap"]
    out["speedup_learned_fp32_vs_plain_fp64"] = (p0 / pl) if (p0 and pl) else None
    return out


def capped_progress(bar, label, device, base, iters, forms):
    """Fixed-length runs of a configuration that does not converge within the
    bench's budget: per form the solver time per iteration (local / global /
    refactor), the energy and inverted elements after `iters` iterations, and
    the speed-up per iteration of each form over the plain FP64 one."""
    from wrapd_b200 import prox_net
    from wrapd_b200.solver import Solver
    out = {"workload": label, "iterations": iters, "gap_1e-6_reached": False, "forms": {}}
    for name, kw in [f for f in FORMS if f[0] in forms]:
        s = Solver(**dict(base, **kw, device=device, max_iters=iters, tol=0.0))
        s.add_tetmesh(bar.rest, bar.init, bar.tets)
        s.set_pins(bar.pins)
        if kw.get("prox_mode") == 2:
            s.set_prox_net(prox_net.load_default())
        s.initialize()
        s.solve()
        d, r = s.algorithm_data(), s.runtime()
        s.close()
        n = len(d.objectives) - 1
        out["forms"][name] = {"ms_per_iter": (r["local_ms"] + r["global_ms"] + r["refactor_ms"]) / n,
                              "local_ms_per_iter": r["local_ms"] / n, "global_ms_per_iter": r["global_ms"] / n,
                              "refactor_ms_per_iter": r["refactor_ms"] / n, "energy_start": float(d.objectives[0]),
                              "energy_end": float(d.objectives[-1]), "energy_min": float(d.objectives.min()),
                              "flips_end": int(d.flips[-1])}
    p0 = out["forms"]["plain_fp64"]["ms_per_iter"]
    for name, f in out["forms"].items():
        f["speedup_per_iter_vs_plain_fp64"] = p0 / f["ms_per_iter"]
    return out


def batch_throughput(device, K):
    """64 uneven bars (n_a, n_b in U{4..16}, n_L in U{8..64}, per-bar E and nu),
    FP32 local / FP64 global, solved as one batch (one handle: shared launches,
    each bar its own ADMM and L-BFGS decisions, a converged bar drops out) and
    one bar after another (64 handles); device time of K iterations after 2
    warm-up ones, setup excluded and reported apart.  Units are the element-
    iterations the bars actually ran (a bar that converged stops counting)."""
    from wrapd_b200 import bars
    from wrapd_b200.solver import Solver
    triples = bars.batch_bars(64, 0)
    ne_total = sum(b.n_tets for b, _, _ in triples)
    base = dict(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, max_iters=100000, precision="mixed", prox_mode=1,
                device=device)

    def run(group):
        t0 = time.perf_counter()
        s = Solver(**base)
        for b, E, nu in group:
            s.add_tetmesh(b.rest, b.init, b.tets, pins=b.pins, youngs=E, poisson=nu)
        s.initialize()
        s.begin_solve()
        setup = time.perf_counter() - t0
        s.iterate(2)
        n0 = [len(s.log("objectives", mesh=i)) for i in range(len(group))]
        r0 = s.runtime()
        done, _ = s.iterate(K)
        r1 = s.runtime()
        n1 = [len(s.log("objectives", mesh=i)) for i in range(len(group))]
        ms = sum(r1[k] - r0[k] for k in ("local_ms", "global_ms", "refactor_ms"))
        units = sum(g[0].n_tets * (b - a) for g, a, b in zip(group, n0, n1))
        its = [b - a for a, b in zip(n0, n1)]
        s.close()
        return ms, done, setup, units, its

    ms_b, done_b, setup_b, units_b, its_b = run(triples)
    ms_s, setup_s, units_s = 0.0, 0.0, 0
    for tr in triples:
        ms, done, setup, units, _ = run([tr])
        ms_s += ms
        setup_s += setup
        units_s += units
    return {"workload": "64 uneven bars (seeds 0-63), %d tets in total" % ne_total, "iterations": K,
            "per_bar_iterations_in_window": its_b,
            "batch_elem_iter_per_s": units_b / (ms_b / 1000.0), "batch_ms_per_iter": ms_b / max(1, done_b),
            "one_by_one_elem_iter_per_s": units_s / (ms_s / 1000.0),
            "batch_speedup": (units_b / ms_b) / (units_s / ms_s),
            "setup_s": {"batch": setup_b, "one_by_one": setup_s}}


# k_local<double>'s DRAM bytes per element and FP64-pipe share, from its
# one-launch ncu capture on the 32x32x64 bar (393,216 tets; the SoA streams
# scale with the element count).  They are copied here, not measured in this
# run: refresh them with that capture whenever the local step changes.
K_LOCAL_NCU = {"dram_bytes_per_elem": (105870080 + 39013120) / 393216, "fp64_pipe_active": 0.408,
               "source": "ncu --set full, one launch of k_local<double> on the 32x32x64 bar, traffic scaled by "
                         "the element count (copied constants, not measured in this run)"}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- our arm ------------------------------------------------------------------------------
def run_ours(args, rank, world, local, pg):
    from wrapd_b200 import bars, capi
    from wrapd_b200.solver import Solver
    import torch

    torch.cuda.set_device(local)
    bar = bars.bar_32x32x128_bent(seed=rank)
    settings = dict(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, rw_every=10, max_iters=100000,
                    precision=args.precision, device=local)
    s = Solver(**settings)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    s.begin_solve()
    for _ in range(args.warmup):
        s.iterate(1)
    rt0, c0 = s.runtime(), s.counters()
    K = args.steps
    barrier(pg)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record()
        done, _ = s.iterate(K)
        torch.cuda.synchronize()
        ev1.record()
        ev1.synchronize()
    barrier(pg)
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(pg, ms)
    ne, nf = bar.n_tets, bar.n_verts - len(bar.pins)
    units = sum_over_ranks(pg, float(ne * done))   # element-iterations of all replicas
    rt1, c1 = s.runtime(), s.counters()
    if done != K:
        raise RuntimeError(f"only {done} of {K} iterations ran")
    value = units / (ms / 1000.0)
    local_ms = rt1["local_ms"] - rt0["local_ms"]
    glob_ms = rt1["global_ms"] - rt0["global_ms"]
    ref_ms = rt1["refactor_ms"] - rt0["refactor_ms"]
    inner = rt1["inner_iters"] - rt0["inner_iters"]
    fp = 4 if args.precision == "mixed" else 8
    peak, peak_kind = peaks()
    # dominant element kernel: the local step (one launch per iteration, timed by
    # CUDA events on the library's stream around exactly that launch)
    lbytes = local_step_bytes(ne, fp)
    achieved = lbytes / (local_ms / K / 1000.0) / 1e9
    traffic = K_LOCAL_NCU["dram_bytes_per_elem"] * ne if args.precision == "fp64" else None
    # Secondary rooflines, from K more iterations with the per-phase device
    # timeline on (outside the timed region): the factorization against the
    # FP64 tensor-core peak measured here, the 3-RHS solve against HBM.
    info = s.info()
    p0, rp0, cp0 = s.profile(), s.runtime(), s.counters()
    s.set_profiling(True)
    s.iterate(K)
    s.set_profiling(False)
    p1, rp1, cp1 = s.profile(), s.runtime(), s.counters()
    n_solves = p1["solve"][1] - p0["solve"][1]
    solve_ms = (p1["solve"][0] - p0["solve"][0]) / max(1, n_solves)
    n_fact = cp1["factorizations"] - cp0["factorizations"]
    fact_ms = (rp1["refactor_ms"] - rp0["refactor_ms"]) / max(1, n_fact)
    dmma = capi.dmma_peak()
    solve_bytes = 16.0 * info["nnz_L"]   # [Y; W] read once forward and once backward, FP64
    solve_gbs = solve_bytes / (solve_ms / 1000.0) / 1e9
    fact_tflops = info["factor_flops"] / (fact_ms / 1000.0) / 1e12
    roof_solve = {"kernel": "k_fwd_queue + k_bwd_queue (3-RHS triangular solve, one queue launch per direction over all levels)", "bound": "hbm",
                  "achieved": solve_gbs, "peak": peak, "unit": "GB/s", "frac": solve_gbs / peak, "traffic": None,
                  "peak_source": peak_kind, "bytes_per_solve": solve_bytes, "ms_per_solve": solve_ms}
    roof_fact = {"kernel": "numeric factorization (k_panel, k_diag, k_trsm, k_update, k_wgemm; FP64 DMMA)",
                 "bound": "tensor", "achieved": fact_tflops, "peak": dmma, "unit": "TFLOP/s",
                 "frac": fact_tflops / dmma, "traffic": None,
                 "peak_source": "FP64 mma.sync m8n8k4 throughput measured on this GPU (wrapd_dmma_peak)",
                 "flops_per_factorization": info["factor_flops"], "ms_per_factorization": fact_ms}
    # e2e: a fresh solve through the C ABI from host buffers, setup included;
    # every rank solves its replica at once, the slowest rank's wall time counts
    parts = set(args.parts.split(","))
    e2e = None
    if "e2e" in parts:
        # three whole solves, the median wall time reported (the host setup runs
        # on a host shared with other jobs, so one sample varies from run to run)
        runs = []
        for _ in range(3):
            barrier(pg)
            t0 = time.perf_counter()
            s2 = Solver(**settings)
            s2.add_tetmesh(bar.rest, bar.init, bar.tets)
            s2.set_pins(bar.pins)
            s2.initialize()
            s2.begin_solve()
            done2, _ = s2.iterate(args.warmup + K)
            X = s2.positions()
            wall = time.perf_counter() - t0
            s2.close()
            if done2 != args.warmup + K or not np.isfinite(X).all():
                raise RuntimeError("the end-to-end solve did not run its iterations to finite positions")
            runs.append(max_over_ranks(pg, wall))
        e2e_s = float(np.median(runs))
        e2e_units = sum_over_ranks(pg, float(ne * done2))
        h2d = bar.rest.nbytes + bar.init.nbytes + bar.tets.nbytes + bar.pins.nbytes
        n_e2e = args.warmup + K
        e2e = {"value": e2e_units / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d // n_e2e),
               "d2h_bytes_per_step": int(X.nbytes // n_e2e), "wall_s": e2e_s, "wall_s_runs": runs,
               "iterations": n_e2e,
               "includes": "a whole solve through the C ABI from host buffers: create + add_tetmesh + initialize "
                           "(symbolic analysis + first factorization) + begin_solve + W+K iterations + positions "
                           "out, on every rank at once; the median of three such solves (the reference arm's e2e "
                           "is its whole process for the same W+K iterations)"}
    # the learned/FP32 form on the same bar: local step (FP32 SVD + network-started Newton)
    learned = None
    if rank == 0 and world == 1 and "learned" in parts:
        from wrapd_b200 import prox_net
        s3 = Solver(**dict(settings, precision="mixed", prox_mode=2))
        s3.add_tetmesh(bar.rest, bar.init, bar.tets)
        s3.set_pins(bar.pins)
        s3.set_prox_net(prox_net.load_default())
        s3.initialize()
        s3.begin_solve()
        s3.iterate(args.warmup)
        r0 = s3.runtime()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s3.iterate(K)
        wall = time.perf_counter() - t0
        r1 = s3.runtime()
        lms = r1["local_ms"] - r0["local_ms"]
        tot = sum(r1[k] - r0[k] for k in ("local_ms", "global_ms", "refactor_ms"))
        learned = {"ms_per_step": tot / K, "local_ms_per_step": lms / K,
                   "local_elems_per_s": ne * K / (lms / 1000.0), "elem_iter_per_s": ne * K / (tot / 1000.0),
                   "wall_ms_per_step": 1000.0 * wall / K,
                   "mean_prox_iters": float(np.mean(s3.log("prox_iters")[-K:]))}
        s3.close()
    gap = None
    if rank == 0 and world == 1 and "gap" in parts:
        # the 8x8x32 bar, and a 786,432-tet bar with the same 180 deg twist (no
        # bend): the bent bar keeps inverted elements and its energy does
        # not settle to a 1e-6 gap
        base = dict(youngs=E_YOUNG, poisson=NU, lbfgs_m=5)
        gap = {"bar_8x8x32": time_to_gap(bars.bar_8x8x32(), "bar 8x8x32 cubes x6 tets (12,288 tets), 180 deg twist, "
                                         "E=1e5 nu=0.45", local, base),
               "bar_32x32x128": time_to_gap(bars.make_bar(32, 32, 128, twist_deg=180.0, noise=0.02, seed=0),
                                            "bar 32x32x128 cubes x6 tets (786,432 tets), 180 deg twist, E=1e5 "
                                            "nu=0.45", local, base, e_star_iters=4000),
               # the headline size, 3.9M tets: with a 180 deg twist it converges ...
               "bar_64x64x160_180deg": time_to_gap(bars.make_bar(64, 64, 160, twist_deg=180.0, noise=0.005,
                                                                 seed=0),
                                                   "bar 64x64x160 cubes x6 tets (3,932,160 tets), 180 deg twist, "
                                                   "E=1e5 nu=0.45", local, base, e_star_iters=GAP_ITERS_64x64x160,
                                                   forms=("plain_fp64", "fp32_newton", "learned_fp32")),
               # ... with the specified 720 deg twist and reweighting every 20 it does not
               "bar_64x64x160": capped_progress(bars.bar_64x64x160(),
                                                "bar 64x64x160 cubes x6 tets (3,932,160 tets), 720 deg twist, E=1e5 "
                                                "nu=0.45, reweight+refactor every 20", local,
                                                dict(base, rw_every=20), PROGRESS_ITERS_64x64x160,
                                                ("plain_fp64", "fp32_newton", "learned_fp32"))}
    batch = None
    if rank == 0 and world == 1 and "batch" in parts:
        batch = batch_throughput(local, min(K, 20))
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": args.warmup,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-local/f64-global",
            "data": "synthetic (seeded bar generator, seed = rank)",
            "config": {"workload": "bar 32x32x128 cubes x6 tets (786,432 tets, 140,481 verts), 360 deg twist "
                                   "+ 90 deg bend, E=1e5 nu=0.45",
                       "solver": f"ADMM, L-BFGS history 5, reweight+refactor every 10 iterations, {args.precision}",
                       "parallelism": f"replicas x{world}", "l2": "inputs > L2 (element state ~0.7 GB)"},
            "local_elems_per_s": world * ne * K / (local_ms / 1000.0),
            "phase_ms_per_step": {"local": local_ms / K, "global": glob_ms / K, "refactor": ref_ms / K},
            "inner_iters_per_step": inner / K,
            "learned_fp32_same_bar": learned,
            "time_to_gap": gap,
            "batch_64_bars": batch,
            "roofline": {"kernel": "k_local (fused local step)", "bound": "hbm", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind, "bytes_per_launch": lbytes,
                         "fp64_pipe_active_ncu": K_LOCAL_NCU["fp64_pipe_active"],
                         "traffic_source": K_LOCAL_NCU["source"],
                         "note": "FP64-arithmetic-bound (Jacobi SVD + L-BFGS prox per element); the HBM "
                                 "fraction is low by design"},
            "roofline_solve": roof_solve,
            "roofline_factorization": roof_fact,
            "gpu_launches": int(c1["kernel_launches"] - c0["kernel_launches"]),
            "factorizations": int(c1["factorizations"] - c0["factorizations"]),
            "clocks": clk.summary(),
            "e2e": e2e,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    s.close()


def main():
    args = parse()
    if args.impl == "reference":
        # the reference's CPU solver: rank 0 alone runs it (no process group);
        # the other ranks of a multi-GPU launch exit without work
        run_reference(args, int(os.environ.get("RANK", "0")))
        return
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        run_ours(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.barrier()
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
