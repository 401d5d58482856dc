"""Measurement tool (not part of the solver's API): a self-contained solve
for kernel profiles and size reports, one bar, a few ADMM iterations through
the C ABI.  The commands recorded in profiles/ run it under ncu.

    python -m wrapd_b200.profile_case [--grid 32 32 64] [--iters 2]
        [--precision fp64|mixed] [--prox-mode 0|1|2]
    python -m wrapd_b200.profile_case --bar 64x64x160 --rw-every 20 --warmup 2 --iters 20 --report
    python -m wrapd_b200.profile_case --net 1000000

The default 32x32x64 bar holds ~0.2 GB of element state (larger than the
126 MB L2) and ~1.5 GB on the device in total, so a profiler capture of one
launch stays small.  ``--bar 32x32x128-bent|64x64x160`` takes the 786,432-tet or the
3,932,160-tet bar instead.  ``--report`` prints one JSON line: device memory
held by the solver (cudaMemGetInfo before create minus after initialize),
setup time, and per-iteration local/global/refactor milliseconds over the
``--iters`` iterations that follow ``--warmup`` ones.  ``--net N`` instead
runs the prox network's kernels on N seeded synthetic samples: one training
epoch (batch 4096) from the shipped blob, then one inference pass.
"""
from __future__ import annotations

import argparse
import json
import time

from . import bars, capi, prox_net
from .solver import Solver


def device_free_bytes() -> int:
    """Free device memory (cudaMemGetInfo through torch)."""
    import torch
    return torch.cuda.mem_get_info()[0]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[32, 32, 64])
    ap.add_argument("--bar", choices=["grid", "32x32x128-bent", "64x64x160"], default="grid")
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=0)
    ap.add_argument("--rw-every", type=int, default=10)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--prox-mode", type=int, default=0)
    ap.add_argument("--report", action="store_true")
    ap.add_argument("--net", type=int, default=0)
    a = ap.parse_args(argv)
    if a.net:
        import numpy as np
        rng = np.random.default_rng(0)
        mu, lam = prox_net.lame(1e5, 0.45)
        sig = np.sort(rng.uniform(0.5, 1.5, (a.net, 3)), axis=1)[:, ::-1].copy()
        wov = 10.0 ** rng.uniform(3.0, 6.0, a.net)
        X = np.column_stack([sig, np.log(wov / mu), np.full(a.net, np.log(mu / lam))]).astype(np.float32)
        T = (sig + 0.01 * rng.standard_normal(sig.shape)).astype(np.float32)
        tr = prox_net.Trainer(prox_net.load_default())
        tr.set_data(X, T)
        losses = tr.train(epochs=1, batch=4096, lr=1e-4, lr_end=1e-5, seed=1)
        out = prox_net.predict(tr.blob(), sig, wov, mu, lam)
        tr.close()
        print(f"net samples {a.net} loss {losses[0]:.3e} predicted {out.shape[0]} finite {bool(np.isfinite(out).all())}")
        return
    if a.bar == "32x32x128-bent":
        bar = bars.bar_32x32x128_bent()
    elif a.bar == "64x64x160":
        bar = bars.bar_64x64x160()
    else:
        na, nb, nl = a.grid
        bar = bars.make_bar(na, nb, nl, twist_deg=360.0 * nl / 128.0, bend_deg=90.0 * nl / 128.0, noise=0.01,
                            seed=0)
    if a.report:
        capi.load()
        free0 = device_free_bytes()
    t0 = time.perf_counter()
    s = Solver(youngs=1e5, poisson=0.45, lbfgs_m=5, rw_every=a.rw_every, max_iters=100000,
               precision=a.precision, prox_mode=a.prox_mode)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    if a.prox_mode == 2:
        s.set_prox_net(prox_net.load_default())
    s.initialize()
    if a.report:
        import torch
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        free1 = device_free_bytes()
    s.begin_solve()
    if a.warmup:
        s.iterate(a.warmup)
    r0, c0 = s.runtime(), s.counters()
    done, _ = s.iterate(a.iters)
    r1, c1 = s.runtime(), s.counters()
    if a.report:
        ms = {k: (r1[k] - r0[k]) / max(1, done) for k in ("local_ms", "global_ms", "refactor_ms")}
        ms["total"] = sum(ms.values())
        print(json.dumps({"tets": bar.n_tets, "verts": bar.n_verts, "precision": a.precision,
                          "prox_mode": a.prox_mode, "device_gb": (free0 - free1) / 1e9, "setup_s": setup_s,
                          "iterations": done, "ms_per_iter": ms,
                          "inner_per_iter": (r1["inner_iters"] - r0["inner_iters"]) / max(1, done),
                          "factorizations": c1["factorizations"] - c0["factorizations"], "info": s.info()}))
    else:
        print(f"tets {bar.n_tets} iterations {done} runtime {s.runtime()}")
    s.close()


if __name__ == "__main__":
    main()
