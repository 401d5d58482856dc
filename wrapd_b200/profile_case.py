"""A small, self-contained solve for kernel profiles: one bar, a few ADMM
iterations through the C ABI.  Sized so that a profiler capture of one launch
stays small (the default 32x32x64 bar holds ~0.2 GB of element state, larger
than the 126 MB L2, and well under a few GB on the device in total).

    python -m wrapd_b200.profile_case [--grid 32 32 64] [--iters 2]
        [--precision fp64|mixed] [--prox-mode 0|1|2]
"""
from __future__ import annotations

import argparse

from . import bars, prox_net
from .solver import Solver


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, nargs=3, default=[32, 32, 64])
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--prox-mode", type=int, default=0)
    a = ap.parse_args(argv)
    na, nb, nl = a.grid
    bar = bars.make_bar(na, nb, nl, twist_deg=360.0 * nl / 128.0, bend_deg=90.0 * nl / 128.0, noise=0.01, seed=0)
    s = Solver(youngs=1e5, poisson=0.45, lbfgs_m=5, rw_every=10, max_iters=a.iters, precision=a.precision,
               prox_mode=a.prox_mode)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    if a.prox_mode == 2:
        s.set_prox_net(prox_net.load_default())
    s.initialize()
    s.begin_solve()
    done, _ = s.iterate(a.iters)
    print(f"tets {bar.n_tets} iterations {done} runtime {s.runtime()}")
    s.close()


if __name__ == "__main__":
    main()
