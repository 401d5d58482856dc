"""Prox-stretch network: harvesting, GPU training and inference.

The network (include/wrapd_gpu.h, wrapd_net_*) predicts the converged prox
stretches of NHProx (src/TetElements.hpp:50-162) from the prox inputs of one
element, and warm-starts the Newton prox of the local step under prox_mode 2.
Everything numeric runs on the GPU through the C ABI:

* ``harvest`` runs the FP64 solver on seeded small bars (8 x 8 x 32 cubes x 6
  tets, twist uniform in [0, 540] degrees, Poisson ratio uniform in
  [0.3, 0.49]) and, every few iterations, records for a random subset of
  elements the inputs of the next local step (singular values of
  S_in = symF + U, w^2 / vol) and the prox solution converged by the Newton
  prox to 1e-10 from the solver's own warm start.
* ``Trainer`` wraps the training kernels (BF16 operands, FP32 accumulation,
  Adam, deterministic per seed).
* ``predict`` runs the inference kernel the local step inlines.

``python -m wrapd_b200.prox_net --out PATH`` harvests, trains and writes the
blob (``.npy``); ``load_default`` reads the blob shipped with the package.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

import numpy as np

from . import bars, capi
from .capi import WrapdError

N_BLOB = capi.NET_BLOB
IN, HID, OUT = 5, 64, 3
B_W1 = 16
DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "prox_net.npy")


def lame(youngs: float, poisson: float):
    """Lame parameters (src/Lame.hpp:50-53)."""
    return youngs / (2.0 * (1.0 + poisson)), youngs * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson))


def features(sig, wov, mu, lam) -> np.ndarray:
    """Raw network inputs (n x 5, float32): sorted singular values of S_in,
    log(w^2 / (vol mu)), log(mu / lambda)."""
    sig = np.asarray(sig, dtype=np.float64).reshape(-1, 3)
    f = np.empty((sig.shape[0], IN), dtype=np.float32)
    f[:, :3] = sig
    f[:, 3] = np.log(np.asarray(wov, dtype=np.float64).ravel() / mu)
    f[:, 4] = np.log(mu / lam)
    return f


def init_blob(X: np.ndarray, T: np.ndarray, seed: int = 0) -> np.ndarray:
    """A fresh blob: normalisation from the data, He-normal weights, zero biases."""
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    rng = np.random.default_rng(seed)
    b = np.zeros(N_BLOB, dtype=np.float32)
    mean, std = X.mean(axis=0), X.std(axis=0)
    std[std < 1e-6] = 1.0
    b[0:5] = mean
    b[5:10] = 1.0 / std
    osc = (T - X[:, :3]).std(axis=0)
    osc[osc < 1e-6] = 1.0
    b[10:13] = osc
    o = B_W1
    b[o:o + HID * IN] = rng.normal(0.0, np.sqrt(2.0 / IN), HID * IN)
    o += HID * IN + HID
    b[o:o + HID * HID] = rng.normal(0.0, np.sqrt(2.0 / HID), HID * HID)
    o += HID * HID + HID
    b[o:o + OUT * HID] = rng.normal(0.0, np.sqrt(1.0 / HID), OUT * HID)
    return b


class Trainer:
    """Device-resident training state (wrapd_net_create ... wrapd_net_destroy)."""

    def __init__(self, blob):
        self.lib = capi.load()
        b = np.ascontiguousarray(blob, dtype=np.float32)
        if b.size != N_BLOB:
            raise ValueError(f"blob must have {N_BLOB} floats")
        h = ctypes.c_void_p()
        rc = self.lib.wrapd_net_create(capi.fptr(b), N_BLOB, ctypes.byref(h))
        if rc != 0:
            raise WrapdError(rc, self.lib.wrapd_net_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != 0:
            raise WrapdError(rc, self.lib.wrapd_net_last_error(self.h).decode())

    def set_data(self, X, T):
        self.X = np.ascontiguousarray(X, dtype=np.float32).reshape(-1, IN)
        self.T = np.ascontiguousarray(T, dtype=np.float32).reshape(-1, 3)
        self._check(self.lib.wrapd_net_set_data(self.h, capi.fptr(self.X), capi.fptr(self.T), self.X.shape[0]))

    def train(self, epochs: int, batch: int = 4096, lr: float = 2e-3, lr_end: float = 1e-5, seed: int = 0):
        losses = np.zeros(epochs)
        self._check(self.lib.wrapd_net_train(self.h, epochs, batch, lr, lr_end, seed, capi.dptr(losses)))
        return losses

    def grad(self, first: int, n: int):
        g = np.empty(N_BLOB - B_W1, dtype=np.float32)
        loss = ctypes.c_double(0.0)
        self._check(self.lib.wrapd_net_grad(self.h, first, n, ctypes.byref(loss), capi.fptr(g)))
        return loss.value, g

    def blob(self) -> np.ndarray:
        b = np.empty(N_BLOB, dtype=np.float32)
        self._check(self.lib.wrapd_net_get(self.h, capi.fptr(b)))
        return b

    def close(self):
        if getattr(self, "h", None):
            self.lib.wrapd_net_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def predict(blob, sig, wov, mu: float, lam: float) -> np.ndarray:
    """Predicted prox stretches (n x 3) from the inference kernel."""
    b = np.ascontiguousarray(blob, dtype=np.float32)
    s = np.ascontiguousarray(sig, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(wov, dtype=np.float64).ravel()
    out = np.empty_like(s)
    lib = capi.load()
    rc = lib.wrapd_net_predict(capi.fptr(b), b.size, s.shape[0], capi.dptr(s), capi.dptr(w), mu, lam, capi.dptr(out))
    if rc != 0:
        raise WrapdError(rc, lib.wrapd_net_last_error(None).decode())
    return out


def load_default() -> np.ndarray:
    """The trained blob shipped with the package."""
    b = np.load(DEFAULT_PATH).astype(np.float32)
    if b.size != N_BLOB:
        raise ValueError(f"{DEFAULT_PATH}: expected {N_BLOB} floats")
    return b


def prox_inputs(solver):
    """Inputs of the next local step of a solver: (sigma_in n x 3, wov n,
    last stretches n x 3), from its device state."""
    symF = solver.get_state("symF").reshape(-1, 9)
    U = solver.get_state("U").reshape(-1, 9)
    w2 = solver.get_state("w2")
    vol = solver.get_state("vol")
    slast = solver.get_state("slast").reshape(-1, 3)
    sig, _, _ = capi.svd3_batch(symF + U)
    return sig, w2 / vol, slast


def _harvest_run(seed: int):
    """Twist angle and Poisson ratio of one harvesting run (seeded)."""
    u = bars.uniform01(0x5EED0000 + seed, 2)
    return 540.0 * float(u[0]), 0.3 + 0.19 * float(u[1])


def harvest(runs: int = 200, seed0: int = 1000, every: int = 4, per_snapshot: int = 1024, max_iters: int = 500,
            youngs: float = 1e5, tol: float = 1e-10, sample_seed: int = 0, log=None):
    """(features n x 5 float32, targets n x 3 float32) from `runs` seeded solves."""
    from .solver import Solver

    rng = np.random.default_rng(sample_seed)
    Xs, Ts = [], []
    for r in range(runs):
        seed = seed0 + r
        twist, nu = _harvest_run(seed)
        mu, lam = lame(youngs, nu)
        bar = bars.make_bar(8, 8, 32, twist_deg=twist, bend_deg=0.0, noise=0.02, seed=seed)
        s = Solver(youngs=youngs, poisson=nu, lbfgs_m=5, max_iters=max_iters, prox_mode=1)
        s.add_tetmesh(bar.rest, bar.init, bar.tets)
        s.set_pins(bar.pins)
        s.initialize()
        s.begin_solve()
        it, snaps = 0, 0
        while it < max_iters:
            sig, wov, slast = prox_inputs(s)
            pick = rng.choice(sig.shape[0], size=min(per_snapshot, sig.shape[0]), replace=False)
            out, its = capi.prox_newton_batch(mu, lam, sig[pick], wov[pick], slast[pick], tol=tol, max_iters=100)
            ok = (its < 100) & np.all(np.isfinite(out), axis=1) & np.all(out > 0.0, axis=1)
            Xs.append(features(sig[pick][ok], wov[pick][ok], mu, lam))
            Ts.append(out[ok].astype(np.float32))
            snaps += 1
            done, conv = s.iterate(every)
            it += done
            if conv or done < every:
                break
        s.close()
        if log:
            log(f"run {r}: seed {seed} twist {twist:.1f} nu {nu:.3f} iters {it} snapshots {snaps}")
    return np.concatenate(Xs), np.concatenate(Ts)


def newton_iterations(blob, sig, wov, slast, mu, lam, tol: float = 1e-10):
    """Newton prox iterations to `tol` from identity, from the last stretches
    and from the network's prediction (each an n-vector), plus the solutions."""
    ones = np.ones_like(sig)
    out_i, it_i = capi.prox_newton_batch(mu, lam, sig, wov, ones, tol=tol, max_iters=100)
    out_l, it_l = capi.prox_newton_batch(mu, lam, sig, wov, slast, tol=tol, max_iters=100)
    pred = predict(blob, sig, wov, mu, lam)
    out_n, it_n = capi.prox_newton_batch(mu, lam, sig, wov, pred, tol=tol, max_iters=100)
    return dict(identity=it_i, last=it_l, network=it_n, out_identity=out_i, out_last=out_l, out_network=out_n,
                prediction=pred)


def main(argv=None):
    ap = argparse.ArgumentParser(description="harvest prox pairs, train the prox network on the GPU")
    ap.add_argument("--out", required=True, help="blob output (.npy)")
    ap.add_argument("--runs", type=int, default=200)
    ap.add_argument("--every", type=int, default=4)
    ap.add_argument("--per-snapshot", type=int, default=1024)
    ap.add_argument("--max-pairs", type=int, default=10_000_000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--report", default=None, help="JSON summary output")
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    X, T = harvest(a.runs, every=a.every, per_snapshot=a.per_snapshot, log=print)
    if X.shape[0] > a.max_pairs:
        keep = np.random.default_rng(a.seed).choice(X.shape[0], a.max_pairs, replace=False)
        X, T = X[keep], T[keep]
    t1 = time.perf_counter()
    print(f"harvested {X.shape[0]} pairs in {t1 - t0:.1f} s", flush=True)
    n_val = min(200_000, X.shape[0] // 10)
    Xv, Tv, Xt, Tt = X[:n_val], T[:n_val], X[n_val:], T[n_val:]
    tr = Trainer(init_blob(Xt, Tt, a.seed))
    tr.set_data(Xt, Tt)
    losses = tr.train(a.epochs, a.batch, a.lr, 1e-5, a.seed)
    t2 = time.perf_counter()
    blob = tr.blob()
    tr.set_data(Xv, Tv)
    vloss, _ = tr.grad(0, min(n_val, 65536))
    print("epoch losses", losses.tolist(), "validation loss", vloss, f"train {t2 - t1:.1f} s", flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    np.save(a.out, blob)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(dict(pairs=int(X.shape[0]), harvest_s=t1 - t0, train_s=t2 - t1, epochs=a.epochs,
                           batch=a.batch, lr=a.lr, epoch_losses=losses.tolist(), validation_loss=vloss), f, indent=1)


if __name__ == "__main__":
    main()
