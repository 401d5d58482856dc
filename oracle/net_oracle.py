"""CPU oracle of the prox-stretch network (test infrastructure only).

A numpy restatement of the network the CUDA kernels train and run
(wrapd_b200/csrc/prox_net.cuh, prox_net.cu): 5 -> 64 -> 64 -> 3 with GELU
(tanh form), BF16 operands and wide accumulation.  The BF16 rounding points of
the kernels are reproduced (round to nearest even), so a float64 evaluation
here differs from the kernels only by their FP32 accumulation order; with
``bf16=False`` it is the plain float64 network, used to check the backward
pass against finite differences.

The network has no counterpart in the reference: the reference warm-starts
its prox from the last stretches (src/TetElements.cpp:313-315).  Blob layout
and loss are those of include/wrapd_gpu.h (wrapd_net_*).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 5, 64, 3
B_MEAN, B_ISTD, B_OSCALE = 0, 5, 10
B_W1 = 16
B_B1 = B_W1 + HID * IN
B_W2 = B_B1 + HID
B_B2 = B_W2 + HID * HID
B_W3 = B_B2 + HID
B_B3 = B_W3 + OUT * HID
N_BLOB = B_B3 + OUT
N_TRAIN = N_BLOB - B_W1
GELU_C = np.sqrt(2.0 / np.pi)
GELU_A = 0.044715


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + GELU_A * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_C * (x + GELU_A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * x * x)


def unpack(blob):
    b = np.asarray(blob, dtype=np.float64)
    return dict(mean=b[B_MEAN:B_MEAN + IN], istd=b[B_ISTD:B_ISTD + IN], oscale=b[B_OSCALE:B_OSCALE + 3],
                W1=b[B_W1:B_B1].reshape(HID, IN), b1=b[B_B1:B_W2], W2=b[B_W2:B_B2].reshape(HID, HID),
                b2=b[B_B2:B_W3], W3=b[B_W3:B_B3].reshape(OUT, HID), b3=b[B_B3:N_BLOB])


def features(sig, wov, mu, lam):
    """Raw features: sorted singular values, log(wov / mu), log(mu / lambda)."""
    sig = np.asarray(sig, dtype=np.float64).reshape(-1, 3)
    n = sig.shape[0]
    f = np.empty((n, IN))
    f[:, :3] = sig
    f[:, 3] = np.log(np.asarray(wov, dtype=np.float64).ravel() / mu)
    f[:, 4] = np.log(mu / lam)
    return f


def _r(x, on):
    return bf16(x) if on else np.asarray(x, dtype=np.float64)


def forward(blob, X, bf=True):
    """Normalised outputs y (n x 3) and the cache for backward.  X: raw features."""
    p = unpack(blob)
    X = np.asarray(X, dtype=np.float64)
    xn = _r((X.astype(np.float32) - p["mean"].astype(np.float32)) * p["istd"].astype(np.float32), bf) if bf else \
        (X - p["mean"]) * p["istd"]
    W1, W2, W3 = _r(p["W1"], bf), _r(p["W2"], bf), _r(p["W3"], bf)
    z1 = xn @ W1.T + p["b1"]
    h1 = _r(gelu(z1), bf)
    z2 = h1 @ W2.T + p["b2"]
    h2 = _r(gelu(z2), bf)
    y = h2 @ W3.T + p["b3"]
    return y, dict(xn=xn, z1=z1, h1=h1, z2=z2, h2=h2, W2=W2, W3=W3)


def predict(blob, sig, wov, mu, lam, bf=True):
    """Predicted prox stretches: sigma_in + oscale * y."""
    p = unpack(blob)
    y, _ = forward(blob, features(sig, wov, mu, lam), bf)
    return np.asarray(sig, dtype=np.float64).reshape(-1, 3) + p["oscale"] * y


def loss_grad(blob, X, T, bf=True):
    """Mean squared error of the normalised output and its gradient with
    respect to the trained part of the blob (N_TRAIN values, blob order).
    T: converged prox stretches (n x 3)."""
    p = unpack(blob)
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    tn = (np.asarray(T, dtype=np.float64) - X[:, :3]) / p["oscale"]
    y, c = forward(blob, X, bf)
    e = y - tn
    loss = float(np.sum(e * e) / (3.0 * n))
    dy = 2.0 * e / (3.0 * n)
    dyb = _r(dy, bf)
    dz2 = (dyb @ c["W3"]) * gelu_grad(c["z2"])
    dz2b = _r(dz2, bf)
    dz1 = (dz2b @ c["W2"]) * gelu_grad(c["z1"])
    dz1b = _r(dz1, bf)
    g = np.empty(N_TRAIN)
    o = -B_W1
    g[B_W1 + o:B_B1 + o] = (dz1b.T @ c["xn"]).ravel()
    g[B_B1 + o:B_W2 + o] = dz1.sum(axis=0)
    g[B_W2 + o:B_B2 + o] = (dz2b.T @ c["h1"]).ravel()
    g[B_B2 + o:B_W3 + o] = dz2.sum(axis=0)
    g[B_W3 + o:B_B3 + o] = (dyb.T @ c["h2"]).ravel()
    g[B_B3 + o:N_BLOB + o] = dy.sum(axis=0)
    return loss, g
