"""The prox network's CPU oracle (oracle/net_oracle.py) checked on its own:
the BF16 rounding against known bit patterns, the float64 backward pass
against central finite differences, and the blob layout against the C header."""
import os
import re

import numpy as np

from conftest import ROOT
from oracle import net_oracle as no


def test_bf16_rounding():
    # BF16 keeps 7 mantissa bits: one unit in the last place at 1 is 2^-7
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 0.0],
                 dtype=np.float32)
    # half-way cases go to the even neighbour
    np.testing.assert_array_equal(no.bf16(x), [1.0, 1.0, 1.0 + 2 ** -6, 1.0 + 2 ** -7, 1.0, -2.5, 0.0])


def test_blob_layout_matches_header():
    h = open(os.path.join(ROOT, "include", "wrapd_gpu.h")).read()
    assert int(re.search(r"#define WRAPD_NET_BLOB (\d+)", h).group(1)) == no.N_BLOB == 4755
    assert no.N_TRAIN == 5 * 64 + 64 + 64 * 64 + 64 + 3 * 64 + 3


def _random_case(seed, n=40):
    rng = np.random.default_rng(seed)
    blob = rng.normal(0.0, 0.3, no.N_BLOB)
    blob[0:5] = [1.0, 0.9, 0.8, 0.5, -1.5]
    blob[5:10] = [3.0, 3.0, 3.0, 0.7, 2.0]
    blob[10:13] = [0.05, 0.04, 0.06]
    blob[13:16] = 0.0
    X = np.column_stack([rng.uniform(0.6, 1.4, (n, 3)), rng.normal(0.5, 1.0, n), np.full(n, -1.5)])
    T = X[:, :3] + rng.normal(0.0, 0.05, (n, 3))
    return blob, X, T


def test_backward_matches_finite_differences():
    blob, X, T = _random_case(1)
    loss, g = no.loss_grad(blob, X, T, bf=False)
    rng = np.random.default_rng(2)
    idx = rng.choice(no.N_TRAIN, 60, replace=False)
    h = 1e-6
    for i in idx:
        bp, bm = blob.copy(), blob.copy()
        bp[no.B_W1 + i] += h
        bm[no.B_W1 + i] -= h
        fd = (no.loss_grad(bp, X, T, bf=False)[0] - no.loss_grad(bm, X, T, bf=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


def test_bf16_forward_close_to_float64():
    blob, X, _ = _random_case(3)
    y64, _ = no.forward(blob, X, bf=False)
    y16, _ = no.forward(blob, X, bf=True)
    # BF16 operands: ~3 significant digits per product
    assert np.abs(y16 - y64).max() <= 0.05 * max(1.0, np.abs(y64).max())
