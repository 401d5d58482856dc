"""The allocation-free energy entry point against the allocating one.

wrapd_potential_energy_batch_noalloc serves callers that may not allocate
device memory (an application that owns all GPU memory through its own
allocator, or a loop that must not call cudaMalloc after start-up).  It takes
device pointers from the caller and keeps its reduction scratch in a fixed
array inside the library, which persists between calls; two calls in a row
check that nothing left over from the first call leaks into the second.  This
file is collected last so that a failure here stops a -x run only after every
other test has run.
"""
import ctypes

import numpy as np
import pytest

from conftest import E_YOUNG, NU

pytestmark = pytest.mark.gpu

MAX_N = 65536 * 256


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    sig = np.abs(rng.normal(1.0, 0.3, size=(n, 3)))
    sig[::89, 1] *= -1.0
    sig[3::41] = rng.uniform(0.05, 0.3, size=sig[3::41].shape)
    vol = rng.uniform(1e-4, 1e-3, size=n)
    return sig, vol


def test_no_alloc_energy_matches_the_allocating_entry(lib_built):
    import torch
    from oracle import pyoracle as po
    from wrapd_b200 import capi

    lib = capi.load()
    mu, lam = po.lame(E_YOUNG, NU)
    # two calls in a row on different batches: the shared scratch and its block
    # counter keep the first call's contents when the second one starts
    for n, seed in ((300_007, 1), (65_537, 2)):
        sig, vol = _inputs(n, seed)
        pe_ref, flips_ref = capi.potential_energy_batch(mu, lam, sig, vol)
        d_sig = torch.from_numpy(sig).cuda()
        d_vol = torch.from_numpy(vol).cuda()
        d_out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.wrapd_potential_energy_batch_noalloc(n, mu, lam, ctypes.c_void_p(d_sig.data_ptr()),
                                                      ctypes.c_void_p(d_vol.data_ptr()),
                                                      ctypes.c_void_p(d_out.data_ptr()), None)
        assert rc == capi.WRAPD_OK
        torch.cuda.synchronize()
        pe, flips = d_out.cpu().numpy()
        assert pe == pytest.approx(pe_ref, rel=1e-12)
        assert int(flips) == flips_ref
    # sizes beyond the fixed scratch are refused, without touching the output
    d_out = torch.full((2,), 7.0, dtype=torch.float64, device="cuda")
    rc = lib.wrapd_potential_energy_batch_noalloc(MAX_N + 1, mu, lam, ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == capi.WRAPD_E_INPUT
    torch.cuda.synchronize()
    assert d_out.cpu().tolist() == [7.0, 7.0]


def test_no_alloc_energy_empty_batch_and_own_stream(lib_built):
    """n == 0 writes zeros; a call queued on the caller's own stream is ready
    once that stream has reached it."""
    import torch
    from oracle import pyoracle as po
    from wrapd_b200 import capi

    lib = capi.load()
    mu, lam = po.lame(E_YOUNG, NU)
    d_out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert lib.wrapd_potential_energy_batch_noalloc(0, mu, lam, None, None, ctypes.c_void_p(d_out.data_ptr()),
                                                    None) == capi.WRAPD_OK
    torch.cuda.synchronize()
    assert d_out.cpu().tolist() == [0.0, 0.0]
    sig, vol = _inputs(100_003, 3)
    pe_ref, flips_ref = capi.potential_energy_batch(mu, lam, sig, vol)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        d_sig = torch.from_numpy(sig).cuda()
        d_vol = torch.from_numpy(vol).cuda()
        d_out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.wrapd_potential_energy_batch_noalloc(sig.shape[0], mu, lam, ctypes.c_void_p(d_sig.data_ptr()),
                                                  ctypes.c_void_p(d_vol.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.c_void_p(stream.cuda_stream))
    assert rc == capi.WRAPD_OK
    stream.synchronize()
    pe, flips = d_out.cpu().numpy()
    assert pe == pytest.approx(pe_ref, rel=1e-12)
    assert int(flips) == flips_ref
