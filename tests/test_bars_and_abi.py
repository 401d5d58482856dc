"""CPU checks: the synthetic bar generator and the C ABI library's surface."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from wrapd_b200 import bars


def _volumes(bar):
    P = bar.rest[bar.tets]
    return np.einsum("ij,ij->i", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0])) / 6.0


@pytest.mark.parametrize("dims,nv,nt,npins", [((8, 8, 32), 2673, 12288, 162), ((2, 3, 5), 72, 180, 24)])
def test_bar_counts_and_volumes(dims, nv, nt, npins):
    b = bars.make_bar(*dims)
    assert (b.n_verts, b.n_tets, len(b.pins)) == (nv, nt, npins)
    v = _volumes(b)
    assert v.min() > 0
    assert v.sum() == pytest.approx(dims[0] * dims[1] * dims[2] * b.h ** 3)
    # every tet vertex id in range, each cube's 6 tets share its main diagonal
    assert b.tets.min() == 0 and b.tets.max() == nv - 1


def test_config_sizes_match_the_workloads():
    # counts quoted for the 32x32x128 and 64x64x160 bars, without building them
    for (a, bb, L), nv, nt in [((32, 32, 128), 140481, 786432), ((64, 64, 160), 680225, 3932160)]:
        assert (a + 1) * (bb + 1) * (L + 1) == nv and 6 * a * bb * L == nt


def test_bar_is_seeded_and_pins_hold():
    a = bars.make_bar(3, 3, 6, twist_deg=90.0, noise=0.05, seed=9)
    b = bars.make_bar(3, 3, 6, twist_deg=90.0, noise=0.05, seed=9)
    c = bars.make_bar(3, 3, 6, twist_deg=90.0, noise=0.05, seed=10)
    np.testing.assert_array_equal(a.init, b.init)
    assert not np.array_equal(a.init, c.init)
    x = a.rest[a.pins, 0]
    assert set(np.unique(x)) == {0.0, a.length}
    # the far face is rotated by the full twist, the near face not at all
    near = a.pins[a.rest[a.pins, 0] == 0.0]
    np.testing.assert_allclose(a.init[near], a.rest[near], atol=1e-15)


def test_golden_tiny_bar_regenerates(golden):
    g = golden("tiny_step.npz")
    b = bars.make_bar(2, 2, 6, twist_deg=90.0, noise=0.05, seed=3)
    np.testing.assert_array_equal(b.init, g["init"])
    np.testing.assert_array_equal(b.tets, g["tets"])


def test_splitmix_known_values():
    # SplitMix64 reference outputs for seed 0 (Steele, Lea, Flood 2014)
    np.testing.assert_array_equal(bars.splitmix64(0, 3),
                                  np.array([0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F],
                                           dtype=np.uint64))


def test_mesh_files_roundtrip(tmp_path):
    b = bars.make_bar(2, 2, 3, noise=0.1, seed=1)
    files = bars.write_bar(b, str(tmp_path), "m")
    np.testing.assert_array_equal(bars.read_node(files["init"]), b.init)
    assert [int(t) for t in open(files["handles"]).read().split()] == list(b.pins)


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "wrapd_gpu.h")).read()
    return sorted(set(re.findall(r"WRAPD_API\s+[\w\s\*]+?\b(wrapd_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol(lib_built):
    lib = ctypes.CDLL(lib_built)
    syms = _header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    from wrapd_b200 import capi
    assert sorted(n for n, _, _ in capi.SIGNATURES) == syms


def test_settings_defaults_follow_the_reference(lib_built):
    from wrapd_b200 import capi
    s = capi.default_settings()
    assert (s.max_iters, s.tol, s.rot_aware, s.reweighting, s.rw_delay, s.gamma) == (5000, 1e-11, 1, 1, 50, 1.5)
    assert (s.global_iters, s.global_ls, s.kappa, s.poisson) == (100, 0, 1.0, 0.45)
    assert (s.beta_static, s.beta_min, s.beta_max, s.prox_iters, s.youngs, s.lbfgs_m) == (1.0, 0.1, 10.0, 20, 1e7, 6)


def test_settings_accept_the_reference_flag_names(lib_built):
    """The Python mirror maps the reference's flag names (-it, -ra, -rw,
    -global_it) onto the settings fields and rejects unknown names."""
    from wrapd_b200.solver import Settings
    s = Settings(it=500, ra=0, rw=0, global_it=7, tol=1e-9, precision="mixed", youngs=1e5)
    assert (s.max_iters, s.rot_aware, s.reweighting, s.global_iters, s.tol) == (500, 0, 0, 7, 1e-9)
    assert (s.precision, s.youngs, s.gamma) == (1, 1e5, 1.5)
    with pytest.raises(ValueError, match="unknown setting"):
        Settings(not_a_flag=1)


def test_no_device_fails_loudly(lib_built):
    """Without a usable GPU the library refuses to run (there is no CPU path)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from wrapd_b200 import capi
    with pytest.raises(capi.WrapdError) as ei:
        capi.Handle(capi.default_settings())
    assert ei.value.name == "WRAPD_E_CUDA"
    with pytest.raises(capi.WrapdError):
        capi.svd3_batch(np.eye(3).reshape(1, 9))
