"""The tile-shape autotuner (settings.autotune = 1): wrapd_initialize times the
solve's candidate chunk lengths per level and direction and the panel-step
forms of the factorization on the system at hand, and the first begin_solve
the local step's tile (elements per CTA), then keeps the fastest.  The
choice changes only the order of partial sums, so the tuned solver must meet
the same FP64 bar against the reference as the fixed rules (positions within
1e-8 of max |x|, identical iteration counts), and report shapes from the
candidate sets."""
import numpy as np
import pytest

from conftest import E_YOUNG, NU
from wrapd_b200 import bars, capi
from wrapd_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(lib_built):
    capi.load()


def _solve(autotune, iters=500):
    bar = bars.bar_8x8x32()
    s = Solver(youngs=E_YOUNG, poisson=NU, max_iters=iters, autotune=autotune)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    X = s.solve()
    return X, s.algorithm_data(), s.tuning(), s.info()


def test_autotuned_solve_matches_reference(golden):
    g = golden("solve_bar_8x8x32.npz")
    X, d, t, info = _solve(1)
    assert len(d.objectives) == len(g["objectives"])
    np.testing.assert_array_equal(d.inner_iters, g["inner"])
    np.testing.assert_allclose(d.objectives, g["objectives"], rtol=1e-8)
    assert np.abs(X - g["x"]).max() <= 1e-8 * np.abs(g["x"]).max()
    assert t["levels"] == int(info["levels"])
    assert len(t["solve_chunk_fwd"]) == len(t["solve_chunk_bwd"]) == t["levels"]
    assert set(t["solve_chunk_fwd"]) | set(t["solve_chunk_bwd"]) <= {256, 128, 64}
    assert t["fused_panel_ctas"] in (0, 148, 592, 2368, 1 << 30)
    assert t["local_tile"] in (64, 128, 256, 512)


def test_fixed_rules_reported_without_autotune():
    _, _, t, _ = _solve(0, iters=3)
    assert t["fused_panel_ctas"] == 592
    assert t["local_tile"] == 512
    assert all(c in (256, 128, 64) for c in t["solve_chunk_fwd"] + t["solve_chunk_bwd"])
