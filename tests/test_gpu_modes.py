"""GPU parity of the solver modes beside the default: the rotation-unaware
global step (-ra 0, UnawareGS: x = A^-1 b every iteration), the ARAP model
(-model arap, with -rw 0 as the reference requires) and the global step's
backtracking line search (-global_ls 1), each against the reference's own
solve (tests/golden/solve_modes.npz, solve_gls.npz) and against the oracle.
FP64: energies and positions within 1e-8 relative, identical logs."""
import numpy as np
import pytest

from conftest import E_YOUNG, NU
from oracle import pyoracle as po
from wrapd_b200 import capi
from wrapd_b200.solver import Solver

pytestmark = pytest.mark.gpu

MODES = {"ra0": dict(rot_aware=0), "arap": dict(model=1, reweighting=0),
         "arap_ra0": dict(model=1, reweighting=0, rot_aware=0)}


@pytest.fixture(scope="module", autouse=True)
def _lib(lib_built):
    capi.load()


def _solve(g, iters, **kw):
    s = Solver(youngs=E_YOUNG, poisson=NU, max_iters=iters, **kw)
    s.add_tetmesh(g["rest"], g["init"], g["tets"])
    s.set_pins(g["pins"])
    s.initialize()
    X = s.solve()
    return X, s.algorithm_data()


@pytest.mark.parametrize("tag", sorted(MODES))
def test_mode_matches_reference(golden, tag):
    g = golden("solve_modes.npz")
    X, d = _solve(g, 60, **MODES[tag])
    np.testing.assert_allclose(d.objectives, g[f"{tag}_objectives"], rtol=1e-8)
    assert np.abs(X - g[f"{tag}_x"]).max() <= 1e-8 * np.abs(g[f"{tag}_x"]).max()
    np.testing.assert_array_equal(d.inner_iters, g[f"{tag}_inner"])
    np.testing.assert_array_equal(d.reweighted, g[f"{tag}_reweighted"])


def test_unaware_mixed_precision_close_to_oracle(golden):
    """-ra 0 with the FP32 local step, run to convergence: final positions
    within 1e-5 of the converged FP64 oracle."""
    g = golden("solve_modes.npz")
    X, d = _solve(g, 3000, rot_aware=0, precision="mixed")
    o = po.Oracle(g["rest"], g["init"], g["tets"], g["pins"], youngs=E_YOUNG, poisson=NU, max_iters=3000,
                  rot_aware=0)
    o.solve()
    assert len(d.objectives) < 3001 and o.iters < 3000   # both converged
    Xo = o.get("X").reshape(-1, 3)
    assert np.abs(X - Xo).max() <= 1e-5 * np.abs(Xo).max()


def test_arap_with_reweighting_is_rejected(golden):
    g = golden("solve_modes.npz")
    s = Solver(youngs=E_YOUNG, poisson=NU, model=1)
    s.add_tetmesh(g["rest"], g["init"], g["tets"])
    s.set_pins(g["pins"])
    with pytest.raises(capi.WrapdError) as e:
        s.initialize()
    assert e.value.name == "WRAPD_E_INPUT"


def test_global_line_search_matches_reference(golden):
    """-global_ls 1 on a 720-degree-twisted bar (-rw 0) where the search
    shortens the step from iteration 33 on: the reference's energies within
    1e-8 of the largest (1e-6 of each: they fall from 1e10 to 1e-3), final
    positions within 1e-8 of max |x|, identical inner-iteration log; and the
    oracle's trajectory to 1e-9 of the largest energy."""
    g = golden("solve_gls.npz")
    X, d = _solve(g, 80, reweighting=0, global_ls=1)
    ref = g["objectives"]
    assert np.abs(d.objectives - ref).max() <= 1e-8 * np.abs(ref).max()
    np.testing.assert_allclose(d.objectives, ref, rtol=1e-6)
    assert np.abs(X - g["x"]).max() <= 1e-8 * np.abs(g["x"]).max()
    np.testing.assert_array_equal(d.inner_iters, g["inner"])
    o = po.Oracle(g["rest"], g["init"], g["tets"], g["pins"], youngs=E_YOUNG, poisson=NU, max_iters=80,
                  reweighting=0, global_ls=1)
    o.solve()
    assert np.abs(d.objectives - o.get("objectives")).max() <= 1e-9 * np.abs(ref).max()
    # the search is live: plain rate-1 steps leave this trajectory
    X0, d0 = _solve(g, 80, reweighting=0)
    assert np.abs(d0.objectives[:60] - ref[:60]).max() > 1e-6 * np.abs(ref).max()
