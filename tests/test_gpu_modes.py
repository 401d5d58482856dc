"""GPU parity of the solver modes beside the default: the rotation-unaware
global step (-ra 0, UnawareGS: x = A^-1 b every iteration) and the ARAP model
(-model arap, with -rw 0 as the reference requires), each against the
reference's own solve (tests/golden/solve_modes.npz) and against the oracle.
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
