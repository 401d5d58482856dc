"""Edge cases of the input through the C ABI: the smallest mesh (one tet, one
free vertex) against the oracle, a ragged batch (a one-tet mesh beside a bar)
whose meshes are each their own solve, and the rejections the reference raises as
exceptions (src/TetElements.cpp:99-101, src/System.cpp:33-44) returned as
error codes -- with the device still usable afterwards."""
import numpy as np
import pytest

from conftest import E_YOUNG, NU
from oracle import pyoracle as po
from wrapd_b200 import bars, capi
from wrapd_b200.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(lib_built):
    capi.load()


def _one_tet():
    rest = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    init = rest.copy()
    init[3] = [0.3, -0.2, 1.6]
    return rest, init, np.array([[0, 1, 2, 3]], dtype=np.int32), np.array([0, 1, 2], dtype=np.int32)


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_single_tet_matches_oracle():
    rest, init, tets, pins = _one_tet()
    s = Solver(youngs=E_YOUNG, poisson=NU, max_iters=200)
    s.add_tetmesh(rest, init, tets)
    s.set_pins(pins)
    s.initialize()
    X = s.solve()
    o = po.Oracle(rest, init, tets, pins, youngs=E_YOUNG, poisson=NU, max_iters=200)
    o.solve()
    Xo = o.get("X").reshape(-1, 3)
    # With one element nothing averages the prox's absolute stop (|d sigma| <
    # 1e-8, src/TetElements.hpp:40-42): a last-ulp difference moves it by an
    # iteration and the energy by ~1e-8 relative, so the stop of the ADMM loop
    # (an energy change below 1e-11 near zero energy) may come an iteration
    # apart.  Trajectory: each energy within 2e-8 of itself plus 1e-9 of the
    # initial energy (it falls five orders in 30 iterations); final positions
    # to 1e-7.
    obj, obj_o = s.log("objectives"), o.get("objectives")
    assert abs(len(obj) - len(obj_o)) <= 2
    assert (np.abs(obj[:30] - obj_o[:30]) <= 2e-8 * np.abs(obj_o[:30]) + 1e-9 * obj_o[0]).all()
    assert _rel(X, Xo) < 1e-7
    # the free vertex relaxes to the rest shape (the energy's minimum)
    assert np.abs(X[3] - rest[3]).max() < 1e-4


def test_ragged_batch_meshes_match_their_own_solves():
    """A single tet beside a bar in one batch: each mesh is its own solve -- the
    tet bit for bit the same as a handle holding it alone (its own comparison
    with the oracle is test_single_tet_matches_oracle), the bar within the FP64
    bar of the oracle's solve of the bar alone (energies 1e-8, positions 1e-8
    of max |x|, identical inner iterations)."""
    rest, init, tets, pins = _one_tet()
    bar = bars.make_bar(4, 4, 12, twist_deg=150.0, noise=0.02, seed=4)
    s = Solver(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, max_iters=60)
    s.add_tetmesh(rest, init, tets, pins=pins)
    s.add_tetmesh(bar.rest, bar.init, bar.tets, pins=bar.pins)
    s.initialize()
    X = s.solve()
    nv0 = rest.shape[0]
    s1 = Solver(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, max_iters=60)
    s1.add_tetmesh(rest, init, tets, pins=pins)
    s1.initialize()
    np.testing.assert_array_equal(X[:nv0], s1.solve())
    np.testing.assert_array_equal(s.log("objectives", mesh=0), s1.log("objectives"))
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU, max_iters=60, lbfgs_m=5)
    o.solve()
    assert len(s.log("objectives", mesh=1)) == len(o.get("objectives"))
    np.testing.assert_allclose(s.log("objectives", mesh=1), o.get("objectives"), rtol=1e-8)
    np.testing.assert_array_equal(s.log("inner_iters", mesh=1), o.get("inner_iters"))
    assert _rel(X[nv0:], o.get("X").reshape(-1, 3)) < 1e-8


def _expect(code, fn):
    with pytest.raises(capi.WrapdError) as ei:
        fn()
    assert ei.value.name in code, ei.value.name


def test_rejections():
    rest, init, tets, pins = _one_tet()

    def all_pinned():
        s = Solver(youngs=E_YOUNG)
        s.add_tetmesh(rest, init, tets)
        s.set_pins(np.arange(4))
        s.initialize()
    _expect(("WRAPD_E_INPUT",), all_pinned)

    def pin_out_of_range():
        s = Solver(youngs=E_YOUNG)
        s.add_tetmesh(rest, init, tets)
        s.set_pins(np.array([0, 1, 7]))
        s.initialize()
    _expect(("WRAPD_E_INPUT",), pin_out_of_range)

    def tet_id_out_of_range():
        s = Solver(youngs=E_YOUNG)
        s.add_tetmesh(rest, init, np.array([[0, 1, 2, 9]], dtype=np.int32))
        s.set_pins(pins)
        s.initialize()
    _expect(("WRAPD_E_INPUT",), tet_id_out_of_range)

    def shape_mismatch():
        s = Solver(youngs=E_YOUNG)
        s.add_tetmesh(rest, init[:3], tets)
    _expect(("WRAPD_E_INPUT",), shape_mismatch)


def test_degenerate_rest_tet_fails_cleanly():
    """A zero-volume rest tet passes the reference's sign check (vol < 0) and
    makes its rest-shape inverse infinite; the solve must end in an error code,
    not a hang or a fault, and the device must stay usable."""
    bar = bars.make_bar(2, 2, 3, noise=0.0, seed=0)
    rest = bar.rest.copy()
    a, b, c, d = bar.tets[5]
    rest[d] = rest[a] + 0.5 * (rest[b] - rest[a]) + 0.5 * (rest[c] - rest[a])   # d in the plane of a, b, c
    s = Solver(youngs=E_YOUNG, max_iters=5)
    s.add_tetmesh(rest, bar.init, bar.tets)
    s.set_pins(bar.pins)

    def run():
        s.initialize()
        s.solve()
    _expect(("WRAPD_E_NOT_SPD", "WRAPD_E_NAN", "WRAPD_E_PROX_NEG", "WRAPD_E_INVERTED_REST"), run)
    s2 = Solver(youngs=E_YOUNG, max_iters=3)
    ok = bars.make_bar(2, 2, 3, noise=0.02, seed=1)
    s2.add_tetmesh(ok.rest, ok.init, ok.tets)
    s2.set_pins(ok.pins)
    s2.initialize()
    assert np.isfinite(s2.solve()).all()
