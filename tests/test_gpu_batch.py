"""GPU parity of batches: several meshes added to one handle form one
block-diagonal system (one local-step launch over all elements, one
factorization with a tree per mesh).  The oracle solves the union of the meshes
as one mesh, with per-element materials when the meshes differ; FP64 bar as
in the single-mesh parity tests: positions within 1e-8 of max |x|, energy
trajectory within 1e-8 relative, the same iteration counts."""
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


def _bars():
    return [bars.make_bar(4, 4, 8, twist_deg=120.0, noise=0.02, seed=1),
            bars.make_bar(5, 4, 10, twist_deg=200.0, noise=0.02, seed=2),
            bars.make_bar(4, 6, 12, twist_deg=90.0, noise=0.02, seed=3)]


def _solve_batch(bs, mats=None, iters=40):
    s = Solver(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, max_iters=iters)
    for i, b in enumerate(bs):
        kw = {} if mats is None else dict(youngs=mats[i][0], poisson=mats[i][1])
        s.add_tetmesh(b.rest, b.init, b.tets, pins=b.pins, **kw)
    s.initialize()
    X = s.solve()
    return X, s.algorithm_data(), s.info()


def _oracle(union, iters, youngs_e=None, poisson_e=None):
    o = po.Oracle(union.rest, union.init, union.tets, union.pins, youngs=E_YOUNG, poisson=NU, max_iters=iters,
                  lbfgs_m=5, youngs_e=youngs_e, poisson_e=poisson_e)
    o.solve()
    return o


def _compare(X, d, o):
    Xo = o.get("X").reshape(-1, 3)
    obj = o.get("objectives")
    assert len(d.objectives) == len(obj)
    np.testing.assert_allclose(d.objectives, obj, rtol=1e-8)
    assert np.abs(X - Xo).max() <= 1e-8 * np.abs(Xo).max()
    np.testing.assert_array_equal(d.inner_iters, o.get("inner_iters"))
    np.testing.assert_array_equal(d.reweighted, o.get("reweighted"))


def test_batch_same_material_matches_oracle_on_union():
    bs = _bars()
    X, d, info = _solve_batch(bs)
    union = bars.concat(bs)
    assert int(info["n_verts"]) == union.n_verts and int(info["n_tets"]) == union.n_tets
    _compare(X, d, _oracle(union, 40))


def test_batch_of_materials_matches_oracle_with_element_materials():
    bs = _bars()
    mats = [(2e4, 0.35), (1e5, 0.45), (6e5, 0.40)]
    X, d, _ = _solve_batch(bs, mats)
    union = bars.concat(bs)
    ye = np.concatenate([np.full(b.n_tets, m[0]) for b, m in zip(bs, mats)])
    pe = np.concatenate([np.full(b.n_tets, m[1]) for b, m in zip(bs, mats)])
    _compare(X, d, _oracle(union, 40, ye, pe))


def test_batch_of_one_equals_single_mesh_path():
    b = bars.bar_8x8x32()
    X1, d1, _ = _solve_batch([b], iters=30)
    s = Solver(youngs=E_YOUNG, poisson=NU, lbfgs_m=5, max_iters=30)
    s.add_tetmesh(b.rest, b.init, b.tets)
    s.set_pins(b.pins)
    s.initialize()
    X2 = s.solve()
    np.testing.assert_array_equal(X1, X2)
