"""GPU batches: several meshes added to one handle share the launches (one
local-step and one gradient launch over all unconverged meshes' element tiles,
one factorization with a tree per mesh), while each mesh is solved as the
reference solves it alone -- a Solver per mesh, with its own L-BFGS history
and early exits (deps/mcloptlib/include/MCL/SplitLBFGS.hpp:138-142, 181-232),
reweighting decision (src/System.cpp:50-63), convergence test
(src/ADMM.cpp:158-169) and, once converged, no further iterations.

The bar is bit-identity: every mesh of a batch ends with the same positions
and logs, bit for bit, as a handle holding that mesh alone (each mesh's tiles
and reductions are its own), and the single-mesh path is already pinned to
the reference (test_gpu_parity.py)."""
import numpy as np
import pytest

from conftest import E_YOUNG, NU
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


BASE = dict(youngs=E_YOUNG, poisson=NU, lbfgs_m=5)
LOGS = ("objectives", "inner_iters", "reweighted", "flips", "x_errors", "ls_delta_al", "gs_delta_al")


def _solve_batch(bs, mats=None, **kw):
    s = Solver(**dict(BASE, **kw))
    for i, b in enumerate(bs):
        m = {} if mats is None else dict(youngs=mats[i][0], poisson=mats[i][1])
        s.add_tetmesh(b.rest, b.init, b.tets, pins=b.pins, **m)
    s.initialize()
    X = s.solve()
    logs = [{k: s.log(k, mesh=i) for k in LOGS} for i in range(len(bs))]
    union = {k: s.log(k) for k in LOGS}
    s.close()
    return X, logs, union


def _solve_one(b, mat=None, **kw):
    m = {} if mat is None else dict(youngs=mat[0], poisson=mat[1])
    s = Solver(**dict(BASE, **kw))
    s.add_tetmesh(b.rest, b.init, b.tets, pins=b.pins, **m)
    s.initialize()
    X = s.solve()
    logs = {k: s.log(k) for k in LOGS}
    s.close()
    return X, logs


def _check(bs, mats=None, **kw):
    X, logs, union = _solve_batch(bs, mats, **kw)
    off = 0
    iters = []
    for i, b in enumerate(bs):
        Xi, li = _solve_one(b, None if mats is None else mats[i], **kw)
        np.testing.assert_array_equal(X[off:off + b.n_verts], Xi)
        for k in LOGS:
            np.testing.assert_array_equal(logs[i][k], li[k], err_msg=f"mesh {i}: {k}")
        iters.append(len(li["objectives"]) - 1)
        off += b.n_verts
    # the batch runs until its last mesh stops; its summary energy is the sum
    assert len(union["objectives"]) - 1 == max(iters)
    last = sum(lg["objectives"][-1] for lg in logs)
    assert union["objectives"][-1] == pytest.approx(last, rel=1e-15)
    return iters


def test_batch_meshes_equal_their_own_solves():
    """Three bars to convergence (tol 1e-11, gamma-rule reweighting past
    rw_delay): each stops at its own iteration, bit for bit its own solve."""
    iters = _check(_bars(), max_iters=600)
    assert len(set(iters)) > 1          # they converge at different iterations


def test_batch_of_materials_equals_their_own_solves():
    _check(_bars(), [(2e4, 0.35), (1e5, 0.45), (6e5, 0.40)], max_iters=300)


def test_batch_reweight_every_and_mixed_precision():
    """Reweight every 10 iterations, FP32 local step: every mesh's
    refinement switch (FP64 local steps near convergence) is its own."""
    _check(_bars(), max_iters=300, rw_every=10, precision=1)


def test_batch_with_a_large_mesh():
    """A mesh above the one-CTA two-loop limit (3 x free vertices > 16384)
    beside small ones: the two forms of the two-loop recursion in one batch."""
    bs = [bars.make_bar(12, 12, 40, twist_deg=150.0, noise=0.02, seed=4)] + _bars()[:2]
    assert 3 * (bs[0].n_verts - len(bs[0].pins)) > 16384
    _check(bs, max_iters=80)


def test_batch_of_one_equals_single_mesh_path():
    b = bars.bar_8x8x32()
    X1, _, _ = _solve_batch([b], max_iters=30)
    s = Solver(**dict(BASE, max_iters=30))
    s.add_tetmesh(b.rest, b.init, b.tets)
    s.set_pins(b.pins)
    s.initialize()
    X2 = s.solve()
    np.testing.assert_array_equal(X1, X2)


def test_batch_rejects_unsupported_modes():
    for kw in (dict(rot_aware=0), dict(global_ls=1)):
        s = Solver(**dict(BASE, **kw))
        for b in _bars()[:2]:
            s.add_tetmesh(b.rest, b.init, b.tets, pins=b.pins)
        with pytest.raises(capi.WrapdError) as ei:
            s.initialize()
        assert ei.value.name == "WRAPD_E_UNSUPPORTED"
        s.close()
