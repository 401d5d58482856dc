"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's golden vectors.

Tolerances (FP64 mode):
  * per-element math (SVD, Hessian eigenvalue): rounding level, 1e-12 relative;
  * the prox: it stops when |dx| < 1e-8 (src/TetElements.hpp:40-42), so its
    output is defined to ~1e-9 and a last-ulp difference can move the stop by
    one iteration: stretches within 5e-8, iteration counts equal in >= 97%;
  * full solves: final positions within 1e-8 of max |x| (the FP64 parity bar),
    energy trajectory within 1e-8 relative, identical iteration counts.
Mixed mode (FP32 element math): final positions within 1e-5 of max |x|.
"""
import numpy as np
import pytest

from conftest import E_YOUNG, NU
from oracle import pyoracle as po
from wrapd_b200 import bars, capi
from wrapd_b200.solver import Settings, Solver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(lib_built):
    capi.load()


def make_solver(bar, **kw):
    kw.setdefault("youngs", E_YOUNG)
    kw.setdefault("poisson", NU)
    s = Solver(**kw)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    return s


def rel_max(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300)


# ---- per-element functions ------------------------------------------------------
def test_svd_matches_reference(golden):
    g = golden("elem_cases.npz")
    s, U, V = capi.svd3_batch(g["F"])
    scale = np.abs(g["sigma"]).max(axis=1, keepdims=True) + 1e-300
    # same Jacobi sweep as the reference; FMA contraction moves the last few bits
    assert np.all(np.abs(s - g["sigma"]) <= 1e-14 * scale + 1e-300)
    # reconstruction U diag(s) V^T = F for every case
    Ur = U.reshape(-1, 3, 3).transpose(0, 2, 1)
    Vr = V.reshape(-1, 3, 3).transpose(0, 2, 1)
    F = g["F"].reshape(-1, 3, 3).transpose(0, 2, 1)
    R = np.einsum("nij,nj,nkj->nik", Ur, s, Vr)
    assert np.all(np.abs(R - F).max(axis=(1, 2)) <= 1e-14 * (np.abs(F).max(axis=(1, 2)) + 1e-300))
    # singular vectors themselves where the singular values are well separated
    gs = np.abs(g["sigma"])
    sep = np.min(np.abs(np.diff(np.sort(gs, axis=1), axis=1)), axis=1) > 1e-6 * (gs.max(axis=1) + 1e-300)
    assert sep.sum() > 300
    assert np.abs(U[sep] - g["U"][sep]).max() < 1e-9
    assert np.abs(V[sep] - g["V"][sep]).max() < 1e-9


def test_svd_fp32(golden):
    g = golden("elem_cases.npz")
    s, _, _ = capi.svd3_batch(g["F"], fp32=True)
    scale = np.abs(g["sigma"]).max(axis=1, keepdims=True)
    ok = scale[:, 0] < 1e30
    assert np.all(np.abs(s - g["sigma"])[ok] <= 1e-5 * scale[ok] + 1e-30)


def test_prox_matches_reference(golden):
    g = golden("elem_cases.npz")
    out, its = capi.prox_batch(float(g["mu"]), float(g["lam"]), g["prox_s0"], g["prox_wov"], g["prox_start"])
    assert np.abs(out - g["prox_out"]).max() < 5e-8
    assert np.mean(its == g["prox_iters"]) >= 0.97


def test_hessian_eigenvalue_matches_reference(golden):
    g = golden("elem_cases.npz")
    lm = capi.hess_lmax_batch(float(g["mu"]), float(g["lam"]), g["hess_sigma"])
    np.testing.assert_allclose(lm, g["hess_lmax"], rtol=1e-12, atol=1e-6)


def test_potential_energy_batch_matches_oracle():
    rng = np.random.default_rng(21)
    n = 100_003
    sig = np.abs(rng.normal(1.0, 0.3, size=(n, 3)))
    sig[::97, 2] *= -1.0
    sig[5::53] = rng.uniform(0.05, 0.3, size=sig[5::53].shape)
    vol = rng.uniform(1e-4, 1e-3, size=n)
    mu, lam = po.lame(E_YOUNG, NU)
    pe, flips = capi.potential_energy_batch(mu, lam, sig, vol)
    lib = po.load_oracle()
    psi = np.array([lib.orc_nh_psi_plain(mu, lam, po._d(np.ascontiguousarray(s))) for s in sig])
    assert pe == pytest.approx(float(np.sum(vol * psi)), rel=1e-12)
    assert flips == int(np.sum((sig < 0).any(axis=1)))


# ---- TetElements-level steps ------------------------------------------------------
def test_tiny_step_matches_reference(golden):
    g = golden("tiny_step.npz")
    bar = bars.Bar(rest=g["rest"], init=g["init"], tets=g["tets"], pins=g["pins"], h=0.5, length=3.0, dims=())
    s = make_solver(bar)
    s.begin_solve()
    dal = s.polar_update(False)
    assert dal == pytest.approx(float(g["dal"]), rel=1e-12)
    s.update_defo_cache()
    v, gr = s.global_grad()
    assert v == pytest.approx(float(g["value"]), rel=1e-8)
    assert rel_max(gr, g["grad"]) < 1e-7
    pe, flips = s.potential_energy()
    assert pe == pytest.approx(float(g["pe"]), rel=1e-13)
    assert flips == int(g["flips"])
    free = np.setdiff1d(np.arange(bar.n_verts), bar.pins)
    _, g2 = s.global_grad(g["X2"][free])
    assert rel_max(g2, g["grad2"]) < 1e-7


def test_local_step_matches_oracle_state():
    bar = bars.make_bar(4, 4, 12, twist_deg=150.0, noise=0.03, seed=4)
    s = make_solver(bar)
    s.begin_solve()
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU)
    o.setup()
    for name in ("Z", "U", "w2"):
        assert rel_max(s.get_state(name), o.get(name)) < 1e-13, name
    d_gpu = s.polar_update(True)
    d_orc = o.polar_update(True)
    assert d_gpu == pytest.approx(d_orc, rel=1e-12)
    for name in ("Z", "U", "slast", "w2c"):
        assert rel_max(s.get_state(name), o.get(name)) < 5e-8, name


@pytest.mark.parametrize("dims", [(3, 3, 8), (8, 8, 32)])
def test_solve_A_matches_oracle(dims):
    bar = bars.make_bar(*dims, twist_deg=100.0, noise=0.02, seed=1)
    s = make_solver(bar)
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU)
    o.setup()
    rng = np.random.default_rng(3)
    b = rng.normal(size=(o.n_free, 3))
    assert rel_max(s.solve_A(b), o.solve_A(b)) < 1e-11


def test_solve_waits_are_bounded():
    """The solve runs each direction as one launch over a work queue whose
    items wait for the fronts they read.  Holding back one leaf's completion
    makes its parent's wait run out: the call returns WRAPD_E_TIMEOUT after
    about a second instead of hanging, and the handle then solves as before,
    bit for bit (the queue's results do not depend on the order CTAs take
    items)."""
    import time
    bar = bars.make_bar(8, 8, 32, twist_deg=100.0, noise=0.02, seed=1)
    s = make_solver(bar)
    b = np.random.default_rng(5).normal(size=(int(s.info()["n_free"]), 3))
    x0 = s.solve_A(b)
    for _ in range(3):
        np.testing.assert_array_equal(s.solve_A(b), x0)
    t0 = time.perf_counter()
    with pytest.raises(capi.WrapdError) as ei:
        s.solve_A_holding(b, 0)   # front 0 is a leaf: its parent waits on it
    assert ei.value.name == "WRAPD_E_TIMEOUT"
    assert time.perf_counter() - t0 < 30.0
    with pytest.raises(capi.WrapdError) as ei:
        s.solve_A_holding(b, int(s.info()["fronts"]))
    assert ei.value.name == "WRAPD_E_INPUT"
    np.testing.assert_array_equal(s.solve_A(b), x0)


# ---- whole solves --------------------------------------------------------------------
def _compare_solve(s, objectives, inner, reweighted, x, tol_x):
    X = s.solve()
    obj = s.log("objectives")
    assert len(obj) == len(objectives)
    np.testing.assert_array_equal(s.log("inner_iters"), inner)
    np.testing.assert_array_equal(s.log("reweighted"), reweighted)
    np.testing.assert_allclose(obj, objectives, rtol=1e-8)
    assert rel_max(X, x) <= tol_x


def test_solve_small_bars_match_reference(golden):
    g = golden("solve_small.npz")
    bar = bars.Bar(rest=g["rest"], init=g["init"], tets=g["tets"], pins=g["pins"], h=1 / 3, length=10 / 3, dims=())
    for tag, rw_delay in (("a", 50), ("b", 5)):
        s = make_solver(bar, max_iters=300, rw_delay=rw_delay)
        _compare_solve(s, g[f"{tag}_objectives"], g[f"{tag}_inner"], g[f"{tag}_reweighted"], g[f"{tag}_x"], 1e-8)


def test_solve_bar_8x8x32_matches_reference(golden):
    g = golden("solve_bar_8x8x32.npz")
    s = make_solver(bars.bar_8x8x32(), max_iters=500)
    _compare_solve(s, g["objectives"], g["inner"], g["reweighted"], g["x"], 1e-8)


def test_solve_bar_8x8x32_mixed_precision(golden):
    g = golden("solve_bar_8x8x32.npz")
    s = make_solver(bars.bar_8x8x32(), max_iters=500, precision=1)
    X = s.solve()
    assert rel_max(X, g["x"]) < 1e-5
    assert s.log("objectives")[-1] == pytest.approx(g["objectives"][-1], rel=1e-6)


def test_solve_bar_8x8x32_newton_prox(golden):
    """prox_mode 1 (Newton) reaches the reference's solution to its convergence level."""
    g = golden("solve_bar_8x8x32.npz")
    s = make_solver(bars.bar_8x8x32(), max_iters=500, prox_mode=1)
    X = s.solve()
    assert rel_max(X, g["x"]) < 1e-6
    assert s.log("objectives")[-1] == pytest.approx(g["objectives"][-1], rel=1e-9)


def test_rw_every_and_history_5_match_oracle():
    bar = bars.make_bar(4, 4, 10, twist_deg=200.0, noise=0.02, seed=8)
    s = make_solver(bar, max_iters=40, lbfgs_m=5, rw_every=10, rw_delay=5)
    X = s.solve()
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU, max_iters=40, lbfgs_m=5,
                  rw_every=10, rw_delay=5)
    o.solve()
    np.testing.assert_array_equal(s.log("reweighted"), o.get("reweighted"))
    np.testing.assert_array_equal(s.log("inner_iters"), o.get("inner_iters"))
    np.testing.assert_allclose(s.log("objectives"), o.get("objectives"), rtol=1e-8)
    assert rel_max(X, o.get("X").reshape(-1, 3)) < 1e-8


# ---- error behaviour -------------------------------------------------------------------
def test_inverted_rest_tet_is_rejected():
    bar = bars.make_bar(2, 2, 3)
    t = bar.tets.copy()
    t[5, [1, 2]] = t[5, [2, 1]]
    s = Solver(youngs=E_YOUNG)
    s.add_tetmesh(bar.rest, bar.init, t)
    s.set_pins(bar.pins)
    with pytest.raises(capi.WrapdError) as ei:
        s.initialize()
    assert ei.value.name == "WRAPD_E_INVERTED_REST"


def test_bad_input_is_rejected():
    bar = bars.make_bar(2, 2, 3)
    s = Solver(youngs=E_YOUNG)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(np.array([0, 0, 1]))
    with pytest.raises(capi.WrapdError) as ei:
        s.initialize()
    assert ei.value.name == "WRAPD_E_INPUT"
    with pytest.raises(capi.WrapdError) as ei:
        Solver(Settings(rot_aware=2))
    assert ei.value.name == "WRAPD_E_INPUT"
    s2 = Solver(youngs=E_YOUNG)
    with pytest.raises(capi.WrapdError) as ei:
        s2.begin_solve()
    assert ei.value.name == "WRAPD_E_STATE"


def test_nan_input_reports_an_error_and_the_context_survives():
    bar = bars.make_bar(2, 2, 4, noise=0.05, seed=2)
    init = bar.init.copy()
    free = np.setdiff1d(np.arange(bar.n_verts), bar.pins)
    init[free[0]] = np.nan
    s = Solver(youngs=E_YOUNG, max_iters=5)
    s.add_tetmesh(bar.rest, init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    with pytest.raises(capi.WrapdError) as ei:
        s.solve()
    assert ei.value.name in ("WRAPD_E_NAN", "WRAPD_E_PROX_NEG", "WRAPD_E_NOT_SPD")
    # the device is still usable
    s2 = make_solver(bars.make_bar(2, 2, 4, noise=0.05, seed=2), max_iters=3)
    s2.solve()


# ---- full-size properties (786,432 tets) ---------------------------------------------
@pytest.fixture(scope="module")
def big():
    bar = bars.bar_32x32x128_bent()
    s = make_solver(bar, lbfgs_m=5, rw_every=10)
    return bar, s


def test_large_bar_solve_A_residual(big):
    """A (A^-1 b) = b for the 138,303-unknown weighted Laplacian, A built on the host."""
    import scipy.sparse as sp
    bar, s = big
    w2 = s.get_state("w2")
    free = -np.ones(bar.n_verts, dtype=np.int64)
    fidx = np.setdiff1d(np.arange(bar.n_verts), bar.pins)
    free[fidx] = np.arange(fidx.size)
    P = bar.rest[bar.tets]
    Dm = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=2)
    S = np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    Di = np.einsum("ab,nbc->nac", S, np.linalg.inv(Dm))          # (n, 4, 3) = (S Dm^-1)
    K = w2[:, None, None] * np.einsum("nac,nbc->nab", Di, Di)   # (n, 4, 4)
    fi = free[bar.tets]
    rows = np.repeat(fi, 4, axis=1).ravel()
    cols = np.tile(fi, (1, 4)).ravel()
    keep = (rows >= 0) & (cols >= 0)
    A = sp.csr_matrix((K.ravel()[keep], (rows[keep], cols[keep])), shape=(fidx.size, fidx.size))
    rng = np.random.default_rng(5)
    b = rng.normal(size=(fidx.size, 3))
    x = s.solve_A(b)
    r = A @ x - b
    assert np.abs(r).max() / np.abs(b).max() < 1e-9


def test_large_bar_gradient_matches_oracle(big):
    """The global gradient at full size for seeded dual variables (at the initial
    state Z = sym(F), U = 0 the gradient vanishes, so Z and U are perturbed)."""
    bar, s = big
    s.begin_solve()
    o = po.Oracle(bar.rest, bar.init, bar.tets, bar.pins, youngs=E_YOUNG, poisson=NU)
    o.init_state()
    rng = np.random.default_rng(12)
    Z = o.get("Z") + 0.05 * rng.normal(size=9 * bar.n_tets)
    U = 0.05 * rng.normal(size=9 * bar.n_tets)
    o.set("Z", Z); o.set("U", U)
    s.set_state("Z", Z); s.set_state("U", U)
    v, g = s.global_grad()
    vo, go = o.grad_cached()
    assert v == pytest.approx(vo, rel=1e-10)
    assert rel_max(g, go) < 1e-10


def test_large_bar_iterations_decrease_energy(big):
    bar, s = big
    s.begin_solve()
    done, _ = s.iterate(12)
    obj = s.log("objectives")
    assert done == 12 and len(obj) == 13
    assert obj[-1] < obj[0]
    assert s.log("reweighted")[10] == 1   # rw_every = 10 fires after iteration index 9
    assert np.isfinite(s.positions()).all()
