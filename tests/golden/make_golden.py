"""Generate the golden vectors in tests/golden/ from the reference itself.

Needs the reference build (``make -C oracle ref``, which compiles the
reference sources into oracle/_ref/).  Run from the repository root:

    python tests/golden/make_golden.py

Outputs (all seeded, reproducible):
  elem_cases.npz    per-element functions: math::svd, the NH prox
                    (LBFGS<3> + cubic backtracking), the prox value/gradient and
                    the candidate-stiffness eigenvalue, on random and edge inputs
  tiny_step.npz     one setup + local step + gradient of TetElements on a small bar
  solve_small.npz   full reference solves of small bars (default and rw_delay 5)
  solve_bar_8x8x32.npz the reference solve of the 8x8x32 bar (E = 1e5, nu = 0.45)
  solve_modes.npz   reference solves of a small bar with -ra 0, -model arap -rw 0
                    and -model arap -rw 0 -ra 0
  solve_gls.npz     the reference solve of a strongly twisted small bar with
                    -global_ls 1 -rw 0 (the global step's backtracking line
                    search shortens steps from iteration 33 on)
  quasi_small.npz   the reference front end's output files for a small bar: the
                    logs, final_mesh.node/.ele/.obj, without and with -soln
  solve_bar_32x32x128_bent.npz
                    the benchmarked configuration: the 786,432-tet bar (360 deg
                    twist + 90 deg bend), 20 ADMM iterations of the patched
                    reference (quasi_ref_m5: L-BFGS history 5, reweight and
                    refactor every 10 iterations), and 60 iterations of the
                    unpatched reference (history 6, gamma rule, which
                    refactors at every iteration from 50 on); one thread each
                    (the deterministic reference), about 45 min of CPU for the
                    two side by side; positions at 16,384 seeded vertices
  iters_bar_64x64x160.npz
                    the 3.9M-tet bar (720 deg twist): the first three ADMM
                    iterations (L-BFGS history 5, FP64) of the oracle, the C
                    restatement pinned against the reference by the files above,
                    with its conjugate-gradient linear solver (the reference's
                    simplicial factorization of 671,775 unknowns, and the
                    oracle's envelope one, do not fit in this host's memory);
                    positions at 16,384 seeded vertices and per-column sums

    python tests/golden/make_golden.py [--only modes|gls|quasi|bar_32x32x128_bent|bar_64x64x160]
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from wrapd_b200 import bars  # noqa: E402

E_YOUNG, NU = 1e5, 0.45
X_SAMPLE = 16384   # vertices whose positions the large-bar fixtures keep


def svd_inputs(rng):
    n = 64
    F = [rng.normal(size=(n, 3, 3))]
    F.append(np.eye(3)[None] + 1e-7 * rng.normal(size=(n, 3, 3)))           # near identity
    F.append(np.tile(np.eye(3), (8, 1, 1)))                                   # exact identity
    refl = np.diag([1.0, 1.0, -1.0])
    F.append(rng.normal(size=(n, 3, 3)) @ refl)                               # random, often inverted
    A = rng.normal(size=(n, 3, 3)); A[:, :, 2] = A[:, :, 1]                   # rank 2
    F.append(A)
    B = rng.normal(size=(n, 3, 3)); B[:, :, 1] = 2 * B[:, :, 0]; B[:, :, 2] = -B[:, :, 0]  # rank 1
    F.append(B)
    F.append(np.zeros((2, 3, 3)))                                             # zero matrix
    D = np.zeros((n, 3, 3))
    for i in range(n):
        D[i] = np.diag(rng.choice([-2.0, -0.5, 0.0, 0.5, 1.0, 3.0], size=3))  # diagonal, signs, ties
    F.append(D)
    R = []
    for i in range(n):                                                        # rotations times stretch
        q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
        R.append(q @ np.diag(rng.uniform(0.05, 3.0, size=3)) @ np.linalg.qr(rng.normal(size=(3, 3)))[0])
    F.append(np.array(R))
    F.append(1e-5 * rng.normal(size=(16, 3, 3)))                              # tiny scale
    F.append(1e5 * rng.normal(size=(16, 3, 3)))                               # large scale
    sym = rng.normal(size=(n, 3, 3)); sym = sym + np.transpose(sym, (0, 2, 1))  # symmetric, like S_in
    F.append(sym)
    F = np.concatenate(F)
    return np.ascontiguousarray(np.transpose(F, (0, 2, 1)).reshape(-1, 9))    # column-major per matrix


def elem_cases(ref, rng):
    Fc = svd_inputs(rng)
    n = Fc.shape[0]
    sig, U, V = np.zeros((n, 3)), np.zeros((n, 9)), np.zeros((n, 9))
    ref.ref_svd3(n, po._d(Fc), po._d(sig), po._d(U), po._d(V))
    mu, lam = po.lame(E_YOUNG, NU)
    k = 2.0066 * mu + 1.0122 * lam
    m = 512
    s0 = np.abs(rng.normal(1.0, 0.3, size=(m, 3)))
    s0[:32, 2] *= -1.0                                  # inverted inputs
    s0[32:48] = rng.uniform(0.05, 0.3, size=(16, 3))    # strongly compressed: J < J0 branch
    s0[48:64] = 1.0                                     # rest
    wov = rng.uniform(0.1, 10.0, size=m) * k
    start = np.abs(rng.normal(1.0, 0.1, size=(m, 3)))
    start[64:96] = 1.0
    out, its = np.zeros((m, 3)), np.zeros(m, dtype=np.int32)
    ref.ref_prox(m, po._d(s0), po._d(wov), po._d(start), mu, lam, po._d(out), its.ctypes.data_as(po._ip))
    xv = np.abs(rng.normal(1.0, 0.4, size=(m, 3)))
    xv[:16] = rng.uniform(0.05, 0.4, size=(16, 3))
    val, grad = np.zeros(m), np.zeros((m, 3))
    ref.ref_prox_value_grad(m, po._d(xv), po._d(s0), po._d(wov), mu, lam, po._d(val), po._d(grad))
    hs = np.concatenate([out, rng.uniform(0.05, 0.5, size=(32, 3)), rng.uniform(0.5, 3.0, size=(32, 3))])
    hl = np.zeros(hs.shape[0])
    ref.ref_hess_lmax(hs.shape[0], po._d(np.ascontiguousarray(hs)), mu, lam, po._d(hl))
    np.savez_compressed(os.path.join(HERE, "elem_cases.npz"), F=Fc, sigma=sig, U=U, V=V, mu=mu, lam=lam,
                        prox_s0=s0, prox_wov=wov, prox_start=start, prox_out=out, prox_iters=its,
                        vg_x=xv, vg_value=val, vg_grad=grad, hess_sigma=hs, hess_lmax=hl)


def tiny_step(ref):
    b = bars.make_bar(2, 2, 6, twist_deg=90.0, noise=0.05, seed=3)
    rng = np.random.default_rng(11)
    X2 = b.init + 0.01 * b.h * rng.normal(size=b.init.shape)
    X2[b.pins] = b.init[b.pins]
    nf = b.n_verts - len(b.pins)
    dal, val, pe = np.zeros(1), np.zeros(1), np.zeros(1)
    flips = np.zeros(1, dtype=np.int32)
    g, g2 = np.zeros((nf, 3)), np.zeros((nf, 3))
    rest, init, X2c = (np.ascontiguousarray(a) for a in (b.rest, b.init, X2))
    tets = np.ascontiguousarray(b.tets, dtype=np.int32)
    pins = np.ascontiguousarray(b.pins, dtype=np.int32)
    ref.ref_local_and_grad(b.n_verts, po._d(rest), po._d(init), po._d(X2c), b.n_tets, tets.ctypes.data_as(po._ip),
                           len(pins), pins.ctypes.data_as(po._ip), E_YOUNG, NU, po._d(dal), po._d(g), po._d(val),
                           po._d(pe), flips.ctypes.data_as(po._ip), po._d(g2))
    np.savez_compressed(os.path.join(HERE, "tiny_step.npz"), rest=b.rest, init=b.init, X2=X2, tets=b.tets,
                        pins=b.pins, dal=dal[0], grad=g, value=val[0], pe=pe[0], flips=flips[0], grad2=g2)


def ref_solve(bar, max_iters, extra=(), binary=po.QUASI_REF):
    with tempfile.TemporaryDirectory() as d:
        files = bars.write_bar(bar, d, "m")
        return po.run_quasi_ref(files, E_YOUNG, NU, max_iters, threads=1, extra=list(extra), outdir=d + "/out",
                                timeout=24 * 3600, binary=binary)


def bar_32x32x128_bent():
    """The benchmarked bar against the reference itself, both builds."""
    import concurrent.futures as cf
    b = bars.bar_32x32x128_bent()
    out = {}
    runs = [("m5", 20, ("-rw_every", "10"), po.QUASI_REF_M5), ("m6", 60, (), po.QUASI_REF)]
    with cf.ThreadPoolExecutor(len(runs)) as ex:   # two single-thread processes side by side
        results = list(ex.map(lambda a: ref_solve(b, a[1], a[2], a[3]), runs))
    # positions: a seeded sample of vertices, the column sums and max |x| (the
    # whole 140,481 x 3 array would make a 7 MB fixture)
    idx = np.sort(np.random.default_rng(32128).choice(b.n_verts, X_SAMPLE, replace=False))
    for (tag, _, _, _), r in zip(runs, results):
        X = np.asarray(r["x"]).reshape(-1, 3)
        out.update({f"{tag}_objectives": r["objectives"], f"{tag}_inner": r["inner_iters"],
                    f"{tag}_reweighted": r["reweighted"], f"{tag}_x_sample": X[idx],
                    f"{tag}_x_colsum": X.sum(axis=0), f"{tag}_x_absmax": np.abs(X).max(),
                    f"{tag}_ls_dal": r["ls_delta_al"], f"{tag}_gs_dal": r["gs_delta_al"],
                    f"{tag}_setup_ms": r["runtime"]["setup_ms"],
                    f"{tag}_acc_time_s": r["accumulated_time_s"]})
        print(tag, "done:", r["runtime"], flush=True)
    np.savez_compressed(os.path.join(HERE, "solve_bar_32x32x128_bent.npz"), x_idx=idx, **out)


def solves():
    out = {}
    small = bars.make_bar(3, 3, 10, twist_deg=120.0, noise=0.03, seed=5)
    for tag, bar, extra, it in [("a", small, (), 300), ("b", small, ("-rw_delay", "5"), 300)]:
        r = ref_solve(bar, it, extra)
        out.update({f"{tag}_objectives": r["objectives"], f"{tag}_inner": r["inner_iters"],
                    f"{tag}_reweighted": r["reweighted"], f"{tag}_x": r["x"],
                    f"{tag}_ls_dal": r["ls_delta_al"], f"{tag}_gs_dal": r["gs_delta_al"]})
    np.savez_compressed(os.path.join(HERE, "solve_small.npz"), rest=small.rest, init=small.init,
                        tets=small.tets, pins=small.pins, **out)
    c0 = bars.bar_8x8x32()
    r = ref_solve(c0, 500)
    np.savez_compressed(os.path.join(HERE, "solve_bar_8x8x32.npz"), objectives=r["objectives"],
                        inner=r["inner_iters"], reweighted=r["reweighted"], x=r["x"],
                        ls_dal=r["ls_delta_al"], gs_dal=r["gs_delta_al"])


def modes():
    b = bars.make_bar(3, 3, 8, twist_deg=90.0, noise=0.02, seed=5)
    out = {}
    for tag, extra in [("ra0", ("-ra", "0")), ("arap", ("-model", "arap", "-rw", "0")),
                       ("arap_ra0", ("-model", "arap", "-rw", "0", "-ra", "0"))]:
        r = ref_solve(b, 60, extra)
        out.update({f"{tag}_objectives": r["objectives"], f"{tag}_inner": r["inner_iters"],
                    f"{tag}_reweighted": r["reweighted"], f"{tag}_x": r["x"],
                    f"{tag}_ls_dal": r["ls_delta_al"], f"{tag}_gs_dal": r["gs_delta_al"]})
    np.savez_compressed(os.path.join(HERE, "solve_modes.npz"), rest=b.rest, init=b.init, tets=b.tets,
                        pins=b.pins, **out)


def global_ls():
    b = bars.make_bar(3, 3, 8, twist_deg=720.0, noise=0.4, seed=7)
    r = ref_solve(b, 80, ("-global_ls", "1", "-rw", "0"))
    np.savez_compressed(os.path.join(HERE, "solve_gls.npz"), rest=b.rest, init=b.init, tets=b.tets, pins=b.pins,
                        objectives=r["objectives"], inner=r["inner_iters"], reweighted=r["reweighted"], x=r["x"],
                        ls_dal=r["ls_delta_al"], gs_dal=r["gs_delta_al"])


def quasi_files():
    b = bars.make_bar(3, 3, 8, twist_deg=90.0, noise=0.02, seed=5)
    out = {}
    with tempfile.TemporaryDirectory() as d:
        files = bars.write_bar(b, d, "q")
        for tag, extra, it in [("plain", (), 40), ("soln", ("-soln", d + "/plain/final_mesh"), 200)]:
            od = os.path.join(d, tag)
            po.run_quasi_ref(files, E_YOUNG, NU, it, threads=1, extra=list(extra), outdir=od)
            for name in ("objectives", "x_errors", "reweighted", "final_mesh.node", "final_mesh.ele",
                         "final_mesh.obj"):
                fn = os.path.join(od, name if "." in name else name + ".txt")
                out[f"{tag}/{name}"] = np.frombuffer(open(fn, "rb").read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "quasi_small.npz"), **out)




def bar_64x64x160():
    """Three oracle iterations on the 3.9M-tet bar (the oracle, not the reference:
    see the module docstring)."""
    b = bars.bar_64x64x160()
    o = po.Oracle(b.rest, b.init, b.tets, b.pins, youngs=E_YOUNG, poisson=NU, max_iters=3, lbfgs_m=5, rw_every=20,
                  linear_solver=1)
    o.solve()
    X = o.get("X").reshape(-1, 3)
    idx = np.sort(np.random.default_rng(64160).choice(b.n_verts, X_SAMPLE, replace=False))
    np.savez_compressed(os.path.join(HERE, "iters_bar_64x64x160.npz"), objectives=o.get("objectives"),
                        inner=o.get("inner_iters").astype(np.int32), flips=o.get("flips").astype(np.int32),
                        ls_dal=o.get("ls_dal"), gs_dal=o.get("gs_dal"), x_idx=idx, x_sample=X[idx],
                        x_colsum=X.sum(axis=0), x_absmax=np.abs(X).max())


def main():
    if not po.ref_available():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` (needs the reference sources)")
    if sys.argv[1:] == ["--only", "modes"]:
        modes()
        print("golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["--only", "gls"]:
        global_ls()
        print("golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["--only", "bar_64x64x160"]:
        bar_64x64x160()
        print("golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["--only", "bar_32x32x128_bent"]:
        bar_32x32x128_bent()
        print("golden vectors written to", HERE)
        return
    if sys.argv[1:] == ["--only", "quasi"]:
        quasi_files()
        print("golden vectors written to", HERE)
        return
    ref = po.load_ref_elem()
    rng = np.random.default_rng(20240611)
    elem_cases(ref, rng)
    tiny_step(ref)
    solves()
    modes()
    global_ls()
    quasi_files()
    bar_32x32x128_bent()
    bar_64x64x160()
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
