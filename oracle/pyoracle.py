"""ctypes bindings for the oracle (test infrastructure; see ``oracle/__init__.py``)."""
from __future__ import annotations

import ctypes
import dataclasses
import os
import subprocess
import tempfile

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
LIBORACLE = os.path.join(ORACLE_DIR, "liboracle.so")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")
QUASI_REF = os.path.join(REF_DIR, "quasi_ref")
# The patched build (oracle/Makefile): global L-BFGS history 5, `-rw_every N`.
QUASI_REF_M5 = os.path.join(REF_DIR, "quasi_ref_m5")
LIBREF_ELEM = os.path.join(REF_DIR, "libref_elem.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class OracleProblem(ctypes.Structure):
    _fields_ = [("n_verts", ctypes.c_int), ("n_tets", ctypes.c_int), ("n_pins", ctypes.c_int),
                ("rest", _dp), ("init", _dp), ("tets", _ip), ("pins", _ip),
                ("youngs", ctypes.c_double), ("poisson", ctypes.c_double),
                ("max_iters", ctypes.c_int), ("tol", ctypes.c_double), ("lbfgs_m", ctypes.c_int),
                ("global_iters", ctypes.c_int), ("kappa", ctypes.c_double),
                ("reweighting", ctypes.c_int), ("rw_delay", ctypes.c_int), ("gamma", ctypes.c_double),
                ("beta_static", ctypes.c_double), ("beta_min", ctypes.c_double),
                ("beta_max", ctypes.c_double), ("rw_every", ctypes.c_int),
                ("youngs_e", _dp), ("poisson_e", _dp), ("rot_aware", ctypes.c_int), ("model", ctypes.c_int),
                ("global_ls", ctypes.c_int), ("linear_solver", ctypes.c_int)]


_lib = None


def load_oracle():
    """Load (building if needed) the C restatement."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBORACLE):
        subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
    lib = ctypes.CDLL(LIBORACLE)
    lib.orc_svd3.argtypes = [_dp, _dp, _dp, _dp]
    lib.orc_nh_psi.restype = ctypes.c_double
    lib.orc_nh_psi.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
    lib.orc_nh_psi_plain.restype = ctypes.c_double
    lib.orc_nh_psi_plain.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
    lib.orc_prox_value_grad.restype = ctypes.c_double
    lib.orc_prox_value_grad.argtypes = [ctypes.c_double, ctypes.c_double, _dp, ctypes.c_double, _dp, _dp]
    lib.orc_prox_lbfgs.restype = ctypes.c_int
    lib.orc_prox_lbfgs.argtypes = [ctypes.c_double, ctypes.c_double, _dp, ctypes.c_double, _dp, ctypes.c_int]
    lib.orc_hess_lmax.restype = ctypes.c_double
    lib.orc_hess_lmax.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
    lib.orc_problem_defaults.argtypes = [ctypes.POINTER(OracleProblem)]
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.POINTER(OracleProblem), _ip]
    lib.orc_destroy.argtypes = [ctypes.c_void_p]
    for f in ("orc_setup", "orc_iterate", "orc_solve", "orc_n_free", "orc_iters", "orc_inversion_count"):
        getattr(lib, f).restype = ctypes.c_int
        getattr(lib, f).argtypes = [ctypes.c_void_p]
    lib.orc_get.restype = ctypes.c_long
    lib.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
    lib.orc_set.restype = ctypes.c_int
    lib.orc_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
    lib.orc_update_defo_cache.argtypes = [ctypes.c_void_p]
    lib.orc_init_state.argtypes = [ctypes.c_void_p]
    lib.orc_polar_update.restype = ctypes.c_double
    lib.orc_polar_update.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.orc_global_grad_cached.restype = ctypes.c_double
    lib.orc_global_grad_cached.argtypes = [ctypes.c_void_p, _dp]
    lib.orc_global_grad.restype = ctypes.c_double
    lib.orc_global_grad.argtypes = [ctypes.c_void_p, _dp, _dp]
    lib.orc_potential_energy.restype = ctypes.c_double
    lib.orc_potential_energy.argtypes = [ctypes.c_void_p]
    lib.orc_solve_A.argtypes = [ctypes.c_void_p, _dp, _dp]
    _lib = lib
    return lib


def lame(youngs: float, poisson: float):
    """mu, lambda from (E, nu), src/Lame.hpp:50-53."""
    return youngs / (2.0 * (1.0 + poisson)), youngs * poisson / ((1.0 + poisson) * (1.0 - 2.0 * poisson))


class Oracle:
    """One oracle solver instance over a mesh (rest, init, tets, pins)."""

    def __init__(self, rest, init, tets, pins, youngs=1e5, poisson=0.45, max_iters=500, tol=1e-11,
                 lbfgs_m=6, reweighting=1, rw_delay=50, gamma=1.5, rw_every=0, global_iters=100,
                 kappa=1.0, beta_static=1.0, beta_min=0.1, beta_max=10.0, youngs_e=None, poisson_e=None,
                 rot_aware=1, model=0, global_ls=0, linear_solver=0):
        """youngs_e / poisson_e: per-element material (a batch of meshes), or None.
        linear_solver = 1: conjugate gradients in place of the envelope LDL^T (large meshes)."""
        self.lib = load_oracle()
        self._keep = [np.ascontiguousarray(rest, dtype=np.float64),
                      np.ascontiguousarray(init, dtype=np.float64),
                      np.ascontiguousarray(tets, dtype=np.int32),
                      np.ascontiguousarray(pins, dtype=np.int32)]
        p = OracleProblem()
        self.lib.orc_problem_defaults(ctypes.byref(p))
        p.n_verts, p.n_tets, p.n_pins = self._keep[0].shape[0], self._keep[2].shape[0], self._keep[3].shape[0]
        p.rest, p.init = _d(self._keep[0]), _d(self._keep[1])
        p.tets, p.pins = _i(self._keep[2]), _i(self._keep[3])
        p.youngs, p.poisson, p.max_iters, p.tol, p.lbfgs_m = youngs, poisson, max_iters, tol, lbfgs_m
        p.reweighting, p.rw_delay, p.gamma, p.rw_every = reweighting, rw_delay, gamma, rw_every
        p.global_iters, p.kappa = global_iters, kappa
        p.beta_static, p.beta_min, p.beta_max = beta_static, beta_min, beta_max
        p.rot_aware, p.model, p.global_ls = rot_aware, model, global_ls
        p.linear_solver = linear_solver
        if youngs_e is not None:
            self._keep += [np.ascontiguousarray(youngs_e, dtype=np.float64),
                           np.ascontiguousarray(poisson_e, dtype=np.float64)]
            p.youngs_e, p.poisson_e = _d(self._keep[-2]), _d(self._keep[-1])
        self.problem = p
        err = ctypes.c_int(0)
        self.h = self.lib.orc_create(ctypes.byref(p), ctypes.byref(err))
        if not self.h:
            raise ValueError(f"oracle rejected the problem (code {err.value})")
        self.mu, self.lam = lame(youngs, poisson)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def n_free(self):
        return self.lib.orc_n_free(self.h)

    @property
    def iters(self):
        return self.lib.orc_iters(self.h)

    def setup(self):
        rc = self.lib.orc_setup(self.h)
        if rc < 0:
            raise RuntimeError(f"oracle setup failed ({rc})")

    def iterate(self):
        rc = self.lib.orc_iterate(self.h)
        if rc < 0:
            raise RuntimeError(f"oracle iterate failed ({rc})")
        return rc == 1

    def solve(self):
        rc = self.lib.orc_solve(self.h)
        if rc < 0:
            raise RuntimeError(f"oracle solve failed ({rc})")
        return rc

    def get(self, name: str) -> np.ndarray:
        n = self.lib.orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.empty(max(n, 0), dtype=np.float64)
        if n:
            self.lib.orc_get(self.h, name.encode(), _d(out))
        return out

    def set(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        if self.lib.orc_set(self.h, name.encode(), _d(a)) != 0:
            raise KeyError(name)

    def init_state(self):
        self.lib.orc_init_state(self.h)

    def update_defo_cache(self):
        self.lib.orc_update_defo_cache(self.h)

    def polar_update(self, update_candidates=True) -> float:
        return self.lib.orc_polar_update(self.h, int(update_candidates))

    def grad_cached(self):
        g = np.zeros(3 * self.n_free)
        v = self.lib.orc_global_grad_cached(self.h, _d(g))
        return v, g.reshape(-1, 3)

    def grad(self, xfree):
        x = np.ascontiguousarray(xfree, dtype=np.float64).ravel()
        g = np.zeros(3 * self.n_free)
        v = self.lib.orc_global_grad(self.h, _d(x), _d(g))
        return v, g.reshape(-1, 3)

    def potential_energy(self) -> float:
        return self.lib.orc_potential_energy(self.h)

    def inversion_count(self) -> int:
        return self.lib.orc_inversion_count(self.h)

    def solve_A(self, b):
        bb = np.ascontiguousarray(b, dtype=np.float64).ravel()
        x = np.empty_like(bb)
        self.lib.orc_solve_A(self.h, _d(bb), _d(x))
        return x.reshape(-1, 3)


# ---- the reference itself ------------------------------------------------------
def ref_available() -> bool:
    return os.path.exists(QUASI_REF) and os.path.exists(LIBREF_ELEM)


_ref = None


def load_ref_elem():
    """The reference's per-element code (oracle/_ref/libref_elem.so)."""
    global _ref
    if _ref is not None:
        return _ref
    lib = ctypes.CDLL(LIBREF_ELEM)
    lib.ref_svd3.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp]
    lib.ref_prox.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _ip]
    lib.ref_prox_value_grad.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp, _dp]
    lib.ref_hess_lmax.argtypes = [ctypes.c_int, _dp, ctypes.c_double, ctypes.c_double, _dp]
    lib.ref_local_and_grad.argtypes = [ctypes.c_int, _dp, _dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                       ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, _ip, _dp,
                                       _dp, _dp, _dp]
    _ref = lib
    return lib


def run_quasi_ref(bar_files: dict, youngs: float, poisson: float, max_iters: int, threads: int = 1,
                  extra=(), outdir: str | None = None, timeout: float = 3600, binary: str = QUASI_REF):
    """Run the reference solver on .node/.ele/handles files; returns its logs.
    binary = QUASI_REF_M5 runs the patched build (history 5, -rw_every)."""
    out = outdir or tempfile.mkdtemp(prefix="quasi_ref_")
    os.makedirs(out, exist_ok=True)
    cmd = [binary, "-rest", bar_files["rest"], "-init", bar_files["init"], "-handles", bar_files["handles"],
           "-youngs", repr(float(youngs)), "-poisson", repr(float(poisson)), "-it", str(int(max_iters)),
           "-p", "0", "-out", out, *extra]
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    subprocess.run(cmd, check=True, capture_output=True, env=env, timeout=timeout)
    res = {}
    for name in ("objectives", "x_errors", "reweighted", "accumulated_time_s", "inner_iters",
                 "ls_delta_al", "gs_delta_al"):
        path = os.path.join(out, name + ".txt")
        a = np.loadtxt(path, ndmin=2) if os.path.getsize(path) else np.zeros((0, 2))
        res[name] = a[:, 1] if a.size else np.zeros(0)
    res["x"] = np.fromfile(os.path.join(out, "final_x.bin"), dtype=np.float64).reshape(-1, 3)
    rt = {}
    with open(os.path.join(out, "runtime.txt")) as f:
        for line in f:
            k, v = line.split()
            rt[k] = float(v)
    res["runtime"] = rt
    res["outdir"] = out
    return res
