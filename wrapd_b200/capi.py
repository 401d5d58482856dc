"""ctypes binding of the C ABI in include/wrapd_gpu.h (libwrapd_gpu.so).

The library is loaded from the package's in-tree build (``wrapd_b200/_lib``).
There is no CPU fallback: if the library is missing, or the CUDA device is
unusable, every call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libwrapd_gpu.so")

WRAPD_OK = 0
ERRORS = {
    -1: "WRAPD_E_INPUT", -2: "WRAPD_E_INVERTED_REST", -3: "WRAPD_E_NOT_SPD", -4: "WRAPD_E_NAN",
    -5: "WRAPD_E_PROX_NEG", -6: "WRAPD_E_TIMEOUT", -7: "WRAPD_E_OOM", -8: "WRAPD_E_CUDA",
    -9: "WRAPD_E_STATE", -10: "WRAPD_E_UNSUPPORTED",
}
globals().update({name: code for code, name in ERRORS.items()})   # WRAPD_E_INPUT = -1, ...
LOGS = {"objectives": 0, "reweighted": 1, "flips": 2, "inner_iters": 3, "ls_delta_al": 4,
        "gs_delta_al": 5, "accumulated_time_s": 6, "x_errors": 7, "prox_iters": 8}
NET_BLOB = 4755


class WrapdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code
        self.name = ERRORS.get(code, str(code))


class Settings(ctypes.Structure):
    """wrapd_settings; field meanings as in include/wrapd_gpu.h."""
    _fields_ = [("max_iters", ctypes.c_int), ("tol", ctypes.c_double), ("rot_aware", ctypes.c_int),
                ("reweighting", ctypes.c_int), ("rw_delay", ctypes.c_int), ("gamma", ctypes.c_double),
                ("global_iters", ctypes.c_int), ("global_ls", ctypes.c_int), ("kappa", ctypes.c_double),
                ("model", ctypes.c_int), ("poisson", ctypes.c_double), ("beta_static", ctypes.c_double),
                ("beta_min", ctypes.c_double), ("beta_max", ctypes.c_double), ("prox_iters", ctypes.c_int),
                ("youngs", ctypes.c_double), ("lbfgs_m", ctypes.c_int), ("rw_every", ctypes.c_int),
                ("precision", ctypes.c_int), ("prox_mode", ctypes.c_int), ("leaf_size", ctypes.c_int),
                ("verbose", ctypes.c_int), ("device", ctypes.c_int),
                ("autotune", ctypes.c_int)]


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_fp = ctypes.POINTER(ctypes.c_float)
_lib = None

# (name, restype, argtypes) for every entry point of include/wrapd_gpu.h
SIGNATURES = [
    ("wrapd_settings_default", ctypes.c_int, [ctypes.POINTER(Settings)]),
    ("wrapd_create", ctypes.c_int, [ctypes.POINTER(Settings), ctypes.POINTER(ctypes.c_void_p)]),
    ("wrapd_add_tetmesh", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int, _ip, ctypes.c_int, _ip,
                                          ctypes.c_int]),
    ("wrapd_add_tetmesh_material", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int, _ip, ctypes.c_int,
                                                   _ip, ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    ("wrapd_initialize", ctypes.c_int, [ctypes.c_void_p]),
    ("wrapd_solve", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("wrapd_begin_solve", ctypes.c_int, [ctypes.c_void_p]),
    ("wrapd_iterate", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_get_positions", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("wrapd_get_log", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_get_mesh_log", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_get_runtime", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("wrapd_get_info", ctypes.c_int, [ctypes.c_void_p, _dp]),
    ("wrapd_get_counters", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    ("wrapd_set_profiling", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("wrapd_get_profile", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int64)]),
    ("wrapd_get_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("wrapd_destroy", None, [ctypes.c_void_p]),
    ("wrapd_get_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _dp, ctypes.c_int64,
                                        ctypes.POINTER(ctypes.c_int64)]),
    ("wrapd_set_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, _dp, ctypes.c_int64]),
    ("wrapd_update_defo_cache", ctypes.c_int, [ctypes.c_void_p]),
    ("wrapd_polar_update", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    ("wrapd_global_grad", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp]),
    ("wrapd_potential_energy", ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_solve_A", ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    ("wrapd_solve_A_holding", ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    ("wrapd_svd3_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp]),
    ("wrapd_prox_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                         _dp, _dp, _dp, _dp, _ip]),
    ("wrapd_hess_lmax_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp]),
    ("wrapd_potential_energy_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp,
                                                     ctypes.POINTER(ctypes.c_int)]),
    ("wrapd_potential_energy_batch_noalloc", ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                             ctypes.c_void_p]),
    ("wrapd_prox_newton_batch", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp, _ip]),
    ("wrapd_net_create", ctypes.c_int, [_fp, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    ("wrapd_net_set_data", ctypes.c_int, [ctypes.c_void_p, _fp, _fp, ctypes.c_int64]),
    ("wrapd_net_train", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                        ctypes.c_uint64, _dp]),
    ("wrapd_net_grad", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, _dp, _fp]),
    ("wrapd_net_get", ctypes.c_int, [ctypes.c_void_p, _fp]),
    ("wrapd_net_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("wrapd_net_destroy", None, [ctypes.c_void_p]),
    ("wrapd_net_predict", ctypes.c_int, [_fp, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_double,
                                          ctypes.c_double, _dp]),
    ("wrapd_set_prox_net", ctypes.c_int, [ctypes.c_void_p, _fp, ctypes.c_int]),
    ("wrapd_dmma_peak", ctypes.c_int, [ctypes.c_int, _dp]),
    ("wrapd_plan_create", ctypes.c_int, [_dp, ctypes.c_int, _ip, ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    ("wrapd_plan_info", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    ("wrapd_plan_fronts", ctypes.c_int, [ctypes.c_void_p, _ip, _ip, _ip, _ip, _ip, ctypes.POINTER(ctypes.c_int64),
                                          _ip, _ip]),
    ("wrapd_plan_destroy", None, [ctypes.c_void_p]),
]


def _check_free(rc: int):
    if rc != WRAPD_OK:
        raise WrapdError(rc, "batch call failed")


def svd3_batch(F, fp32: bool = False):
    """math::svd on n x 9 column-major matrices; returns (sigma, U, V)."""
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 9)
    n = F.shape[0]
    s, U, V = np.empty((n, 3)), np.empty((n, 9)), np.empty((n, 9))
    _check_free(load().wrapd_svd3_batch(n, int(fp32), dptr(F), dptr(s), dptr(U), dptr(V)))
    return s, U, V


def prox_batch(mu, lam, sigma0, wov, start, max_iters: int = 20, fp32: bool = False):
    """The NH prox per element; returns (stretches, iteration counts)."""
    s0 = np.ascontiguousarray(sigma0, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(wov, dtype=np.float64).ravel()
    st = np.ascontiguousarray(start, dtype=np.float64).reshape(-1, 3)
    n = s0.shape[0]
    out, its = np.empty((n, 3)), np.empty(n, dtype=np.int32)
    _check_free(load().wrapd_prox_batch(n, int(fp32), mu, lam, max_iters, dptr(s0), dptr(w), dptr(st), dptr(out),
                                        iptr(its)))
    return out, its


def prox_newton_batch(mu, lam, sigma0, wov, start, tol: float = 1e-10, max_iters: int = 100, fp32: bool = False):
    """The Newton prox per element; returns (stretches, iteration counts)."""
    s0 = np.ascontiguousarray(sigma0, dtype=np.float64).reshape(-1, 3)
    w = np.ascontiguousarray(wov, dtype=np.float64).ravel()
    st = np.ascontiguousarray(start, dtype=np.float64).reshape(-1, 3)
    n = s0.shape[0]
    out, its = np.empty((n, 3)), np.empty(n, dtype=np.int32)
    _check_free(load().wrapd_prox_newton_batch(n, int(fp32), mu, lam, tol, max_iters, dptr(s0), dptr(w), dptr(st),
                                               dptr(out), iptr(its)))
    return out, its


def potential_energy_batch(mu, lam, sigma, vol):
    """(sum vol * psi(sigma), inverted count) over a batch of stretch triples."""
    s = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(vol, dtype=np.float64).ravel()
    pe, fl = ctypes.c_double(0.0), ctypes.c_int(0)
    _check_free(load().wrapd_potential_energy_batch(s.shape[0], mu, lam, dptr(s), dptr(v), ctypes.byref(pe),
                                                    ctypes.byref(fl)))
    return pe.value, fl.value


def hess_lmax_batch(mu, lam, sigma):
    s = np.ascontiguousarray(sigma, dtype=np.float64).reshape(-1, 3)
    out = np.empty(s.shape[0])
    _check_free(load().wrapd_hess_lmax_batch(s.shape[0], mu, lam, dptr(s), dptr(out)))
    return out


def dmma_peak(iters: int = 20000) -> float:
    """Measured FP64 tensor-core throughput (TFLOP/s)."""
    v = ctypes.c_double(0.0)
    _check_free(load().wrapd_dmma_peak(iters, ctypes.byref(v)))
    return v.value


PLAN_INFO = ("n_free", "fronts", "levels", "nnz_L", "f_pool_bytes", "y_pool_bytes", "total_rows", "flops")


def plan(rest, tets, pins, leaf_size: int = 0) -> dict:
    """Host-only symbolic analysis of one mesh (wrapd_plan_*; needs no GPU):
    the sizes of PLAN_INFO, the order `perm` (free index per new column) and
    per front `first`, `ncols`, `parent`, `level`, `row_ptr`, `rows`, `relmap`."""
    lib = load()
    X = np.ascontiguousarray(rest, dtype=np.float64).reshape(-1, 3)
    T = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
    P = np.ascontiguousarray(pins, dtype=np.int32).ravel()
    h = ctypes.c_void_p()
    rc = lib.wrapd_plan_create(dptr(X), X.shape[0], iptr(T), T.shape[0], iptr(P), P.size, leaf_size,
                               ctypes.byref(h))
    if rc != WRAPD_OK:
        raise WrapdError(rc, lib.wrapd_last_error(None).decode())
    try:
        info = np.zeros(8, dtype=np.int64)
        lib.wrapd_plan_info(h, info.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        out = dict(zip(PLAN_INFO, (int(v) for v in info)))
        nf, nfr, nr = out["n_free"], out["fronts"], out["total_rows"]
        arr = {k: np.zeros(n, dtype=np.int32) for k, n in
               (("perm", nf), ("first", nfr), ("ncols", nfr), ("parent", nfr), ("level", nfr), ("rows", nr),
                ("relmap", nr))}
        arr["row_ptr"] = np.zeros(nfr + 1, dtype=np.int64)
        _check_free(lib.wrapd_plan_fronts(h, iptr(arr["perm"]), iptr(arr["first"]), iptr(arr["ncols"]),
                                          iptr(arr["parent"]), iptr(arr["level"]),
                                          arr["row_ptr"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                          iptr(arr["rows"]), iptr(arr["relmap"])))
        out.update(arr)
        return out
    finally:
        lib.wrapd_plan_destroy(h)


def load():
    """Load libwrapd_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing; build it with `python -m wrapd_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def fptr(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def default_settings() -> Settings:
    s = Settings()
    load().wrapd_settings_default(ctypes.byref(s))
    return s


class Handle:
    """Owns one wrapd_handle (one mesh, one CUDA stream)."""

    def __init__(self, settings: Settings):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.wrapd_create(ctypes.byref(settings), ctypes.byref(h))
        if rc != WRAPD_OK:
            raise WrapdError(rc, self.lib.wrapd_last_error(None).decode())
        self.h = h

    def check(self, rc: int):
        if rc != WRAPD_OK:
            raise WrapdError(rc, self.lib.wrapd_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.wrapd_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()
