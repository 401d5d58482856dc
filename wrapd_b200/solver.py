"""Python mirror of the reference's solver interface over the C ABI.

``Solver`` follows wrapd::Solver (src/Solver.hpp:37-72): construct with a
``Settings``, add a tet mesh (binding::add_tetmesh,
samples/utils/AddMeshes.hpp:61-132), ``set_pins``, ``initialize``, ``solve``,
then read ``algorithm_data()`` (AlgorithmData, src/AlgorithmData.hpp:43-73)
and the final positions.  Errors raise ``WrapdError`` where the reference
throws ``std::runtime_error`` or calls ``exit(0)``.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import capi
from .capi import WrapdError


def Settings(**kw) -> capi.Settings:
    """wrapd::Settings defaults (src/Settings.hpp:154-162) with overrides.

    Reference flag names are accepted as aliases: it, tol, ra, rw, rw_delay,
    gamma, global_it, global_ls, kappa, poisson, beta_static, beta_min,
    beta_max; extensions: youngs, lbfgs_m, rw_every, precision, prox_mode,
    leaf_size, device.
    """
    alias = {"it": "max_iters", "ra": "rot_aware", "rw": "reweighting", "global_it": "global_iters"}
    s = capi.default_settings()
    for k, v in kw.items():
        k = alias.get(k, k)
        if k == "precision" and isinstance(v, str):
            v = {"fp64": 0, "mixed": 1}[v]
        if not hasattr(s, k):
            raise ValueError(f"unknown setting {k}")
        setattr(s, k, v)
    return s


@dataclasses.dataclass
class AlgorithmData:
    objectives: np.ndarray
    reweighted: np.ndarray
    flips: np.ndarray
    inner_iters: np.ndarray
    ls_delta_al: np.ndarray
    gs_delta_al: np.ndarray
    accumulated_time_s: np.ndarray
    x_errors: np.ndarray
    prox_iters: np.ndarray
    runtime_ms: dict


class Solver:
    def __init__(self, settings: capi.Settings | None = None, **kw):
        self.settings = settings if settings is not None else Settings(**kw)
        self._h = capi.Handle(self.settings)
        self.n_verts = 0
        self._meshes = []

    # -- mesh ---------------------------------------------------------------
    def add_tetmesh(self, rest, init, tets, soln=None, pins=None, youngs=None, poisson=None):
        """Add a mesh; call again for a batch (meshes solved as one block-diagonal
        system, positions returned in the order added).  youngs/poisson give this
        mesh its own material (both or neither)."""
        rest = np.ascontiguousarray(rest, dtype=np.float64).reshape(-1, 3)
        init = np.ascontiguousarray(init, dtype=np.float64).reshape(-1, 3)
        tets = np.ascontiguousarray(tets, dtype=np.int32).reshape(-1, 4)
        if rest.shape != init.shape:
            raise WrapdError(-1, "Rest mesh and init mesh do not have the same number of vertices.")
        if (youngs is None) != (poisson is None):
            raise ValueError("give both youngs and poisson, or neither")
        soln = None if soln is None else np.ascontiguousarray(soln, dtype=np.float64).reshape(-1, 3)
        self._meshes.append(dict(rest=rest, init=init, tets=tets, soln=soln, pins=None, youngs=youngs,
                                 poisson=poisson))
        if pins is not None:
            self.set_pins(pins)
        self.n_verts += rest.shape[0]

    def set_pins(self, inds):
        """Pin vertices of the last added mesh in place (src/System.cpp:33-44)."""
        if not self._meshes:
            raise WrapdError(-9, "set_pins before add_tetmesh")
        self._meshes[-1]["pins"] = np.ascontiguousarray(inds, dtype=np.int32).ravel()

    def initialize(self):
        if not self._meshes:
            raise WrapdError(-9, "initialize before add_tetmesh")
        h = self._h
        for m in self._meshes:
            pins = m["pins"] if m["pins"] is not None else np.zeros(0, dtype=np.int32)
            args = (h.h, capi.dptr(m["rest"]), capi.dptr(m["init"]),
                    capi.dptr(m["soln"]) if m["soln"] is not None else None, m["rest"].shape[0],
                    capi.iptr(m["tets"]), m["tets"].shape[0], capi.iptr(pins), pins.shape[0])
            if m["youngs"] is None:
                h.check(h.lib.wrapd_add_tetmesh(*args))
            else:
                h.check(h.lib.wrapd_add_tetmesh_material(*args, float(m["youngs"]), float(m["poisson"])))
        h.check(h.lib.wrapd_initialize(h.h))
        return True

    # -- solve --------------------------------------------------------------
    def solve(self) -> np.ndarray:
        x = np.empty((self.n_verts, 3))
        self._h.check(self._h.lib.wrapd_solve(self._h.h, capi.dptr(x)))
        self.X = x
        return x

    def begin_solve(self):
        self._h.check(self._h.lib.wrapd_begin_solve(self._h.h))

    def iterate(self, n: int = 1):
        done, conv = ctypes.c_int(0), ctypes.c_int(0)
        self._h.check(self._h.lib.wrapd_iterate(self._h.h, n, ctypes.byref(done), ctypes.byref(conv)))
        return done.value, bool(conv.value)

    def positions(self) -> np.ndarray:
        x = np.empty((self.n_verts, 3))
        self._h.check(self._h.lib.wrapd_get_positions(self._h.h, capi.dptr(x)))
        return x

    # -- data ---------------------------------------------------------------
    def log(self, name: str, mesh: int | None = None) -> np.ndarray:
        """AlgorithmData log `name`; of a batch, the batch summary, or with
        mesh = m the log of the m-th mesh added (its own solve)."""
        n = ctypes.c_int(0)
        h = self._h

        def get(out, cap):
            if mesh is None:
                return h.lib.wrapd_get_log(h.h, capi.LOGS[name], out, cap, ctypes.byref(n))
            return h.lib.wrapd_get_mesh_log(h.h, int(mesh), capi.LOGS[name], out, cap, ctypes.byref(n))
        h.check(get(None, 0))
        out = np.empty(n.value)
        if n.value:
            h.check(get(capi.dptr(out), n.value))
        return out

    def runtime(self) -> dict:
        ms = np.zeros(6)
        self._h.check(self._h.lib.wrapd_get_runtime(self._h.h, capi.dptr(ms)))
        return dict(zip(["setup_ms", "local_ms", "global_ms", "refactor_ms", "finish_ms", "inner_iters"], ms))

    def info(self) -> dict:
        v = np.zeros(8)
        self._h.check(self._h.lib.wrapd_get_info(self._h.h, capi.dptr(v)))
        return dict(zip(["n_verts", "n_tets", "n_free", "n_pins", "fronts", "levels", "nnz_L", "factor_flops"], v))

    def counters(self) -> dict:
        v = (ctypes.c_int64 * 4)()
        self._h.check(self._h.lib.wrapd_get_counters(self._h.h, v))
        return dict(zip(["kernel_launches", "factorizations", "solves", "host_syncs"], list(v)))

    def tuning(self) -> dict:
        """Tile shapes in use (wrapd_get_tuning): the fused panel-step limit, the
        solve chunk length per level and direction, the local step's tile."""
        n = ctypes.c_int(0)
        self._h.check(self._h.lib.wrapd_get_tuning(self._h.h, None, 0, ctypes.byref(n)))
        out = (ctypes.c_int * n.value)()
        self._h.check(self._h.lib.wrapd_get_tuning(self._h.h, out, n.value, ctypes.byref(n)))
        v = list(out)
        L = v[1]
        return {"fused_panel_ctas": v[0], "levels": L, "solve_chunk_fwd": v[2:2 + L],
                "solve_chunk_bwd": v[2 + L:2 + 2 * L], "local_tile": v[2 + 2 * L]}

    def set_prox_net(self, blob):
        """Install the prox network for prox_mode 2 (an FP32 blob, capi.NET_BLOB floats)."""
        b = np.ascontiguousarray(blob, dtype=np.float32).ravel()
        self._h.check(self._h.lib.wrapd_set_prox_net(self._h.h, capi.fptr(b), b.size))

    def set_profiling(self, on: bool = True):
        self._h.check(self._h.lib.wrapd_set_profiling(self._h.h, int(on)))

    def profile(self) -> dict:
        ms, n = np.zeros(6), (ctypes.c_int64 * 6)()
        self._h.check(self._h.lib.wrapd_get_profile(self._h.h, capi.dptr(ms), n))
        names = ["local", "grad_gather", "vector", "solve", "unused", "host_gaps"]
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(names)}

    def algorithm_data(self, mesh: int | None = None) -> AlgorithmData:
        return AlgorithmData(**{k: self.log(k, mesh) for k in capi.LOGS}, runtime_ms=self.runtime())

    # -- TetElements-level components ------------------------------------------
    def get_state(self, name: str) -> np.ndarray:
        n = ctypes.c_int64(0)
        h = self._h
        h.check(h.lib.wrapd_get_state(h.h, name.encode(), None, 0, ctypes.byref(n)))
        out = np.empty(n.value)
        h.check(h.lib.wrapd_get_state(h.h, name.encode(), capi.dptr(out), n.value, ctypes.byref(n)))
        return out

    def set_state(self, name: str, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64).ravel()
        self._h.check(self._h.lib.wrapd_set_state(self._h.h, name.encode(), capi.dptr(a), a.size))

    def update_defo_cache(self):
        self._h.check(self._h.lib.wrapd_update_defo_cache(self._h.h))

    def polar_update(self, update_candidates: bool = True) -> float:
        d = ctypes.c_double(0.0)
        self._h.check(self._h.lib.wrapd_polar_update(self._h.h, int(update_candidates), ctypes.byref(d)))
        return d.value

    def global_grad(self, xfree=None):
        nf = int(self.info()["n_free"])
        g = np.empty((nf, 3))
        v = ctypes.c_double(0.0)
        x = None if xfree is None else np.ascontiguousarray(xfree, dtype=np.float64)
        self._h.check(self._h.lib.wrapd_global_grad(self._h.h, capi.dptr(x) if x is not None else None,
                                                    capi.dptr(g), ctypes.byref(v)))
        return v.value, g

    def potential_energy(self):
        pe, fl = ctypes.c_double(0.0), ctypes.c_int(0)
        self._h.check(self._h.lib.wrapd_potential_energy(self._h.h, ctypes.byref(pe), ctypes.byref(fl)))
        return pe.value, fl.value

    def solve_A(self, b):
        bb = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, 3)
        x = np.empty_like(bb)
        self._h.check(self._h.lib.wrapd_solve_A(self._h.h, capi.dptr(bb), capi.dptr(x)))
        return x

    def solve_A_holding(self, b, front):
        """wrapd_solve_A_holding: the solve with one front never reporting
        completion; raises WrapdError (WRAPD_E_TIMEOUT) when the waits ran out."""
        bb = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, 3)
        x = np.empty_like(bb)
        self._h.check(self._h.lib.wrapd_solve_A_holding(self._h.h, capi.dptr(bb), capi.dptr(x), int(front)))
        return x

    def close(self):
        self._h.close()


def solve_bar(bar, **settings):
    """Convenience: run the solver on a ``bars.Bar``; returns (solver, X)."""
    s = Solver(**settings)
    s.add_tetmesh(bar.rest, bar.init, bar.tets)
    s.set_pins(bar.pins)
    s.initialize()
    X = s.solve()
    return s, X
