"""Seeded synthetic tetrahedral bars (the workloads the solver is measured on).

A bar is an ``n_a x n_b x n_L`` grid of cubes of edge ``h = 1/n_a`` whose long
axis is x (``n_L`` cells).  Every cube is split into 6 positive-volume tets
along its main diagonal (Kuhn/Freudenthal split).  Vertex id is
``i + (n_L+1)*(j + (n_a+1)*k)`` with ``i`` along x, ``j`` along y (``n_a``
cells) and ``k`` along z (``n_b`` cells).  Handles are every vertex on the
x = 0 and x = L faces.

The deformed initial pose twists each vertex's (y, z) about the bar's centre
line by ``theta(x) = Theta * x / L``, optionally bends the twisted bar onto an
arc of total angle ``Phi`` (radius ``R = L / Phi``), and adds N(0, (sigma_n*h)^2)
noise to free vertices only.  Noise comes from a SplitMix64 stream turned into
normals by Box-Muller, so a seed reproduces a mesh bit for bit on any host.

Rest/init meshes are written in the TetGen ``.node/.ele`` text format that
``samples/utils/MeshIO.hpp:182-315`` (``load_elenode``) reads, 0-based, with
17 significant digits so a reader recovers every double exactly; handles as
whitespace-separated 0-based vertex ids (``samples/tests/quasi.cpp:146-159``).
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """The first ``count`` outputs of SplitMix64 started at ``seed``."""
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed: int, count: int) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of each SplitMix64 output."""
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def normals(seed: int, count: int) -> np.ndarray:
    """Standard normals by Box-Muller (cosine branch), two uniforms per normal."""
    u = uniform01(seed, 2 * count)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


@dataclasses.dataclass
class Bar:
    rest: np.ndarray      # (n_verts, 3) float64
    init: np.ndarray      # (n_verts, 3) float64
    tets: np.ndarray      # (n_tets, 4) int32, positive rest volume
    pins: np.ndarray      # (n_pins,) int32, sorted
    h: float
    length: float
    dims: tuple

    @property
    def n_verts(self) -> int:
        return int(self.rest.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])


# Kuhn split: for each permutation of the axes, the tet walks corner 000 ->
# +e_a -> +e_a+e_b -> 111.  Odd permutations swap the middle two corners so
# every tet has positive volume.
_PERMS = [((0, 1, 2), False), ((1, 2, 0), False), ((2, 0, 1), False),
          ((0, 2, 1), True), ((2, 1, 0), True), ((1, 0, 2), True)]


def make_bar(n_a: int, n_b: int, n_L: int, *, twist_deg: float = 180.0,
             bend_deg: float = 0.0, noise: float = 0.02, seed: int = 0,
             h: float | None = None) -> Bar:
    """Build a twisted (optionally bent) noisy bar.  See the module docstring."""
    if min(n_a, n_b, n_L) < 1:
        raise ValueError("bar dimensions must be >= 1")
    h = 1.0 / n_a if h is None else float(h)
    nx, ny, nz = n_L + 1, n_a + 1, n_b + 1
    i = np.arange(nx)
    j = np.arange(ny)
    k = np.arange(nz)
    K, J, I = np.meshgrid(k, j, i, indexing="ij")  # id = i + nx*(j + ny*k)
    rest = np.stack([I.ravel() * h, J.ravel() * h, K.ravel() * h], axis=1).astype(np.float64)
    vid = lambda a, b, c: a + nx * (b + ny * c)

    ci, cj, ck = np.meshgrid(np.arange(n_L), np.arange(n_a), np.arange(n_b), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    # order cubes by (k, j, i) so tets follow vertex order
    order = np.lexsort((ci, cj, ck))
    ci, cj, ck = ci[order], cj[order], ck[order]
    corner = lambda d: vid(ci + d[0], cj + d[1], ck + d[2])
    tets = []
    for perm, odd in _PERMS:
        p0 = np.zeros(3, dtype=int)
        p1 = p0.copy(); p1[perm[0]] = 1
        p2 = p1.copy(); p2[perm[1]] = 1
        p3 = np.ones(3, dtype=int)
        a, b, c, d = corner(p0), corner(p1), corner(p2), corner(p3)
        if odd:
            b, c = c, b
        tets.append(np.stack([a, b, c, d], axis=1))
    tets = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int32)

    length = n_L * h
    pin_mask = (I.ravel() == 0) | (I.ravel() == n_L)
    pins = np.nonzero(pin_mask)[0].astype(np.int32)

    yc, zc = 0.5 * n_a * h, 0.5 * n_b * h
    theta = math.radians(twist_deg) * rest[:, 0] / length
    dy, dz = rest[:, 1] - yc, rest[:, 2] - zc
    init = rest.copy()
    init[:, 1] = yc + np.cos(theta) * dy - np.sin(theta) * dz
    init[:, 2] = zc + np.sin(theta) * dy + np.cos(theta) * dz
    if bend_deg != 0.0:
        phi = math.radians(bend_deg)
        R = length / phi
        x, z = init[:, 0].copy(), init[:, 2].copy()
        init[:, 0] = (R - z) * np.sin(x / R)
        init[:, 2] = R - (R - z) * np.cos(x / R)
    free = np.nonzero(~pin_mask)[0]
    if noise > 0.0 and free.size:
        g = normals(seed, 3 * free.size).reshape(free.size, 3)
        init[free] += (noise * h) * g
    return Bar(rest=rest, init=init, tets=tets, pins=pins, h=h, length=length,
               dims=(n_a, n_b, n_L))


# The bar workloads, by the sizes they are quoted at.
def bar_8x8x32(seed: int = 0) -> Bar:
    """8x8x32 cubes (12,288 tets, 2,673 verts), 180 deg twist, noise 0.02 h."""
    return make_bar(8, 8, 32, twist_deg=180.0, noise=0.02, seed=seed)


def bar_32x32x128_bent(seed: int = 0) -> Bar:
    """32x32x128 cubes (786,432 tets, 140,481 verts), 360 deg twist + 90 deg bend, noise 0.01 h."""
    return make_bar(32, 32, 128, twist_deg=360.0, bend_deg=90.0, noise=0.01, seed=seed)


def bar_64x64x160(seed: int = 0) -> Bar:
    """64x64x160 cubes (3,932,160 tets, 680,225 verts), 720 deg twist, noise 0.005 h."""
    return make_bar(64, 64, 160, twist_deg=720.0, noise=0.005, seed=seed)


def batch_bars(count: int = 64, seed0: int = 0):
    """Uneven bars: n_a, n_b in U{4..16}, n_L in U{8..64}, twist U[0, 360] deg,
    E log-uniform [1e4, 1e6], nu U[0.35, 0.48].  Returns (bar, youngs, poisson) triples."""
    out = []
    for s in range(seed0, seed0 + count):
        u = uniform01(s ^ 0x5DEECE66D, 6)
        n_a = 4 + int(u[0] * 13)
        n_b = 4 + int(u[1] * 13)
        n_L = 8 + int(u[2] * 57)
        twist = 360.0 * u[3]
        E = 10.0 ** (4.0 + 2.0 * u[4])
        nu = 0.35 + 0.13 * u[5]
        out.append((make_bar(n_a, n_b, n_L, twist_deg=twist, noise=0.02, seed=s), E, nu))
    return out


def concat(bars_list) -> Bar:
    """The batch as one mesh: vertices, tets and pins of each bar in turn, ids
    shifted by the vertices before it (the order a batch's positions come in)."""
    rest, init, tets, pins, off = [], [], [], [], 0
    for b in bars_list:
        rest.append(b.rest)
        init.append(b.init)
        tets.append(b.tets + off)
        pins.append(np.asarray(b.pins) + off)
        off += b.rest.shape[0]
    first = bars_list[0]
    return dataclasses.replace(first, rest=np.concatenate(rest), init=np.concatenate(init),
                               tets=np.concatenate(tets).astype(np.int32), pins=np.concatenate(pins).astype(np.int32))


def write_elenode(path_stem: str, verts: np.ndarray, tets: np.ndarray) -> None:
    """Write ``<stem>.node`` and ``<stem>.ele`` (0-based, exact doubles)."""
    n = verts.shape[0]
    node = np.concatenate([np.arange(n, dtype=np.float64)[:, None], verts], axis=1)
    np.savetxt(path_stem + ".node", node, fmt=["%d", "%.17g", "%.17g", "%.17g"],
               header=f"{n} 3 0 0", comments="")
    m = tets.shape[0]
    ele = np.concatenate([np.arange(m, dtype=np.int64)[:, None], tets.astype(np.int64)], axis=1)
    np.savetxt(path_stem + ".ele", ele, fmt="%d", header=f"{m} 4 0", comments="")


def write_handles(path: str, pins: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("\n".join(str(int(p)) for p in pins) + "\n")


def write_bar(bar: Bar, directory: str, name: str = "bar") -> dict:
    """Write rest/init/handles files for the ``quasi`` front ends; returns their paths."""
    os.makedirs(directory, exist_ok=True)
    rest = os.path.join(directory, name + "_rest")
    init = os.path.join(directory, name + "_init")
    handles = os.path.join(directory, name + "_handles.txt")
    write_elenode(rest, bar.rest, bar.tets)
    write_elenode(init, bar.init, bar.tets)
    write_handles(handles, bar.pins)
    return {"rest": rest + ".node", "init": init + ".node", "handles": handles}


def read_node(path: str) -> np.ndarray:
    """Read a ``.node`` file (0- or 1-based, like ``MeshIO.hpp:267-300``)."""
    with open(path) as f:
        n = int(f.readline().split()[0])
        out = np.empty((n, 3), dtype=np.float64)
        base = None
        for _ in range(n):
            parts = f.readline().split()
            idx = int(parts[0])
            if base is None:
                base = 1 if idx == 1 else 0
            out[idx - base] = [float(parts[1]), float(parts[2]), float(parts[3])]
    return out
