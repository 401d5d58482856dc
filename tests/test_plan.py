"""The host-side symbolic analysis on the CPU (wrapd_plan_*, no GPU needed):
the nested-dissection order, the assembly tree of dense fronts, their row
structures and relative-index maps, and a multifrontal Cholesky run in numpy
on exactly those structures.  The GPU factorization consumes the same
structures (the extend-add follows `relmap`, each level is one launch)."""
import dataclasses

import numpy as np
import pytest

from wrapd_b200 import bars, capi


@pytest.fixture(scope="module")
def lib(lib_built):
    return capi.load()


def free_graph(bar):
    """Free numbering (ascending vertex id, pins skipped) and adjacency sets."""
    nv = bar.n_verts
    pinned = np.zeros(nv, bool)
    pinned[bar.pins] = True
    fov = -np.ones(nv, dtype=np.int64)
    fov[~pinned] = np.arange(int((~pinned).sum()))
    nf = int((~pinned).sum())
    adj = [set() for _ in range(nf)]
    for t in bar.tets:
        f = [int(fov[v]) for v in t if fov[v] >= 0]
        for a in f:
            adj[a].update(b for b in f if b != a)
    return nf, adj


def small_bars():
    yield "8x8x32", bars.bar_8x8x32()
    yield "3x4x9", bars.make_bar(3, 4, 9, twist_deg=45.0, noise=0.02, seed=3)
    b = bars.make_bar(4, 4, 12, twist_deg=0.0, noise=0.0, seed=1)
    rng = np.random.default_rng(5)
    extra = rng.choice(np.setdiff1d(np.arange(b.n_verts), b.pins), 17, replace=False)
    yield "4x4x12 scattered pins", dataclasses.replace(b, pins=np.sort(np.concatenate([b.pins, extra])).astype(b.pins.dtype))


@pytest.mark.parametrize("name,bar", list(small_bars()), ids=[n for n, _ in small_bars()])
def test_fronts_are_a_valid_assembly_tree(lib, name, bar):
    p = capi.plan(bar.rest, bar.tets, bar.pins, leaf_size=16)
    nf, adj = free_graph(bar)
    assert p["n_free"] == nf
    perm = p["perm"]
    assert np.array_equal(np.sort(perm), np.arange(nf))
    iperm = np.empty(nf, dtype=np.int64)
    iperm[perm] = np.arange(nf)
    first, ncols, parent, level = p["first"], p["ncols"], p["parent"], p["level"]
    rp, rows, rel = p["row_ptr"], p["rows"], p["relmap"]
    nfr = p["fronts"]
    # post-order, contiguous columns
    assert np.array_equal(first, np.concatenate([[0], np.cumsum(ncols)[:-1]]))
    assert first[-1] + ncols[-1] == nf and (ncols > 0).all()
    children = [[] for _ in range(nfr)]
    for f in range(nfr):
        if parent[f] >= 0:
            assert parent[f] > f
            children[parent[f]].append(f)
    # levels: one more than the highest child; p["levels"] of them
    for f in range(nfr):
        want = 1 + max(level[c] for c in children[f]) if children[f] else 0
        assert level[f] == want
    assert p["levels"] == level.max() + 1
    # row structure: exactly the neighbours beyond the front of its subtree's vertices
    sub0 = first.copy()
    for f in range(nfr):
        for c in children[f]:
            sub0[f] = min(sub0[f], sub0[c])
    for f in range(nfr):
        last = first[f] + ncols[f]
        want = set()
        for j in range(sub0[f], last):
            want.update(int(iperm[v]) for v in adj[perm[j]] if iperm[v] >= last)
        got = rows[rp[f]:rp[f + 1]]
        assert np.array_equal(got, np.array(sorted(want), dtype=got.dtype)), f"front {f}"
        if parent[f] < 0:
            assert got.size == 0
    # relative maps into the parent's front
    for f in range(nfr):
        q = parent[f]
        if q < 0:
            continue
        kq, qrows = ncols[q], rows[rp[q]:rp[q + 1]]
        for i, pos in zip(rows[rp[f]:rp[f + 1]], rel[rp[f]:rp[f + 1]]):
            if pos < kq:
                assert first[q] + pos == i
            else:
                assert qrows[pos - kq] == i
    # sizes
    k = ncols.astype(np.int64)
    r = np.diff(rp)
    ld = (k + r + 1) & ~1
    assert p["nnz_L"] == int((k * (k + 1) // 2 + k * r).sum())
    assert p["f_pool_bytes"] == 8 * int((ld * ld).sum())
    assert p["y_pool_bytes"] == 8 * int((ld * k).sum())
    assert p["total_rows"] == rows.size


def fill_structure(nf, adj, perm, iperm):
    """Row structure of each column of L for the permuted matrix (symbolic
    elimination: column j's structure is its lower neighbours plus its
    elimination-tree children's structures)."""
    struct = [None] * nf
    kids = [[] for _ in range(nf)]
    for j in range(nf):
        s = {int(iperm[v]) for v in adj[perm[j]] if iperm[v] > j}
        for c in kids[j]:
            s.update(i for i in struct[c] if i > j)
        struct[j] = s
        if s:
            kids[min(s)].append(j)
    return struct


@pytest.mark.parametrize("name,bar", list(small_bars()), ids=[n for n, _ in small_bars()])
def test_fronts_cover_the_fill(lib, name, bar):
    p = capi.plan(bar.rest, bar.tets, bar.pins, leaf_size=16)
    nf, adj = free_graph(bar)
    perm = p["perm"]
    iperm = np.empty(nf, dtype=np.int64)
    iperm[perm] = np.arange(nf)
    struct = fill_structure(nf, adj, perm, iperm)
    true_nnz = nf + sum(len(s) for s in struct)
    assert true_nnz <= p["nnz_L"]
    for f in range(p["fronts"]):
        a, k = p["first"][f], p["ncols"][f]
        allowed = set(range(a, a + k)) | set(p["rows"][p["row_ptr"][f]:p["row_ptr"][f + 1]].tolist())
        for j in range(a, a + k):
            assert struct[j] <= allowed, f"column {j} of front {f}"


def multifrontal_cholesky(A, p):
    """Dense-front multifrontal Cholesky of the permuted A on the plan's
    structures; returns L (n x n, new order)."""
    n = A.shape[0]
    L = np.zeros((n, n))
    first, ncols, parent = p["first"], p["ncols"], p["parent"]
    rp, rows, rel = p["row_ptr"], p["rows"], p["relmap"]
    upd = {}
    for f in range(p["fronts"]):
        a, k = int(first[f]), int(ncols[f])
        fr = rows[rp[f]:rp[f + 1]].astype(np.int64)
        idx = np.concatenate([np.arange(a, a + k), fr])
        F = np.tril(A[np.ix_(idx, idx)])
        F[:, k:] = 0.0                                  # only the front's own columns are assembled
        for c in [c for c in range(f) if parent[c] == f]:
            pos = rel[rp[c]:rp[c + 1]].astype(np.int64)
            F[np.ix_(pos, pos)] += upd.pop(c)
        F = np.tril(F) + np.tril(F, -1).T
        L11 = np.linalg.cholesky(F[:k, :k])
        L21 = np.linalg.solve(L11, F[:k, k:]).T
        L[a:a + k, a:a + k] = L11
        L[fr, a:a + k] = L21
        if parent[f] >= 0:
            upd[f] = F[k:, k:] - L21 @ L21.T
    return L


def test_multifrontal_factor_on_the_plan_reproduces_A(lib):
    bar = bars.bar_8x8x32()
    p = capi.plan(bar.rest, bar.tets, bar.pins)
    nf, adj = free_graph(bar)
    perm = p["perm"]
    # an SPD matrix with the mesh's sparsity: graph Laplacian + identity,
    # with random positive edge weights
    rng = np.random.default_rng(0)
    A = np.zeros((nf, nf))
    for i in range(nf):
        for j in adj[i]:
            if j > i:
                w = rng.uniform(0.5, 2.0)
                A[i, j] = A[j, i] = -w
    A[np.diag_indices(nf)] = -A.sum(axis=1) + 1.0
    Ap = A[np.ix_(perm, perm)]
    L = multifrontal_cholesky(Ap, p)
    assert np.allclose(L @ L.T, Ap, rtol=0, atol=1e-10 * np.abs(Ap).max())
    b = rng.standard_normal(nf)
    x = np.linalg.solve(L.T, np.linalg.solve(L, b[perm]))
    xs = np.empty(nf)
    xs[perm] = x
    assert np.abs(A @ xs - b).max() < 1e-9 * np.abs(b).max()


def test_plan_sizes_of_the_786k_bar(lib):
    """The 786,432-tet bar's factor: the flops, factor entries and level count
    that the GPU solver reports for it (wrapd_get_info: 73,234,058,435 flops,
    61.3 M entries, 12 levels, i.e. 12 solve launches per direction), and its
    front count as a regression value."""
    bar = bars.bar_32x32x128_bent()
    p = capi.plan(bar.rest, bar.tets, bar.pins)
    assert (p["n_free"], p["fronts"], p["levels"]) == (138303, 2943, 12)
    assert p["flops"] == 73234058435
    assert p["nnz_L"] == 61277250


def test_plan_sizes_of_the_3m9_bar(lib):
    """The 3,932,160-tet bar: the host plan gives what the GPU solver reported
    for it (wrapd_get_info: 16,383 fronts, 14 levels, 567,452,252 factor
    entries, 2,247,282,490,463 flops) and the two pools that make up 33.7 of
    the 36.6 GB it holds on the device."""
    bar = bars.bar_64x64x160()
    p = capi.plan(bar.rest, bar.tets, bar.pins)
    assert (p["n_free"], p["fronts"], p["levels"]) == (671775, 16383, 14)
    assert (p["nnz_L"], p["flops"]) == (567452252, 2247282490463)
    assert round((p["f_pool_bytes"] + p["y_pool_bytes"]) / 1e9, 1) == 33.7


def test_plan_rejects_bad_meshes(lib):
    bar = bars.make_bar(2, 2, 4, twist_deg=0.0, noise=0.0, seed=0)
    bad_tets = bar.tets.copy()
    bad_tets[0, 0] = bar.n_verts
    with pytest.raises(capi.WrapdError, match="out of range"):
        capi.plan(bar.rest, bad_tets, bar.pins)
    with pytest.raises(capi.WrapdError, match="distinct"):
        capi.plan(bar.rest, bar.tets, np.array([0, 0], dtype=np.int32))
    with pytest.raises(capi.WrapdError):
        capi.plan(bar.rest, bar.tets, np.arange(bar.n_verts, dtype=np.int32))


def test_quasi_plan_flag_needs_no_gpu(lib, tmp_path):
    """`quasi -plan 1` prints the same analysis from .node/.ele/handles files
    and exits before any CUDA call."""
    import os
    import subprocess
    bar = bars.bar_8x8x32()
    files = bars.write_bar(bar, str(tmp_path), "bar")
    quasi = os.path.join(os.path.dirname(capi.LIB_PATH), "quasi")
    r = subprocess.run([quasi, "-rest", files["rest"], "-init", files["init"], "-handles", files["handles"],
                        "-plan", "1"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    got = {k: int(v) for k, v in (line.rsplit(" ", 1) for line in r.stdout.strip().splitlines())}
    p = capi.plan(bar.rest, bar.tets, bar.pins)
    assert got == {"free vertices": p["n_free"], "fronts": p["fronts"], "levels": p["levels"],
                   "factor entries": p["nnz_L"], "factor flops": p["flops"], "F pool bytes": p["f_pool_bytes"],
                   "Y pool bytes": p["y_pool_bytes"]}
