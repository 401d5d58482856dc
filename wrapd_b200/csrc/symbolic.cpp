// Geometric nested dissection + multifrontal symbolic analysis (see symbolic.hpp).
#include "symbolic.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <memory>
#include <exception>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace wrapd {

namespace {

// Host threads for `n` items of work: one per `grain` items, at most the
// hardware's threads, 16, and WRAPD_HOST_THREADS when that is set to a
// positive number; at least one.  The results do not depend on the count.
int host_threads(int64_t n, int64_t grain) {
    int64_t cap = std::min<int64_t>(16, std::max(1u, std::thread::hardware_concurrency()));
    if (const char* env = std::getenv("WRAPD_HOST_THREADS")) {
        const long v = std::strtol(env, nullptr, 10);
        if (v > 0) cap = std::min<int64_t>(cap, v);
    }
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(n / grain, cap)));
}

// fn(t, lo, hi) over `nthreads` contiguous ranges of [0, n), range t on its own
// thread (range 0 on the caller's); exceptions are rethrown after the join.
template <typename F>
void parallel_ranges(int n, int nthreads, F&& fn) {
    std::vector<std::thread> th;
    std::vector<std::exception_ptr> err(nthreads);
    auto run = [&](int t) {
        const int lo = static_cast<int>((int64_t)n * t / nthreads), hi = static_cast<int>((int64_t)n * (t + 1) / nthreads);
        try {
            fn(t, lo, hi);
        } catch (...) {
            err[t] = std::current_exception();
        }
    };
    for (int t = 1; t < nthreads; ++t) th.emplace_back(run, t);
    run(0);
    for (auto& x : th) x.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// Per-vertex membership marks shared by dissections of disjoint vertex sets
// that run at the same time: a split writes tag * 4 + side (1 left, 2 right,
// 3 separator) for its own vertices only, with a tag no other split uses, and
// compares its neighbours' marks against its own tag, so marks left by other
// splits never match (relaxed atomics: only equality with one's own writes
// matters).
struct Marks {
    std::unique_ptr<std::atomic<int64_t>[]> side;
    std::atomic<int64_t> next{1};
    explicit Marks(int n) : side(new std::atomic<int64_t>[n]) {
        for (int i = 0; i < n; ++i) side[i].store(0, std::memory_order_relaxed);
    }
    void set(int v, int64_t m) { side[v].store(m, std::memory_order_relaxed); }
    int64_t get(int v) const { return side[v].load(std::memory_order_relaxed); }
};

struct Split {
    std::vector<int> left, right, sep;
};

// One bisection: median cut along the longest box axis of `verts` (whose
// size exceeds the leaf size), then the smaller one-sided vertex separator.
Split split(std::vector<int> verts, const std::vector<int>& ptr, const std::vector<int>& adj,
            const std::vector<double>& xyz, Marks& marks) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int v : verts)
        for (int d = 0; d < 3; ++d) {
            lo[d] = std::min(lo[d], xyz[3 * v + d]);
            hi[d] = std::max(hi[d], xyz[3 * v + d]);
        }
    int axis = 0;
    for (int d = 1; d < 3; ++d)
        if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
    const size_t mid = verts.size() / 2;
    std::nth_element(verts.begin(), verts.begin() + mid, verts.end(), [&](int a, int b) {
        double xa = xyz[3 * a + axis], xb = xyz[3 * b + axis];
        return xa < xb || (xa == xb && a < b);
    });
    // Put every vertex on the median coordinate into the right half, so a
    // grid plane is never split between the halves.
    const double cut = xyz[3 * verts[mid] + axis];
    std::vector<int> L, R;
    L.reserve(mid + 1);
    R.reserve(verts.size() - mid + 1);
    for (int v : verts) (xyz[3 * v + axis] < cut ? L : R).push_back(v);
    if (L.empty() || R.empty()) {  // degenerate (all on one plane): split by index
        std::sort(verts.begin(), verts.end());
        L.assign(verts.begin(), verts.begin() + mid);
        R.assign(verts.begin() + mid, verts.end());
    }
    const int64_t tag = 4 * marks.next.fetch_add(1, std::memory_order_relaxed);
    for (int v : L) marks.set(v, tag + 1);
    for (int v : R) marks.set(v, tag + 2);
    // One-sided separators: right vertices touching the left, or left
    // vertices touching the right; keep the smaller.
    std::vector<int> sepR, sepL;
    for (int v : R)
        for (int k = ptr[v]; k < ptr[v + 1]; ++k)
            if (marks.get(adj[k]) == tag + 1) { sepR.push_back(v); break; }
    for (int v : L)
        for (int k = ptr[v]; k < ptr[v + 1]; ++k)
            if (marks.get(adj[k]) == tag + 2) { sepL.push_back(v); break; }
    const bool use_right = sepR.size() <= sepL.size();
    Split out;
    out.sep = use_right ? std::move(sepR) : std::move(sepL);
    for (int v : out.sep) marks.set(v, tag + 3);
    for (int v : L) if (marks.get(v) == tag + 1) out.left.push_back(v);
    for (int v : R) if (marks.get(v) == tag + 2) out.right.push_back(v);
    return out;
}

// A dissected vertex set: its columns in post-order (new -> old), its fronts
// (ids and first columns local to this piece) and its root fronts.
struct Piece {
    std::vector<int> order;
    std::vector<Front> fronts;
    std::vector<int> roots;

    int make_front(std::vector<int> verts, const std::vector<int>& children) {
        Front f;
        f.first = static_cast<int>(order.size());
        f.ncols = static_cast<int>(verts.size());
        for (int v : verts) order.push_back(v);
        f.children = children;
        const int id = static_cast<int>(fronts.size());
        for (int c : children) fronts[c].parent = id;
        fronts.push_back(std::move(f));
        return id;
    }

    // Appends another piece after this one (its fronts renumbered, its columns
    // shifted) and returns the appended piece's roots in the new numbering.
    std::vector<int> append(Piece&& o) {
        const int fo = static_cast<int>(fronts.size()), co = static_cast<int>(order.size());
        order.insert(order.end(), o.order.begin(), o.order.end());
        for (Front& f : o.fronts) {
            f.first += co;
            if (f.parent >= 0) f.parent += fo;
            for (int& c : f.children) c += fo;
            fronts.push_back(std::move(f));
        }
        std::vector<int> r = std::move(o.roots);
        for (int& x : r) x += fo;
        return r;
    }
};

struct Dissector {
    const std::vector<int>& ptr;
    const std::vector<int>& adj;
    const std::vector<double>& xyz;
    int leaf;
    Marks& marks;

    // Serial recursion into `piece`; returns the root fronts built over `verts`.
    std::vector<int> run(Piece& piece, std::vector<int> verts) {
        if (verts.empty()) return {};
        if (static_cast<int>(verts.size()) <= leaf) {
            std::sort(verts.begin(), verts.end());
            return {piece.make_front(std::move(verts), {})};
        }
        Split sp = split(std::move(verts), ptr, adj, xyz, marks);
        std::vector<int> roots = run(piece, std::move(sp.left));
        std::vector<int> rr = run(piece, std::move(sp.right));
        roots.insert(roots.end(), rr.begin(), rr.end());
        if (sp.sep.empty()) return roots;
        std::sort(sp.sep.begin(), sp.sep.end());
        return {piece.make_front(std::move(sp.sep), roots)};
    }

    // The same dissection with the two halves of the top `par_levels` splits
    // on their own threads; the pieces are joined in the serial order (left,
    // right, separator), so the result is the serial one.
    Piece build(std::vector<int> verts, int par_levels) {
        Piece piece;
        if (par_levels <= 0 || static_cast<int>(verts.size()) <= std::max(leaf, 4096)) {
            piece.roots = run(piece, std::move(verts));
            return piece;
        }
        Split sp = split(std::move(verts), ptr, adj, xyz, marks);
        Piece left;
        std::exception_ptr err;
        std::thread th([&] {
            try {
                left = build(std::move(sp.left), par_levels - 1);
            } catch (...) {
                err = std::current_exception();
            }
        });
        Piece right;
        try {
            right = build(std::move(sp.right), par_levels - 1);
        } catch (...) {
            th.join();
            throw;
        }
        th.join();
        if (err) std::rethrow_exception(err);
        piece = std::move(left);
        std::vector<int> roots = std::move(piece.roots);
        std::vector<int> rr = piece.append(std::move(right));
        roots.insert(roots.end(), rr.begin(), rr.end());
        if (sp.sep.empty()) {
            piece.roots = std::move(roots);
            return piece;
        }
        std::sort(sp.sep.begin(), sp.sep.end());
        piece.roots = {piece.make_front(std::move(sp.sep), roots)};
        return piece;
    }
};

}  // namespace

void free_vertex_graph(int nf, int ne, const int* tets, const int* free_of_vert, std::vector<int>& vinc_ptr,
                       std::vector<int>& vinc, std::vector<int>& ptr, std::vector<int>& adj) {
    vinc_ptr.assign(nf + 1, 0);
    for (int64_t t = 0; t < 4 * (int64_t)ne; ++t) {
        const int i = free_of_vert[tets[t]];
        if (i >= 0) vinc_ptr[i + 1]++;
    }
    for (int i = 0; i < nf; ++i) vinc_ptr[i + 1] += vinc_ptr[i];
    vinc.resize(vinc_ptr[nf]);
    {
        std::vector<int> fill(vinc_ptr.begin(), vinc_ptr.end() - 1);
        for (int e = 0; e < ne; ++e)
            for (int a = 0; a < 4; ++a) {
                const int i = free_of_vert[tets[4 * (int64_t)e + a]];
                if (i >= 0) vinc[fill[i]++] = e * 4 + a;
            }
    }
    // Neighbour lists by vertex range, one range per host thread: a marker per
    // vertex (the id of the vertex whose list last took it) keeps each list
    // unique before the short sort; the ranges are concatenated in order.
    const int nthreads = host_threads(nf, 16384);
    std::vector<std::vector<int>> part_adj(nthreads), part_cnt(nthreads);
    parallel_ranges(nf, nthreads, [&](int t, int lo, int hi) {
        std::vector<int> mark(nf, -1);
        std::vector<int>& out = part_adj[t];
        std::vector<int>& cnt = part_cnt[t];
        out.reserve(16 * (size_t)(hi - lo));
        cnt.reserve(hi - lo);
        for (int i = lo; i < hi; ++i) {
            const size_t start = out.size();
            mark[i] = i;
            for (int q = vinc_ptr[i]; q < vinc_ptr[i + 1]; ++q) {
                const int e = vinc[q] >> 2;
                for (int b = 0; b < 4; ++b) {
                    const int j = free_of_vert[tets[4 * (int64_t)e + b]];
                    if (j >= 0 && mark[j] != i) { mark[j] = i; out.push_back(j); }
                }
            }
            std::sort(out.begin() + start, out.end());
            cnt.push_back(static_cast<int>(out.size() - start));
        }
    });
    ptr.assign(nf + 1, 0);
    {
        int i = 0;
        for (int t = 0; t < nthreads; ++t)
            for (int c : part_cnt[t]) { ptr[i + 1] = ptr[i] + c; ++i; }
    }
    adj.resize(ptr[nf]);
    {
        size_t at = 0;
        for (int t = 0; t < nthreads; ++t) {
            std::copy(part_adj[t].begin(), part_adj[t].end(), adj.begin() + at);
            at += part_adj[t].size();
        }
    }
}

Symbolic analyse(int n, const std::vector<int>& adj_ptr, const std::vector<int>& adj,
                 const std::vector<double>& coords, int leaf) {
    if (n <= 0) throw std::invalid_argument("analyse: empty matrix");
    Marks marks(n);
    Dissector d{adj_ptr, adj, coords, std::max(1, leaf), marks};
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    int par_levels = 0;
    for (int t = host_threads(n, 16384); t > 1; t >>= 1) ++par_levels;
    Piece piece = d.build(std::move(all), par_levels);
    Symbolic S;
    S.n = n;
    S.perm = std::move(piece.order);
    S.fronts = std::move(piece.fronts);
    if (static_cast<int>(S.perm.size()) != n) throw std::logic_error("analyse: ordering incomplete");
    S.iperm.assign(n, -1);
    for (int i = 0; i < n; ++i) S.iperm[S.perm[i]] = i;

    // Levels.
    int maxlev = 0;
    for (Front& f : S.fronts) {
        int lv = 0;
        for (int c : f.children) lv = std::max(lv, S.fronts[c].level + 1);
        f.level = lv;
        maxlev = std::max(maxlev, lv);
        S.max_children = std::max(S.max_children, static_cast<int>(f.children.size()));
    }
    S.levels.assign(maxlev + 1, {});
    for (size_t fi = 0; fi < S.fronts.size(); ++fi) S.levels[S.fronts[fi].level].push_back(static_cast<int>(fi));
    // Row structures, level by level (a front's children are on lower levels):
    // the front's columns' neighbours beyond it, and its children's rows
    // beyond it.  The fronts of a level are split over host threads, each with
    // its own marks (tag = front id).
    const int rthreads = host_threads(n, 16384);
    std::vector<std::vector<int>> marks_of(rthreads);
    for (const std::vector<int>& lv : S.levels) {
        const int nt = std::max(1, std::min<int>(rthreads, static_cast<int>(lv.size())));
        parallel_ranges(static_cast<int>(lv.size()), nt, [&](int t, int lo, int hi) {
            std::vector<int>& mark = marks_of[t];
            if (mark.empty()) mark.assign(n, -1);
            for (int q = lo; q < hi; ++q) {
                const int fi = lv[q];
                Front& f = S.fronts[fi];
                const int last = f.first + f.ncols;
                std::vector<int> rows;
                for (int j = f.first; j < last; ++j) {
                    const int v = S.perm[j];
                    for (int k = adj_ptr[v]; k < adj_ptr[v + 1]; ++k) {
                        const int i = S.iperm[adj[k]];
                        if (i >= last && mark[i] != fi) { mark[i] = fi; rows.push_back(i); }
                    }
                }
                for (int c : f.children)
                    for (int i : S.fronts[c].rows)
                        if (i >= last && mark[i] != fi) { mark[i] = fi; rows.push_back(i); }
                std::sort(rows.begin(), rows.end());
                f.rows = std::move(rows);
            }
        });
    }
    // Pools, relative maps, statistics.
    int64_t fo = 0, yo = 0, uo = 0, ro = 0;
    for (Front& f : S.fronts) {
        const int64_t k = f.ncols, r = f.nrows(), ld = k + r, ldp = f.ld();
        f.f_off = fo; fo += ldp * ldp;
        f.y_off = yo; yo += yw_ld(k, r) * k;
        f.u_off = uo; uo += r * 3;
        f.rel_off = ro; ro += r;
        S.nnz_L += k * (k + 1) / 2 + k * r;
        // partial Cholesky of k columns of a (k + r) front
        for (int64_t j = 0; j < k; ++j) {
            const double m = static_cast<double>(ld - j - 1);
            S.flops += m + m * (m + 1.0);  // column scale + rank-1 update of the trailing lower triangle
        }
    }
    S.f_pool = fo; S.y_pool = yo; S.u_pool = uo;
    S.relmap.assign(ro, -1);
    for (Front& f : S.fronts) {
        if (f.parent < 0) continue;
        const Front& p = S.fronts[f.parent];
        const int plast = p.first + p.ncols;
        size_t q = 0;
        for (int t = 0; t < f.nrows(); ++t) {
            const int i = f.rows[t];
            int pos;
            if (i < plast) {
                if (i < p.first) throw std::logic_error("analyse: child row below parent columns");
                pos = i - p.first;
            } else {
                while (q < p.rows.size() && p.rows[q] < i) ++q;
                if (q == p.rows.size() || p.rows[q] != i) throw std::logic_error("analyse: child row not in parent");
                pos = p.ncols + static_cast<int>(q);
            }
            S.relmap[f.rel_off + t] = pos;
        }
    }
    for (const Front& f : S.fronts)
        if (f.parent < 0 && f.nrows() != 0) throw std::logic_error("analyse: root with off-diagonal rows");
    return S;
}

void assembly_map(const Symbolic& S, const std::vector<int>& vinc_ptr, const std::vector<int>& vinc,
                  const std::vector<int>& ptr, const std::vector<int>& adj, std::vector<int64_t>& A_pos,
                  std::vector<int>& A_ptr, std::vector<int>& A_con) {
    const int nf = S.n;
    std::vector<int> col2front(nf, -1);
    for (size_t f = 0; f < S.fronts.size(); ++f)
        for (int j = 0; j < S.fronts[f].ncols; ++j) col2front[S.fronts[f].first + j] = static_cast<int>(f);
    std::vector<int64_t> ebase(nf + 1, 0);
    for (int i = 0; i < nf; ++i) {
        const int* lo = adj.data() + ptr[i];
        const int* hi = adj.data() + ptr[i + 1];
        ebase[i + 1] = ebase[i] + 1 + (hi - std::upper_bound(lo, hi, i));
    }
    const int64_t nentries = ebase[nf];
    auto entry_of = [&](int fa, int fb) -> int64_t {   // fa <= fb
        if (fa == fb) return ebase[fa];
        const int* lo = adj.data() + ptr[fa];
        const int* hi = adj.data() + ptr[fa + 1];
        const int* up = std::upper_bound(lo, hi, fa);
        return ebase[fa] + 1 + (std::lower_bound(up, hi, fb) - up);
    };
    // Contributions of entry {i, j}: the elements holding both vertices, in
    // element order (a merge of the two incidence lists).
    auto entry_contribs = [&](int i, int j, auto&& out) {
        if (i == j) {
            for (int q = vinc_ptr[i]; q < vinc_ptr[i + 1]; ++q) out((vinc[q] >> 2) * 16 + (vinc[q] & 3) * 5);
            return;
        }
        int p = vinc_ptr[i], q = vinc_ptr[j];
        while (p < vinc_ptr[i + 1] && q < vinc_ptr[j + 1]) {
            const int ep = vinc[p] >> 2, eq = vinc[q] >> 2;
            if (ep < eq) ++p;
            else if (eq < ep) ++q;
            else { out(ep * 16 + (vinc[p] & 3) * 4 + (vinc[q] & 3)); ++p; ++q; }
        }
    };
    // Vertex i owns entries ebase[i] .. ebase[i+1]-1, so ranges of vertices
    // write disjoint parts of every output: count, prefix, fill.
    const int nthreads = host_threads(nf, 16384);
    A_ptr.assign(nentries + 1, 0);
    parallel_ranges(nf, nthreads, [&](int, int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            int64_t id = ebase[i];
            int n = 0;
            entry_contribs(i, i, [&](int) { ++n; });
            A_ptr[id + 1] = n;
            for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
                if (adj[q] <= i) continue;
                n = 0;
                entry_contribs(i, adj[q], [&](int) { ++n; });
                A_ptr[++id + 1] = n;
            }
        }
    });
    for (int64_t t = 0; t < nentries; ++t) A_ptr[t + 1] += A_ptr[t];
    A_con.resize(A_ptr[nentries]);
    A_pos.resize(nentries);
    parallel_ranges(nf, nthreads, [&](int, int lo, int hi) {
        for (int i = lo; i < hi; ++i) {
            int64_t id = ebase[i];
            int w = A_ptr[id];
            entry_contribs(i, i, [&](int c) { A_con[w++] = c; });
            for (int q = ptr[i]; q < ptr[i + 1]; ++q) {
                if (adj[q] <= i) continue;
                w = A_ptr[++id];
                entry_contribs(i, adj[q], [&](int c) { A_con[w++] = c; });
            }
            // pool position of each entry: lower triangle in the dissection order
            auto put = [&](int j) {
                const int si = S.iperm[i], sj = S.iperm[j];
                const int r = std::max(si, sj), c = std::min(si, sj);
                const Front& F = S.fronts[col2front[c]];
                int lr;
                if (r < F.first + F.ncols) lr = r - F.first;
                else lr = F.ncols + static_cast<int>(std::lower_bound(F.rows.begin(), F.rows.end(), r) - F.rows.begin());
                A_pos[entry_of(i, j)] = F.f_off + lr + static_cast<int64_t>(c - F.first) * F.ld();
            };
            put(i);
            for (int q = ptr[i]; q < ptr[i + 1]; ++q)
                if (adj[q] > i) put(adj[q]);
        }
    });
}

void host_parallel(int n, int64_t grain, const std::function<void(int, int)>& fn) {
    parallel_ranges(n, host_threads(n, grain), [&](int, int lo, int hi) { fn(lo, hi); });
}

Symbolic merge(const std::vector<Symbolic>& parts) {
    if (parts.size() == 1) return parts[0];
    Symbolic S;
    int off = 0, foff = 0;
    int64_t fo = 0, yo = 0, uo = 0, ro = 0;
    for (const Symbolic& P : parts) {
        for (int v : P.perm) S.perm.push_back(v + off);
        if (S.levels.size() < P.levels.size()) S.levels.resize(P.levels.size());
        for (size_t l = 0; l < P.levels.size(); ++l)
            for (int f : P.levels[l]) S.levels[l].push_back(f + foff);
        for (const Front& F : P.fronts) {
            Front G = F;
            G.first += off;
            for (int& r : G.rows) r += off;
            if (G.parent >= 0) G.parent += foff;
            for (int& c : G.children) c += foff;
            G.f_off += fo; G.y_off += yo; G.u_off += uo; G.rel_off += ro;
            S.fronts.push_back(std::move(G));
        }
        S.relmap.insert(S.relmap.end(), P.relmap.begin(), P.relmap.end());
        off += P.n;
        foff += static_cast<int>(P.fronts.size());
        fo += P.f_pool; yo += P.y_pool; uo += P.u_pool; ro += static_cast<int64_t>(P.relmap.size());
        S.nnz_L += P.nnz_L;
        S.flops += P.flops;
        S.max_children = std::max(S.max_children, P.max_children);
    }
    S.n = off;
    S.f_pool = fo; S.y_pool = yo; S.u_pool = uo;
    S.iperm.assign(S.n, -1);
    for (int i = 0; i < S.n; ++i) S.iperm[S.perm[i]] = i;
    return S;
}

}  // namespace wrapd
