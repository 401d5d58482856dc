// Geometric nested dissection + multifrontal symbolic analysis (see symbolic.hpp).
#include "symbolic.hpp"

#include <algorithm>
#include <cstring>
#include <numeric>
#include <stdexcept>

namespace wrapd {

namespace {

struct Dissector {
    int n;
    const std::vector<int>& ptr;
    const std::vector<int>& adj;
    const std::vector<double>& xyz;
    int leaf;
    std::vector<int> order;          // new -> old, filled in post-order
    std::vector<Front> fronts;
    std::vector<int> side;           // scratch: 0 = not in set, 1 = left, 2 = right, 3 = separator
    Dissector(int n_, const std::vector<int>& p, const std::vector<int>& a, const std::vector<double>& c, int l)
        : n(n_), ptr(p), adj(a), xyz(c), leaf(l), side(n_, 0) {}

    int make_front(const std::vector<int>& verts, const std::vector<int>& children) {
        Front f;
        f.first = static_cast<int>(order.size());
        f.ncols = static_cast<int>(verts.size());
        for (int v : verts) order.push_back(v);
        f.children = children;
        int id = static_cast<int>(fronts.size());
        for (int c : children) fronts[c].parent = id;
        fronts.push_back(std::move(f));
        return id;
    }

    // Returns the root fronts of the subtree built over `verts`.
    std::vector<int> run(std::vector<int> verts) {
        if (verts.empty()) return {};
        if (static_cast<int>(verts.size()) <= leaf) {
            std::sort(verts.begin(), verts.end());
            return {make_front(verts, {})};
        }
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
        for (int v : L) side[v] = 1;
        for (int v : R) side[v] = 2;
        // One-sided separators: right vertices touching the left, or left
        // vertices touching the right; keep the smaller.
        std::vector<int> sepR, sepL;
        for (int v : R)
            for (int k = ptr[v]; k < ptr[v + 1]; ++k)
                if (side[adj[k]] == 1) { sepR.push_back(v); break; }
        for (int v : L)
            for (int k = ptr[v]; k < ptr[v + 1]; ++k)
                if (side[adj[k]] == 2) { sepL.push_back(v); break; }
        const bool use_right = sepR.size() <= sepL.size();
        std::vector<int>& sep = use_right ? sepR : sepL;
        for (int v : sep) side[v] = 3;
        std::vector<int> L2, R2;
        for (int v : L) if (side[v] == 1) L2.push_back(v);
        for (int v : R) if (side[v] == 2) R2.push_back(v);
        for (int v : verts) side[v] = 0;
        std::vector<int>().swap(L);
        std::vector<int>().swap(R);
        std::vector<int>().swap(verts);
        std::vector<int> roots = run(std::move(L2));
        std::vector<int> rr = run(std::move(R2));
        roots.insert(roots.end(), rr.begin(), rr.end());
        if (sep.empty()) return roots;
        std::sort(sep.begin(), sep.end());
        return {make_front(sep, roots)};
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
    ptr.assign(nf + 1, 0);
    adj.clear();
    adj.reserve(16 * (size_t)nf);
    std::vector<int> cand;
    for (int i = 0; i < nf; ++i) {
        cand.clear();
        for (int q = vinc_ptr[i]; q < vinc_ptr[i + 1]; ++q) {
            const int e = vinc[q] >> 2;
            for (int b = 0; b < 4; ++b) {
                const int j = free_of_vert[tets[4 * (int64_t)e + b]];
                if (j >= 0 && j != i) cand.push_back(j);
            }
        }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
        adj.insert(adj.end(), cand.begin(), cand.end());
        ptr[i + 1] = static_cast<int>(adj.size());
    }
}

Symbolic analyse(int n, const std::vector<int>& adj_ptr, const std::vector<int>& adj,
                 const std::vector<double>& coords, int leaf) {
    if (n <= 0) throw std::invalid_argument("analyse: empty matrix");
    Dissector d(n, adj_ptr, adj, coords, std::max(1, leaf));
    std::vector<int> all(n);
    std::iota(all.begin(), all.end(), 0);
    d.run(std::move(all));
    Symbolic S;
    S.n = n;
    S.perm = std::move(d.order);
    S.fronts = std::move(d.fronts);
    if (static_cast<int>(S.perm.size()) != n) throw std::logic_error("analyse: ordering incomplete");
    S.iperm.assign(n, -1);
    for (int i = 0; i < n; ++i) S.iperm[S.perm[i]] = i;

    // Row structures, bottom-up (fronts are stored in post-order).
    std::vector<int> mark(n, -1);
    for (size_t fi = 0; fi < S.fronts.size(); ++fi) {
        Front& f = S.fronts[fi];
        const int last = f.first + f.ncols;
        std::vector<int> rows;
        const int tag = static_cast<int>(fi);
        for (int j = f.first; j < last; ++j) {
            const int v = S.perm[j];
            for (int k = adj_ptr[v]; k < adj_ptr[v + 1]; ++k) {
                const int i = S.iperm[adj[k]];
                if (i >= last && mark[i] != tag) { mark[i] = tag; rows.push_back(i); }
            }
        }
        for (int c : f.children)
            for (int i : S.fronts[c].rows)
                if (i >= last && mark[i] != tag) { mark[i] = tag; rows.push_back(i); }
        std::sort(rows.begin(), rows.end());
        f.rows = std::move(rows);
    }
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
