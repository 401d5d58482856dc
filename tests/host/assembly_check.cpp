// CPU check of the host-side setup that the GPU factorization consumes: the
// free-vertex graph, the symbolic analysis and the assembly scatter map of A
// (free_vertex_graph, analyse, assembly_map in wrapd_b200/csrc/symbolic.cpp).
//
//   assembly_check <rest.bin> <tets.bin> <pins.bin> <threads>
//
// Reads a mesh (float64 n x 3, int32 m x 4, int32 pins), then checks that
//   * every entry {i, j} of A lists exactly the element slots that hold both
//     vertices, in element order (e * 16 + a * 4 + b; e * 16 + a * 5 on the
//     diagonal), as the reference's triplet loop visits them
//     (src/TetElements.cpp:483-510);
//   * every entry lands in the lower triangle of the front that owns its
//     column, at the row of its other vertex;
//   * graph, analysis and map are identical with 1 and with <threads> host
//     threads (WRAPD_HOST_THREADS).
// Prints "ok" and exits 0, or names the first mismatch and exits 1.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../wrapd_b200/csrc/symbolic.hpp"

using namespace wrapd;

namespace {

template <typename T>
std::vector<T> read_all(const char* path) {
    FILE* f = std::fopen(path, "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path); std::exit(2); }
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f) / static_cast<long>(sizeof(T));
    std::fseek(f, 0, SEEK_SET);
    std::vector<T> v(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != static_cast<size_t>(n)) { std::fprintf(stderr, "short read\n"); std::exit(2); }
    std::fclose(f);
    return v;
}

struct Setup {
    std::vector<int> vinc_ptr, vinc, ptr, adj;
    Symbolic S;
    std::vector<int64_t> A_pos;
    std::vector<int> A_ptr, A_con;
};

Setup run(const std::vector<double>& X, const std::vector<int>& T, const std::vector<int>& fov, int nf) {
    Setup s;
    const int nv = static_cast<int>(X.size() / 3), ne = static_cast<int>(T.size() / 4);
    free_vertex_graph(nf, ne, T.data(), fov.data(), s.vinc_ptr, s.vinc, s.ptr, s.adj);
    std::vector<double> c(3 * static_cast<size_t>(nf));
    for (int i = 0; i < nv; ++i)
        if (fov[i] >= 0)
            for (int d = 0; d < 3; ++d) c[3 * static_cast<size_t>(fov[i]) + d] = X[3 * static_cast<size_t>(i) + d];
    s.S = analyse(nf, s.ptr, s.adj, c, 64);
    assembly_map(s.S, s.vinc_ptr, s.vinc, s.ptr, s.adj, s.A_pos, s.A_ptr, s.A_con);
    return s;
}

bool same(const Setup& a, const Setup& b) {
    if (a.vinc_ptr != b.vinc_ptr || a.vinc != b.vinc || a.ptr != b.ptr || a.adj != b.adj) return false;
    if (a.A_pos != b.A_pos || a.A_ptr != b.A_ptr || a.A_con != b.A_con) return false;
    const Symbolic &x = a.S, &y = b.S;
    if (x.perm != y.perm || x.levels != y.levels || x.relmap != y.relmap || x.fronts.size() != y.fronts.size()) return false;
    if (x.f_pool != y.f_pool || x.y_pool != y.y_pool || x.nnz_L != y.nnz_L || x.flops != y.flops) return false;
    for (size_t f = 0; f < x.fronts.size(); ++f) {
        const Front &p = x.fronts[f], &q = y.fronts[f];
        if (p.first != q.first || p.ncols != q.ncols || p.rows != q.rows || p.parent != q.parent ||
            p.children != q.children || p.level != q.level || p.f_off != q.f_off || p.y_off != q.y_off)
            return false;
    }
    return true;
}

int fail(const std::string& what) {
    std::printf("mismatch: %s\n", what.c_str());
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 5) { std::fprintf(stderr, "usage: assembly_check rest.bin tets.bin pins.bin threads\n"); return 2; }
    const std::vector<double> X = read_all<double>(argv[1]);
    const std::vector<int> T = read_all<int>(argv[2]);
    std::vector<int> P = read_all<int>(argv[3]);
    const int nv = static_cast<int>(X.size() / 3);
    std::sort(P.begin(), P.end());
    std::vector<int> fov(nv, -1);
    int nf = 0;
    for (int i = 0, j = 0; i < nv; ++i) {
        if (j < static_cast<int>(P.size()) && i == P[j]) ++j;
        else fov[i] = nf++;
    }
    setenv("WRAPD_HOST_THREADS", argv[4], 1);
    const Setup s = run(X, T, fov, nf);
    setenv("WRAPD_HOST_THREADS", "1", 1);
    const Setup s1 = run(X, T, fov, nf);
    if (!same(s, s1)) return fail(std::string("results differ between 1 and ") + argv[4] + " host threads");

    const Symbolic& S = s.S;
    std::vector<int> col2front(nf);
    for (size_t f = 0; f < S.fronts.size(); ++f)
        for (int j = 0; j < S.fronts[f].ncols; ++j) col2front[S.fronts[f].first + j] = static_cast<int>(f);
    // slot of each free vertex in each element (-1 if absent)
    auto slot = [&](int e, int i) {
        for (int a = 0; a < 4; ++a)
            if (fov[T[4 * static_cast<size_t>(e) + a]] == i) return a;
        return -1;
    };
    int64_t t = 0;
    for (int i = 0; i < nf; ++i) {
        std::vector<int> js = {i};
        for (int q = s.ptr[i]; q < s.ptr[i + 1]; ++q)
            if (s.adj[q] > i) js.push_back(s.adj[q]);
        for (int j : js) {
            // expected contributions, element order
            std::vector<int> want;
            for (int q = s.vinc_ptr[i]; q < s.vinc_ptr[i + 1]; ++q) {
                const int e = s.vinc[q] >> 2, a = s.vinc[q] & 3;
                if (slot(e, i) != a) return fail("incidence slot of vertex " + std::to_string(i));
                if (i == j) want.push_back(e * 16 + a * 5);
                else if (const int b = slot(e, j); b >= 0) want.push_back(e * 16 + a * 4 + b);
            }
            const std::vector<int> got(s.A_con.begin() + s.A_ptr[t], s.A_con.begin() + s.A_ptr[t + 1]);
            if (got != want || want.empty())
                return fail("contributions of entry {" + std::to_string(i) + ", " + std::to_string(j) + "}");
            // pool position: lower triangle of the front owning the column
            const int si = S.iperm[i], sj = S.iperm[j];
            const int r = std::max(si, sj), c = std::min(si, sj);
            const Front& F = S.fronts[col2front[c]];
            const int64_t off = s.A_pos[t] - F.f_off;
            const int64_t lr = off % F.ld(), lc = off / F.ld();
            const int row = lr < F.ncols ? F.first + static_cast<int>(lr)
                                         : (lr - F.ncols < F.nrows() ? F.rows[lr - F.ncols] : -1);
            if (off < 0 || lc != c - F.first || row != r || lr < lc)
                return fail("pool position of entry {" + std::to_string(i) + ", " + std::to_string(j) + "}");
            ++t;
        }
    }
    if (t + 1 != static_cast<int64_t>(s.A_ptr.size())) return fail("entry count");
    std::printf("ok: %d free vertices, %lld entries, %zu fronts\n", nf, static_cast<long long>(t), S.fronts.size());
    return 0;
}
