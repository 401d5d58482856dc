// Host-side symbolic analysis for the GPU multifrontal Cholesky of the
// free-vertex weighted Laplacian A = sum_e w_e^2 D_e^T D_e (the matrix the
// reference factors with Eigen's SimplicialLDLT in
// deps/mcloptlib/include/MCL/LinearSolver.hpp:279-298, built by
// src/TetElements.cpp:483-510).  Integer work only, done once per mesh:
//   * a fill-reducing order by geometric nested dissection on the rest
//     positions (recursive median cuts along the longest box axis, one-sided
//     vertex separators);
//   * the separator tree as the assembly tree: every separator or leaf block
//     is one dense front whose columns are contiguous in the new order;
//   * each front's row structure, the relative-index maps for extend-add,
//     the device pool offsets, and the level schedule (a front's level is one
//     more than its highest child's, so each level can run as one launch).
#pragma once
#include <cstdint>
#include <functional>
#include <vector>

namespace wrapd {

struct Front {
    int first = 0;             // first column (new numbering)
    int ncols = 0;             // k
    std::vector<int> rows;     // r struct rows (new numbering, sorted, > last column)
    int parent = -1;
    std::vector<int> children;
    int level = 0;
    int64_t f_off = 0;         // F pool: (k + r) x (k + r) column-major, leading dimension ld()
    int64_t y_off = 0;         // Y pool: [inv(L_ss); L_rs inv(L_ss)], (k + r) x k column-major, ld yw_ld(k, r)
    int64_t u_off = 0;         // solve update pool: r x 3
    int64_t rel_off = 0;       // this front's map of `rows` into the parent's front rows
    // leading dimension of the front's F-pool block: k + r rounded up to even (the
    // padding row and column stay zero), so columns start on 16-byte boundaries
    int ld() const { return (ncols + static_cast<int>(rows.size()) + 1) & ~1; }
    int nrows() const { return static_cast<int>(rows.size()); }
};

// Leading dimension of a front's block in the Y pool: k + r rounded up to even,
// so every 64-row band of a column starts on a 16-byte boundary.
inline int64_t yw_ld(int64_t k, int64_t r) { return (k + r + 1) & ~int64_t(1); }

struct Symbolic {
    int n = 0;
    std::vector<int> perm;    // new -> old
    std::vector<int> iperm;   // old -> new
    std::vector<Front> fronts;
    std::vector<std::vector<int>> levels;  // front ids per level (level 0 = leaves)
    std::vector<int> relmap;  // concatenated child -> parent relative row maps
    int64_t f_pool = 0, y_pool = 0, u_pool = 0;
    int max_children = 0;
    // statistics
    int64_t nnz_L = 0;        // stored entries of the factor panels (dense fronts)
    double flops = 0.0;       // factorization flops (dense front model)
};

// The free-vertex graph of a tet mesh (the sparsity of A, src/TetElements.cpp:
// 483-510).  free_of_vert[v] is vertex v's free index (ascending vertex id,
// pinned vertices skipped) or -1 for a pinned vertex.  Outputs, per free vertex
// i: vinc[vinc_ptr[i] .. vinc_ptr[i+1]) its element incidences e * 4 + a (slot
// a of element e) in element order, and adj[ptr[i] .. ptr[i+1]) the other free
// vertices of those elements, sorted and unique.
void free_vertex_graph(int nf, int ne, const int* tets, const int* free_of_vert, std::vector<int>& vinc_ptr,
                       std::vector<int>& vinc, std::vector<int>& ptr, std::vector<int>& adj);

// adj_ptr/adj: symmetric adjacency of the n free vertices (no self loops).
// coords: n x 3 positions used for the geometric cuts.  leaf: max leaf size.
Symbolic analyse(int n, const std::vector<int>& adj_ptr, const std::vector<int>& adj,
                 const std::vector<double>& coords, int leaf);

// The assembly scatter map of A's lower triangle into the F pool (A is the
// sum of the reference's triplets, src/TetElements.cpp:483-510).  Entries are
// the unordered free-vertex pairs {i, j}, i <= j (free numbering), entry ids
// ebase[i] + the rank of j in {i} + {neighbours of i above i}.  Entry t sums
// the contributions A_con[A_ptr[t] .. A_ptr[t+1]) = e * 16 + a * 4 + b (slot a
// of element e holds the lower free index, slot b the other) in element
// order, and lands at F-pool offset A_pos[t] (lower triangle in the
// dissection order of S).  vinc/ptr/adj as free_vertex_graph gives them.
void assembly_map(const Symbolic& S, const std::vector<int>& vinc_ptr, const std::vector<int>& vinc,
                  const std::vector<int>& ptr, const std::vector<int>& adj, std::vector<int64_t>& A_pos,
                  std::vector<int>& A_ptr, std::vector<int>& A_con);

// The analysis of a block-diagonal matrix from the analyses of its blocks (one
// per mesh of a batch), block p taking the columns after blocks 0..p-1: the
// forest of their trees, level l holding every block's level-l fronts.
Symbolic merge(const std::vector<Symbolic>& parts);

// fn(lo, hi) over contiguous ranges of [0, n) on host threads (one per `grain`
// items, at most 16 or WRAPD_HOST_THREADS); exceptions are rethrown after the
// join.
void host_parallel(int n, int64_t grain, const std::function<void(int, int)>& fn);

}  // namespace wrapd
