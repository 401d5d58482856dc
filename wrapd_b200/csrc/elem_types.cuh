// Device views of the per-element state shared by the kernels and the host
// orchestration.
#pragma once
#include "common.cuh"

namespace wrapd {

enum : int { MODEL_NH = 0, MODEL_ARAP = 1 };

struct Material {
    double mu, lambda;
    double wr, wmin, wmax;   // rest stiffness k and its beta_min / beta_max multiples
    int model;               // MODEL_NH or MODEL_ARAP (ARAP: psi = |F - R|^2 / 2, k = 1)
    int pad;
};

struct ElemView {
    int ne;
    const int4* idx;     // per vertex slot: free vertex (dissection order) or -(pin + 1)
    const double* Di;    // 12 x ne: Di(r, a) at [(r + 3a) * ne + e], Di = (S Dm^-1)^T
    const double* vol;
    double* w2;
    double* w2c;
    double* Z;           // 9 x ne, the reference's Mat3x3 m_Zi (column-major)
    double* U;           // 9 x ne, m_Ui
    double* symF;        // 9 x ne, cached V diag(sigma) V^T at the last gradient point
    double* sig;         // 3 x ne, cached singular values at the last gradient point
    double* slast;       // 3 x ne, prox warm start (m_last_sigma)
    double* gel;         // 12 x ne, per-element gradient rows g(a, r) at [(r + 3a) * ne + e]
    const int* mid;      // per element: index into mats (a batch of meshes of several materials), or null
    const Material* mats;
};

// ---- per-mesh vectors of the global step ------------------------------------
// Each mesh of a batch keeps its own L-BFGS state (SplitLBFGS, one per
// reference Solver): its gradients, its history and its decisions.  The
// n x 3 vectors are shared buffers in which each mesh owns its range of free
// vertices; which buffer plays which role is per mesh:
//   gradients: a ring of three, cur = G[grot % 3], new = G[(grot + 1) % 3],
//     old = G[(grot + 2) % 3]; "grad_old <- grad, grad <- grad_new" is grot + 1;
//   history: a ring of M + 1 (s, y) slots, logical entry i (oldest first) at
//     slot (head + i) % (M + 1), the next pair written to `stage`, the one slot
//     no live entry uses; "erase the oldest, push" is head + 1.
constexpr int kMaxHistory = 32;   // longest global L-BFGS history (lbfgs_m)
constexpr int kHistSlots = kMaxHistory + 1;
struct MeshCtl {
    int grot;      // gradient ring position
    int head;      // history slot of the oldest live entry
    int k;         // live history entries (SplitLBFGS m_k)
    int it;        // two-loop length of the current inner iteration, min(M, k)
    int stage;     // history slot that receives the next s and y
    int small;     // the two-loop runs in one CTA (3 x free vertices <= kTwoLoopMaxN)
    int v0, v1;    // the mesh's range in the n x 3 vectors, in doubles
};
// Slots of the two-loop recursion's scalars in a mesh's scalar block.
struct TwoLoopSlots {
    int alpha, c, dir;    // offsets in a mesh's scalar block
};
struct VecPools {
    double* G[3];
    double* S[kHistSlots];
    double* Y[kHistSlots];
    int M;         // history length (lbfgs_m); slots are taken mod M + 1
};

// The material of element e: the batch's per-mesh table when there is one,
// else the handle's single material m0 (also for lanes past the end).
__device__ __forceinline__ Material elem_material(const ElemView& E, const Material& m0, int e) {
    return (E.mid && e < E.ne) ? E.mats[E.mid[e]] : m0;
}

}  // namespace wrapd
