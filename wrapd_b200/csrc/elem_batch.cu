// Batched entry points over the per-element device math (the same svd3,
// prox_lbfgs and hess_lmax the ADMM kernels inline), for parity checks of
// each function on its own.  Handle-free; they run on the current device.
#include <mutex>
#include <vector>

#include "elem_math.cuh"

namespace wrapd {
namespace {

template <typename T>
__global__ void k_svd_batch(int n, const double* __restrict__ F, double* __restrict__ sig, double* __restrict__ U,
                            double* __restrict__ V) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    T f[9], s[3], u[9], v[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) f[i] = T(F[9 * (size_t)e + i]);
    svd3(f, s, u, v);
#pragma unroll
    for (int i = 0; i < 3; ++i) sig[3 * (size_t)e + i] = s[i];
#pragma unroll
    for (int i = 0; i < 9; ++i) { U[9 * (size_t)e + i] = u[i]; V[9 * (size_t)e + i] = v[i]; }
}

template <typename T>
__global__ void k_prox_batch(int n, double mu, double lambda, int max_iters, const double* __restrict__ s0,
                             const double* __restrict__ wov, const double* __restrict__ start, double* __restrict__ out,
                             int* __restrict__ iters) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    Prox<T> P;
    P.nh.mu = T(mu);
    P.nh.lambda = T(lambda);
    T x[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { P.x0[i] = T(s0[3 * (size_t)e + i]); x[i] = T(start[3 * (size_t)e + i]); }
    P.wov = T(wov[e]);
    extern __shared__ unsigned char prox_hist_raw[];   // 48 x blockDim values of T
    T* hist = reinterpret_cast<T*>(prox_hist_raw);
    iters[e] = prox_lbfgs(P, x, max_iters, ProxHistory<T>{hist + threadIdx.x, (int)blockDim.x});
#pragma unroll
    for (int i = 0; i < 3; ++i) out[3 * (size_t)e + i] = x[i];
}

template <typename T>
__global__ void k_newton_batch(int n, double mu, double lambda, double tol, int max_iters,
                               const double* __restrict__ s0, const double* __restrict__ wov,
                               const double* __restrict__ start, double* __restrict__ out, int* __restrict__ iters) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    Prox<T> P;
    P.nh.mu = T(mu);
    P.nh.lambda = T(lambda);
    T x[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { P.x0[i] = T(s0[3 * (size_t)e + i]); x[i] = T(start[3 * (size_t)e + i]); }
    P.wov = T(wov[e]);
    const int it = prox_newton(P, x, max_iters, T(tol));
    if (iters) iters[e] = it;
#pragma unroll
    for (int i = 0; i < 3; ++i) out[3 * (size_t)e + i] = x[i];
}

// potential_energy_x + inversion_count over a batch of stretch triples
// (src/TetElements.cpp:598-635, 444-468): out[0] = sum vol * psi(sigma),
// out[1] = number of triples with a negative entry.  Deterministic two-level
// sum: per-block partials in `partials`, added in block order by the last block.
__global__ void __launch_bounds__(256) k_energy_batch(int n, double mu, double lambda,
                                                      const double* __restrict__ sigma,
                                                      const double* __restrict__ vol, double* partials,
                                                      unsigned* counter, double* out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double red[2] = {0.0, 0.0};
    if (e < n) {
        const double* s = sigma + 3 * (size_t)e;
        red[0] = vol[e] * NH<double>{mu, lambda}.psi_plain(s[0], s[1], s[2]);
        red[1] = (s[0] < 0.0 || s[1] < 0.0 || s[2] < 0.0) ? 1.0 : 0.0;
    }
    grid_reduce<2>(red, partials, counter, out);
}

__global__ void k_hess_batch(int n, double mu, double lambda, const double* __restrict__ s, double* __restrict__ out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const double x[3] = {s[3 * (size_t)e], s[3 * (size_t)e + 1], s[3 * (size_t)e + 2]};
    out[e] = NH<double>{mu, lambda}.hess_lmax(x);
}

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t bytes) {
        if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) { cudaGetLastError(); p = nullptr; }
    }
    ~DevBuf() { if (p) cudaFree(p); }
    template <typename X> X* as() const { return static_cast<X*>(p); }
};

int finish(cudaError_t e) {
    if (e == cudaErrorMemoryAllocation) return WRAPD_E_OOM;
    return e == cudaSuccess ? WRAPD_OK : WRAPD_E_CUDA;
}

// ---- fixed scratch for wrapd_potential_energy_batch_noalloc ------------------
// The reduction needs one partial pair per 256-element block plus a block
// counter.  This array is that scratch, sized for the largest batch the entry
// point accepts; every device that loads the library holds it (about 1 MiB)
// until the process exits.
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 65536;                       // 16,777,216 elements per call
constexpr int kNoAllocScratch = 2 * kNoAllocMaxBlocks + 32;    // partials, then the counter
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratch];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_addr[kMaxDevices] = {};   // device address of the array, per device

// Host code may not hand `g_noalloc_scratch` to a kernel: on the host that name
// is only a stand-in for the device variable.  Look the device address up
// once per device, with that device current.
int noalloc_scratch(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) { cudaGetLastError(); return WRAPD_E_CUDA; }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) { cudaGetLastError(); return WRAPD_E_CUDA; }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_addr[dev];
    return WRAPD_OK;
}

}  // namespace
}  // namespace wrapd

using namespace wrapd;

extern "C" {

WRAPD_API int wrapd_svd3_batch(int n, int fp32, const double* F, double* sigma, double* U, double* V) {
    if (n < 0 || (n > 0 && (!F || !sigma || !U || !V))) return WRAPD_E_INPUT;
    if (n == 0) return WRAPD_OK;
    DevBuf dF(9 * (size_t)n * 8), dS(3 * (size_t)n * 8), dU(9 * (size_t)n * 8), dV(9 * (size_t)n * 8);
    if (!dF.p || !dS.p || !dU.p || !dV.p) return WRAPD_E_OOM;
    cudaError_t e = cudaMemcpy(dF.p, F, 9 * (size_t)n * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return finish(e);
    const int b = (n + 127) / 128;
    if (fp32) k_svd_batch<float><<<b, 128>>>(n, dF.as<double>(), dS.as<double>(), dU.as<double>(), dV.as<double>());
    else k_svd_batch<double><<<b, 128>>>(n, dF.as<double>(), dS.as<double>(), dU.as<double>(), dV.as<double>());
    if ((e = cudaGetLastError()) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(sigma, dS.p, 3 * (size_t)n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(U, dU.p, 9 * (size_t)n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(V, dV.p, 9 * (size_t)n * 8, cudaMemcpyDeviceToHost));
}

WRAPD_API int wrapd_prox_batch(int n, int fp32, double mu, double lambda, int max_iters, const double* sigma0,
                               const double* wov, const double* start, double* out, int* iters) {
    if (n < 0 || max_iters < 1 || (n > 0 && (!sigma0 || !wov || !start || !out || !iters))) return WRAPD_E_INPUT;
    if (n == 0) return WRAPD_OK;
    DevBuf d0(3 * (size_t)n * 8), dw((size_t)n * 8), ds(3 * (size_t)n * 8), dout(3 * (size_t)n * 8), dit((size_t)n * 4);
    if (!d0.p || !dw.p || !ds.p || !dout.p || !dit.p) return WRAPD_E_OOM;
    cudaError_t e;
    if ((e = cudaMemcpy(d0.p, sigma0, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(dw.p, wov, (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(ds.p, start, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    const int b = fp32 ? (n + 127) / 128 : (n + 63) / 64;
    if (fp32)
        k_prox_batch<float><<<b, 128, 48 * 128 * sizeof(float)>>>(n, mu, lambda, max_iters, d0.as<double>(),
                                                                  dw.as<double>(), ds.as<double>(), dout.as<double>(),
                                                                  dit.as<int>());
    else
        k_prox_batch<double><<<b, 64, 48 * 64 * sizeof(double)>>>(n, mu, lambda, max_iters, d0.as<double>(),
                                                                  dw.as<double>(), ds.as<double>(), dout.as<double>(),
                                                                  dit.as<int>());
    if ((e = cudaGetLastError()) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(out, dout.p, 3 * (size_t)n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(iters, dit.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
}

WRAPD_API int wrapd_prox_newton_batch(int n, int fp32, double mu, double lambda, double tol, int max_iters,
                                      const double* sigma0, const double* wov, const double* start, double* out,
                                      int* iters) {
    if (n < 0 || max_iters < 0 || !(tol > 0.0) || (n > 0 && (!sigma0 || !wov || !start || !out))) return WRAPD_E_INPUT;
    if (n == 0) return WRAPD_OK;
    DevBuf d0(3 * (size_t)n * 8), dw((size_t)n * 8), ds(3 * (size_t)n * 8), dout(3 * (size_t)n * 8),
        dit((size_t)n * 4);
    if (!d0.p || !dw.p || !ds.p || !dout.p || !dit.p) return WRAPD_E_OOM;
    cudaError_t e;
    if ((e = cudaMemcpy(d0.p, sigma0, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(dw.p, wov, (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(ds.p, start, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    const int b = (n + 127) / 128;
    if (fp32)
        k_newton_batch<float><<<b, 128>>>(n, mu, lambda, tol, max_iters, d0.as<double>(), dw.as<double>(),
                                          ds.as<double>(), dout.as<double>(), dit.as<int>());
    else
        k_newton_batch<double><<<b, 128>>>(n, mu, lambda, tol, max_iters, d0.as<double>(), dw.as<double>(),
                                           ds.as<double>(), dout.as<double>(), dit.as<int>());
    if ((e = cudaGetLastError()) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(out, dout.p, 3 * (size_t)n * 8, cudaMemcpyDeviceToHost)) != cudaSuccess) return finish(e);
    if (!iters) return finish(cudaDeviceSynchronize());
    return finish(cudaMemcpy(iters, dit.p, (size_t)n * 4, cudaMemcpyDeviceToHost));
}

WRAPD_API int wrapd_potential_energy_batch(int n, double mu, double lambda, const double* sigma, const double* vol,
                                           double* pe, int* flips) {
    if (n < 0 || !pe || !flips || (n > 0 && (!sigma || !vol))) return WRAPD_E_INPUT;
    if (n == 0) { *pe = 0.0; *flips = 0; return WRAPD_OK; }
    const int blocks = (n + 255) / 256;
    DevBuf ds(3 * (size_t)n * 8), dv((size_t)n * 8), dp(2 * (size_t)blocks * 8), dc(sizeof(unsigned)), dout(16);
    if (!ds.p || !dv.p || !dp.p || !dc.p || !dout.p) return WRAPD_E_OOM;
    cudaError_t e;
    if ((e = cudaMemcpy(ds.p, sigma, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemcpy(dv.p, vol, (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    if ((e = cudaMemset(dc.p, 0, sizeof(unsigned))) != cudaSuccess) return finish(e);
    k_energy_batch<<<blocks, 256>>>(n, mu, lambda, ds.as<double>(), dv.as<double>(), dp.as<double>(),
                                    dc.as<unsigned>(), dout.as<double>());
    if ((e = cudaGetLastError()) != cudaSuccess) return finish(e);
    double out[2];
    if ((e = cudaMemcpy(out, dout.p, 16, cudaMemcpyDeviceToHost)) != cudaSuccess) return finish(e);
    *pe = out[0];
    *flips = (int)out[1];
    return WRAPD_OK;
}

// Same sums as wrapd_potential_energy_batch, for callers that cannot allocate
// device memory: inputs and the output live in caller memory on the device and
// the reduction's scratch is the fixed array above, so this call allocates
// nothing.  See include/wrapd_gpu.h for the contract.
WRAPD_API int wrapd_potential_energy_batch_noalloc(int n, double mu, double lambda, const double* d_sigma,
                                                   const double* d_vol, double* d_out, void* stream) {
    if (n < 0 || n > kNoAllocMaxBlocks * kNoAllocThreads || !d_out || (n > 0 && (!d_sigma || !d_vol)))
        return WRAPD_E_INPUT;
    double* scratch = nullptr;
    const int rc = noalloc_scratch(&scratch);
    if (rc != WRAPD_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned* counter = reinterpret_cast<unsigned*>(scratch + 2 * kNoAllocMaxBlocks);
    // the array keeps the previous call's contents: the block counter must start at zero
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return finish(e);
    if (n == 0) return finish(cudaMemsetAsync(d_out, 0, 2 * sizeof(double), st));
    const int blocks = (n + kNoAllocThreads - 1) / kNoAllocThreads;
    k_energy_batch<<<blocks, kNoAllocThreads, 0, st>>>(n, mu, lambda, d_sigma, d_vol, scratch, counter, d_out);
    return finish(cudaGetLastError());
}

WRAPD_API int wrapd_hess_lmax_batch(int n, double mu, double lambda, const double* sigma, double* out) {
    if (n < 0 || (n > 0 && (!sigma || !out))) return WRAPD_E_INPUT;
    if (n == 0) return WRAPD_OK;
    DevBuf ds(3 * (size_t)n * 8), dout((size_t)n * 8);
    if (!ds.p || !dout.p) return WRAPD_E_OOM;
    cudaError_t e;
    if ((e = cudaMemcpy(ds.p, sigma, 3 * (size_t)n * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return finish(e);
    k_hess_batch<<<(n + 127) / 128, 128>>>(n, mu, lambda, ds.as<double>(), dout.as<double>());
    if ((e = cudaGetLastError()) != cudaSuccess) return finish(e);
    return finish(cudaMemcpy(out, dout.p, (size_t)n * 8, cudaMemcpyDeviceToHost));
}

}  // extern "C"
