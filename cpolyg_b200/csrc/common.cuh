// Shared definitions of the cpolyg_b200 library: context, error handling,
// launch accounting, Legendre basis and quadrature rules on the device.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/cpolyg.h"

struct cpg_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t launches = 0;
    int num_sms = 148;
    // grow-only device scratch for reductions and small vectors
    double *scratch = nullptr;
    size_t scratch_cap = 0;  // doubles
    // pinned host staging for small read-backs
    double *pinned = nullptr;
    size_t pinned_cap = 0;
    int *flag_dev = nullptr;  // device status word (singular pivots etc.)
    // 1: cpg_precond_apply and cpg_assemble leave their device status words
    // to the next cpg_ctx_sync instead of synchronizing to read them
    int deferred_checks = 0;
    // while a Krylov cycle is enqueued without host synchronisation: device
    // word that is set once every system of the solve has converged; the
    // block-row and sweep kernels then return at once (null otherwise)
    const int *skip_dev = nullptr;
    // grow-only Krylov workspace (basis vectors), kept across solves
    double *kws = nullptr;
    size_t kws_cap = 0;  // doubles
};

namespace cpg {

cpg_status fail(cpg_ctx *ctx, cpg_status s, const std::string &msg);
cpg_status cuda_fail(cpg_ctx *ctx, cudaError_t e, const char *where);
// device scratch of at least n doubles (grow-only, stream ordered)
cpg_status scratch(cpg_ctx *ctx, size_t n, double **out);
cpg_status pinned(cpg_ctx *ctx, size_t n, double **out);
// check the last launch; increments the launch counter
cpg_status launched(cpg_ctx *ctx, const char *what);
// Raises a kernel's dynamic shared-memory limit to `bytes` (or leaves it if
// already raised) on the context's device, once: the first call for a
// (kernel, device) sets it and records it under a process-wide lock, later
// calls only look it up.  Callers pass the largest size the kernel is ever
// launched with.  The driver does not tolerate the attribute being set while
// another host thread launches the same kernel (one context per thread in
// the serving loop), so no launch site may set it directly.
cpg_status smem_limit_once(cpg_ctx *ctx, const void *kernel, int bytes);
// slot of ctx->flag_dev where the residual kernel records the first cell
// (+1) whose state is not admissible (0 = none)
constexpr int FLAG_NONPHYS = 8;
// synchronizes the context's stream, then reads and clears that slot:
// CPG_ERR_NONPHYSICAL naming the cell and `where` if it was set
cpg_status check_state(cpg_ctx *ctx, const std::string &where);

template <class T>
cpg_status dmalloc(cpg_ctx *ctx, T **p, size_t n) {
    *p = nullptr;
    if (n == 0) return CPG_OK;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        (void)cudaGetLastError();
        return fail(ctx, CPG_ERR_OOM, std::string("cudaMalloc of ") + std::to_string(n * sizeof(T)) + " bytes failed");
    }
    return CPG_OK;
}
template <class T>
cpg_status upload(cpg_ctx *ctx, T **p, const std::vector<T> &h) {
    cpg_status s = dmalloc(ctx, p, h.size());
    if (s != CPG_OK || h.empty()) return s;
    cudaError_t e = cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload");
    e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "upload sync");
    return CPG_OK;
}
inline void dfree(void *p) {
    if (p) cudaFree(p);
}

#define CPG_TRY(expr)                          \
    do {                                       \
        cpg_status _s = (expr);                \
        if (_s != CPG_OK) return _s;           \
    } while (0)

#define CPG_CUDA(ctx, expr)                                   \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) return cpg::cuda_fail(ctx, _e, #expr); \
    } while (0)

// ---------------------------------------------------------------------------
// Legendre polynomials P_0..P_3 and derivatives (Leg2D, src/Legendre.h:51-68;
// the derivative coefficients of LegDerX/Y, src/Legendre.cpp:34-124, are the
// exact derivatives P_l' evaluated here directly).
// ---------------------------------------------------------------------------
template <int P>
__host__ __device__ __forceinline__ void legendre(double x, double *v, double *d) {
    v[0] = 1.0;
    d[0] = 0.0;
    if (P >= 1) {
        v[1] = x;
        d[1] = 1.0;
    }
    if (P >= 2) {
        v[2] = 0.5 * (3.0 * x * x - 1.0);
        d[2] = 3.0 * x;
    }
    if (P >= 3) {
        v[3] = 0.5 * x * (5.0 * x * x - 3.0);
        d[3] = 7.5 * x * x - 1.5;
    }
}
template <int P>
__host__ __device__ __forceinline__ void legendre_v(double x, double *v) {
    v[0] = 1.0;
    if (P >= 1) v[1] = x;
    if (P >= 2) v[2] = 0.5 * (3.0 * x * x - 1.0);
    if (P >= 3) v[3] = 0.5 * x * (5.0 * x * x - 3.0);
}
// basis index k <-> (i, j): x-degree outer, y-degree inner (Legendre.h:20-35)
template <int P>
__host__ __device__ constexpr int nbasis() { return (P + 1) * (P + 2) / 2; }

// psi_k(x, y) for all k
template <int P>
__host__ __device__ __forceinline__ void basis(double xi, double eta, double *psi) {
    double px[P + 1], py[P + 1];
    legendre_v<P>(xi, px);
    legendre_v<P>(eta, py);
    int k = 0;
#pragma unroll
    for (int i = 0; i <= P; i++)
#pragma unroll
        for (int j = 0; j <= P - i; j++) psi[k++] = px[i] * py[j];
}
// psi_k and its physical gradient (scaled by 2/w, 2/h)
template <int P>
__host__ __device__ __forceinline__ void basis_grad(double xi, double eta, double sx, double sy,
                                                    double *psi, double *dx, double *dy) {
    double px[P + 1], py[P + 1], dpx[P + 1], dpy[P + 1];
    legendre<P>(xi, px, dpx);
    legendre<P>(eta, py, dpy);
    int k = 0;
#pragma unroll
    for (int i = 0; i <= P; i++)
#pragma unroll
        for (int j = 0; j <= P - i; j++) {
            psi[k] = px[i] * py[j];
            dx[k] = sx * dpx[i] * py[j];
            dy[k] = sy * px[i] * dpy[j];
            k++;
        }
}

}  // namespace cpg
