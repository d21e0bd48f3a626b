// Block-sparse matrices: storage, matvec (BlockMatrix::matvec), block ILU(0)
// factor/apply (BlockILU0) and block Jacobi (BlockJacobi).
//
// All row operations share one streaming kernel: a CTA walks the contiguous
// value array of one block row with vector loads.  Because the load stride
// (threads x vector width) is a multiple of the block size, every thread
// keeps the same block rows for the whole walk and only the column (and the
// block) advances; partial sums of the column groups meet in shared memory.
//   MATVEC   y_i = sum_k A_k x_{c_k}
//   FORWARD  x_i = x_i - sum_k L_k x_{c_k}           (ILU forward sweep)
//   BACKWARD x_i = D^{-1}_i x_i - sum_k U_k x_{c_k}   (ILU backward sweep,
//            the row's first block is D^{-1}_i; block Jacobi has only it)
// Triangular sweeps either run sync-free (k_sweep, one launch per sweep) or
// one launch per level of the level schedule computed from the block pattern.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "internal.hpp"

using namespace cpg;

namespace {

enum { MODE_MATVEC = 0, MODE_FORWARD = 1, MODE_BACKWARD = 2 };

template <class T, int VEC>
struct VecLoad;
template <>
struct VecLoad<double, 1> {
    static __device__ __forceinline__ void ld(const double *p, double *v) { v[0] = __ldcs(p); }
};
template <>
struct VecLoad<double, 2> {
    static __device__ __forceinline__ void ld(const double *p, double *v) {
        const double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
        v[0] = a.x;
        v[1] = a.y;
    }
};
template <>
struct VecLoad<float, 1> {
    static __device__ __forceinline__ void ld(const float *p, double *v) { v[0] = (double)__ldcs(p); }
};
template <>
struct VecLoad<float, 2> {
    static __device__ __forceinline__ void ld(const float *p, double *v) {
        const float2 a = __ldcs(reinterpret_cast<const float2 *>(p));
        v[0] = a.x;
        v[1] = a.y;
    }
};
template <>
struct VecLoad<float, 4> {
    static __device__ __forceinline__ void ld(const float *p, double *v) {
        const float4 a = __ldcs(reinterpret_cast<const float4 *>(p));
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
};

constexpr int MAX_ROW_BLOCKS = 64;

template <class T, int BL, int VEC, int TPR>
__global__ void __launch_bounds__(TPR) k_rows(const int *__restrict__ rows, const int *__restrict__ rowptr,
                                              const int *__restrict__ col, const T *__restrict__ vals,
                                              const double *x, double *y, int mode) {
    static_assert((TPR * VEC) % BL == 0, "stride must be a multiple of the block size");
    static_assert(BL % VEC == 0, "vector width must divide the block size");
    constexpr int S = TPR * VEC, G = S / BL, BL2 = BL * BL;
    __shared__ int scol[MAX_ROW_BLOCKS];
    __shared__ double red[G][BL];
    const int i = rows ? rows[blockIdx.x] : blockIdx.x;
    const int k0 = rowptr[i], nblk = rowptr[i + 1] - k0;
    const int tid = threadIdx.x;
    for (int q = tid; q < nblk && q < MAX_ROW_BLOCKS; q += TPR) scol[q] = col[k0 + q];
    __syncthreads();
    const int e0 = tid * VEC;
    const int r0 = e0 % BL, g = e0 / BL;
    double acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) acc[v] = 0.0;
    const T *base = vals + (size_t)k0 * BL2;
    const int E = nblk * BL2;
    // the start offset may lie beyond the first block when the stride
    // exceeds bl^2 (small blocks)
    int blk = e0 / BL2, within = e0 % BL2;
    const double s0 = (mode == MODE_FORWARD) ? -1.0 : 1.0;
    const double sr = (mode == MODE_MATVEC) ? 1.0 : -1.0;
#pragma unroll 4
    for (int e = e0; e < E; e += S) {
        const int c = within / BL;
        double a[VEC];
        VecLoad<T, VEC>::ld(base + e, a);
        const int cb = blk < MAX_ROW_BLOCKS ? scol[blk] : __ldg(col + k0 + blk);
        const double xv = __ldg(x + (size_t)cb * BL + c) * (blk == 0 ? s0 : sr);
#pragma unroll
        for (int v = 0; v < VEC; v++) acc[v] += a[v] * xv;
        within += S;
        while (within >= BL2) {
            within -= BL2;
            blk++;
        }
    }
#pragma unroll
    for (int v = 0; v < VEC; v++) red[g][r0 + v] = acc[v];
    __syncthreads();
    if (tid < BL) {
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < G; q++) s += red[q][tid];
        double *yi = y + (size_t)i * BL;
        if (mode == MODE_FORWARD) s = yi[tid] + s;
        yi[tid] = s;
    }
}

// generic block size: scalar loads, TPR = block size * groups
template <class T>
__global__ void __launch_bounds__(256) k_rows_dyn(int BL, int G, const int *__restrict__ rows,
                                                  const int *__restrict__ rowptr, const int *__restrict__ col,
                                                  const T *__restrict__ vals, const double *x, double *y, int mode) {
    extern __shared__ double red_dyn[];
    __shared__ int scol[MAX_ROW_BLOCKS];
    const int i = rows ? rows[blockIdx.x] : blockIdx.x;
    const int k0 = rowptr[i], nblk = rowptr[i + 1] - k0;
    const int tid = threadIdx.x, S = BL * G, BL2 = BL * BL;
    for (int q = tid; q < nblk && q < MAX_ROW_BLOCKS; q += blockDim.x) scol[q] = col[k0 + q];
    __syncthreads();
    double acc = 0.0;
    if (tid < S) {
        const int r0 = tid % BL;
        (void)r0;
        const T *base = vals + (size_t)k0 * BL2;
        const int E = nblk * BL2;
        int blk = tid / BL2, within = tid % BL2;
        const double s0 = (mode == MODE_FORWARD) ? -1.0 : 1.0;
        const double sr = (mode == MODE_MATVEC) ? 1.0 : -1.0;
        for (int e = tid; e < E; e += S) {
            const int c = within / BL;
            const int cb = blk < MAX_ROW_BLOCKS ? scol[blk] : __ldg(col + k0 + blk);
        const double xv = __ldg(x + (size_t)cb * BL + c) * (blk == 0 ? s0 : sr);
            acc += (double)base[e] * xv;
            within += S;
            while (within >= BL2) {
                within -= BL2;
                blk++;
            }
        }
        red_dyn[tid] = acc;
    }
    __syncthreads();
    if (tid < BL) {
        double s = 0.0;
        for (int q = 0; q < G; q++) s += red_dyn[q * BL + tid];
        double *yi = y + (size_t)i * BL;
        if (mode == MODE_FORWARD) s = yi[tid] + s;
        yi[tid] = s;
    }
}

// ---------------------------------------------------------------------------
// Sync-free triangular sweep: one launch for a whole forward or backward
// ILU(0) sweep.  CTAs claim rows in level order from a counter; a row first
// waits until every row it reads (its L columns, or its U columns) has
// published its value (flags[j] == gen), then computes exactly as k_rows and
// publishes its own.  A CTA only ever waits on rows claimed before its own,
// by CTAs that are running, so the sweep always progresses; every wait is
// bounded and reports through err instead of hanging.
// ---------------------------------------------------------------------------
constexpr long long SWEEP_MAX_SPINS = 1LL << 22;  // x >= 64 ns sleeps: >= 0.27 s

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

template <class T, int BL, int VEC, int TPR>
__global__ void __launch_bounds__(TPR) k_sweep(const int *__restrict__ order, int n, const int *__restrict__ rowptr,
                                               const int *__restrict__ col, const T *__restrict__ vals, double *x,
                                               int mode, int *flags, int gen, int *counter, int *err) {
    static_assert((TPR * VEC) % BL == 0, "stride must be a multiple of the block size");
    static_assert(BL % VEC == 0, "vector width must divide the block size");
    static_assert(TPR >= 64, "the claiming thread lives in the second warp");
    constexpr int S = TPR * VEC, G = S / BL, BL2 = BL * BL;
    constexpr int CLAIMER = 32;  // warp 0 holds the dependency waits
    __shared__ int s_row[2];
    __shared__ int scol[MAX_ROW_BLOCKS];
    __shared__ double red[G][BL];
    const int tid = threadIdx.x;
    const int e0 = tid * VEC;
    const int r0 = e0 % BL, g = e0 / BL;
    const double s0 = (mode == MODE_FORWARD) ? -1.0 : 1.0;
    const double sr = -1.0;
    if (tid == CLAIMER) s_row[0] = atomicAdd(counter, 1);
    __syncthreads();
    for (int cur = 0;; cur ^= 1) {
        const int q = s_row[cur];
        if (q >= n) break;
        // claim the next row now, so the atomic's round trip hides behind this row
        if (tid == CLAIMER) s_row[cur ^ 1] = atomicAdd(counter, 1);
        const int i = order[q];
        const int k0 = rowptr[i], nblk = rowptr[i + 1] - k0;
        // the backward row's first block is D^{-1}_i (its own column)
        const int first_dep = (mode == MODE_BACKWARD) ? 1 : 0;
        for (int b = tid; b < nblk; b += TPR) {
            const int j = col[k0 + b];
            if (b < MAX_ROW_BLOCKS) scol[b] = j;
            if (b >= first_dep) {
                long long spins = 0;
                while (ld_acquire(flags + j) != gen) {
                    // once any wait has given up, nobody waits any more
                    if (++spins > SWEEP_MAX_SPINS || ((spins & 255) == 0 && ld_acquire(err) != 0)) {
                        atomicExch(err, 1);
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        __syncthreads();
        double acc[VEC];
#pragma unroll
        for (int v = 0; v < VEC; v++) acc[v] = 0.0;
        const T *base = vals + (size_t)k0 * BL2;
        const int E = nblk * BL2;
        int blk = e0 / BL2, within = e0 % BL2;
#pragma unroll 4
        for (int e = e0; e < E; e += S) {
            const int c = within / BL;
            double a[VEC];
            VecLoad<T, VEC>::ld(base + e, a);
            const int cb = blk < MAX_ROW_BLOCKS ? scol[blk] : col[k0 + blk];
            // values published during this sweep: read through L2, not L1
            const double xv = __ldcg(x + (size_t)cb * BL + c) * (blk == 0 ? s0 : sr);
#pragma unroll
            for (int v = 0; v < VEC; v++) acc[v] += a[v] * xv;
            within += S;
            while (within >= BL2) {
                within -= BL2;
                blk++;
            }
        }
#pragma unroll
        for (int v = 0; v < VEC; v++) red[g][r0 + v] = acc[v];
        __syncthreads();
        if (tid < BL) {
            double s = 0.0;
#pragma unroll
            for (int qq = 0; qq < G; qq++) s += red[qq][tid];
            double *xi = x + (size_t)i * BL;
            if (mode == MODE_FORWARD) s = __ldcg(xi + tid) + s;
            __stcg(xi + tid, s);
        }
        __syncthreads();  // the row's stores (and the next claim) are done
        if (tid == 0) {
            __threadfence();
            st_release(flags + i, gen);
        }
    }
}

template <class T, int BL, int VEC, int TPR>
cpg_status launch_sweep_cfg(cpg_ctx *ctx, int nrows, const int *order, const int *rowptr, const int *col,
                            const T *vals, double *x, int mode, int *flags, int gen, int *counter, int *err) {
    int per_sm = 0;
    CPG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep<T, BL, VEC, TPR>, TPR, 0));
    const int grid = std::max(1, std::min(nrows, std::max(1, per_sm) * ctx->num_sms));
    CPG_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
    k_sweep<T, BL, VEC, TPR><<<grid, TPR, 0, ctx->stream>>>(order, nrows, rowptr, col, vals, x, mode, flags, gen,
                                                           counter, err);
    return launched(ctx, "sync-free sweep kernel");
}

// wide rows: a row's latency sits on the sweep's critical path, so each row
// is streamed by many threads (every thread issues ~1-2 vector loads per block)
template <class T>
cpg_status launch_sweep_t(cpg_ctx *ctx, int bl, int nrows, const int *order, const int *rowptr, const int *col,
                          const T *vals, double *x, int mode, int *flags, int gen, int *counter, int *err) {
    constexpr bool F32 = std::is_same<T, float>::value;
#define CPG_SWEEP(BLV, V, TT) \
    return launch_sweep_cfg<T, BLV, V, TT>(ctx, nrows, order, rowptr, col, vals, x, mode, flags, gen, counter, err)
    switch (bl) {
        case 6: CPG_SWEEP(6, 2, 384);
        case 10: CPG_SWEEP(10, 2, 640);
        case 24:
            if constexpr (F32) { CPG_SWEEP(24, 4, 288); }
            else { CPG_SWEEP(24, 2, 576); }
        case 40:
            if constexpr (F32) { CPG_SWEEP(40, 4, 640); }
            else { CPG_SWEEP(40, 2, 640); }
        default: return CPG_ERR_UNSUPPORTED;
    }
#undef CPG_SWEEP
}

template <class T>
cpg_status launch_rows_t(cpg_ctx *ctx, int bl, int nrows, const int *rows, const int *rowptr, const int *col,
                         const T *vals, const double *x, double *y, int mode, int variant) {
    if (nrows <= 0) return CPG_OK;
    cudaStream_t s = ctx->stream;
    constexpr bool F32 = std::is_same<T, float>::value;
    // threads per row: variants 0/1/2 use about 8/16/32 column groups; the
    // matvec picks its variant by timing (autotune below), level sweeps take
    // the widest variant because they are latency bound
#define CPG_ROWS3(BLV, V, T0, T1, T2)                                                                    \
    switch (variant) {                                                                                   \
        case 0: k_rows<T, BLV, V, T0><<<nrows, T0, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break;  \
        case 1: k_rows<T, BLV, V, T1><<<nrows, T1, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break;  \
        default: k_rows<T, BLV, V, T2><<<nrows, T2, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break; \
    }
    switch (bl) {
        case 1: k_rows<T, 1, 1, 32><<<nrows, 32, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break;
        case 3: k_rows<T, 3, 1, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break;
        case 4: k_rows<T, 4, 2, 64><<<nrows, 64, 0, s>>>(rows, rowptr, col, vals, x, y, mode); break;
        case 6: CPG_ROWS3(6, 2, 96, 192, 384) break;
        case 10: CPG_ROWS3(10, 2, 160, 320, 640) break;
        case 12:
            if constexpr (F32) k_rows<T, 12, 4, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode);
            else k_rows<T, 12, 2, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode);
            break;
        case 24:
            if constexpr (F32) { CPG_ROWS3(24, 4, 96, 192, 288) }
            else { CPG_ROWS3(24, 2, 192, 384, 576) }
            break;
        case 40:
            if constexpr (F32) { CPG_ROWS3(40, 4, 160, 320, 640) }
            else { CPG_ROWS3(40, 2, 160, 320, 640) }
            break;
        case 48:
            if constexpr (F32) { CPG_ROWS3(48, 4, 192, 384, 768) }
            else { CPG_ROWS3(48, 2, 192, 384, 768) }
            break;
        default: {
            if (bl > 256) return fail(ctx, CPG_ERR_UNSUPPORTED, "block size above 256");
            const int G = std::max(1, 256 / bl);
            k_rows_dyn<T><<<nrows, 256, sizeof(double) * bl * G, s>>>(bl, G, rows, rowptr, col, vals, x, y, mode);
        }
    }
#undef CPG_ROWS3
    return launched(ctx, "block-row kernel");
}

cpg_status launch_rows_v(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                         const int *col, const void *vals, const double *x, double *y, int mode, int variant) {
    if (precision == CPG_F32)
        return launch_rows_t<float>(ctx, bl, nrows, rows, rowptr, col, (const float *)vals, x, y, mode, variant);
    return launch_rows_t<double>(ctx, bl, nrows, rows, rowptr, col, (const double *)vals, x, y, mode, variant);
}

// ---------------------------------------------------------------------------
// Autotuner keyed on block size and precision: the first full matvec of a
// tunable block size times each threads-per-row variant on the caller's
// matrix (CUDA events, two warm-up and three timed launches each) and keeps
// the fastest for the rest of the process.  CPG_AUTOTUNE=0 disables it
// (variant 0).
// ---------------------------------------------------------------------------
std::mutex g_tune_mu;
int g_tune[2][64];  // [precision][block size] -> variant + 1 (0 = untuned)

bool tunable(int bl) { return bl == 6 || bl == 10 || bl == 24 || bl == 40 || bl == 48; }

int tuned_variant(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rowptr, const int *col,
                  const void *vals, const double *x, double *y) {
    if (!tunable(bl)) return 0;
    // held for the whole tuning: concurrent first calls (serving threads)
    // wait and then read the one decision, so every solve of the process
    // uses the same variant and sums in the same order
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune[precision][bl]) return g_tune[precision][bl] - 1;
    const char *env = std::getenv("CPG_AUTOTUNE");
    if ((env && std::strcmp(env, "0") == 0) || nrows < 2048) return 0;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return 0;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return 0;
    }
    int best = 0;
    float best_ms = 1e30f;
    for (int v = 0; v < 3; v++) {
        bool ok = true;
        for (int r = 0; r < 2 && ok; r++)
            ok = launch_rows_v(ctx, precision, bl, nrows, nullptr, rowptr, col, vals, x, y, MODE_MATVEC, v) == CPG_OK;
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 3 && ok; r++)
            ok = launch_rows_v(ctx, precision, bl, nrows, nullptr, rowptr, col, vals, x, y, MODE_MATVEC, v) == CPG_OK;
        cudaEventRecord(e1, ctx->stream);
        float ms = 1e30f;
        if (ok && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        if (ok && ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g_tune[precision][bl] = best + 1;
    return best;
}

cpg_status launch_rows(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                       const int *col, const void *vals, const double *x, double *y, int mode) {
    int variant = 2;  // level sweeps: widest rows
    if (mode == MODE_MATVEC && rows == nullptr)
        variant = tuned_variant(ctx, precision, bl, nrows, rowptr, col, vals, x, y);
    return launch_rows_v(ctx, precision, bl, nrows, rows, rowptr, col, vals, x, y, mode, variant);
}

}  // namespace

namespace cpg {
cpg_status rows_op(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                   const int *col, const void *vals, const double *x, double *y, int mode) {
    return launch_rows(ctx, precision, bl, nrows, rows, rowptr, col, vals, x, y, mode);
}
cpg_status sweep_op(cpg_ctx *ctx, int precision, int bl, int nrows, const int *order, const int *rowptr,
                    const int *col, const void *vals, double *x, int mode, int *flags, int gen, int *counter,
                    int *err) {
    if (precision == CPG_F32)
        return launch_sweep_t<float>(ctx, bl, nrows, order, rowptr, col, (const float *)vals, x, mode, flags, gen,
                                     counter, err);
    return launch_sweep_t<double>(ctx, bl, nrows, order, rowptr, col, (const double *)vals, x, mode, flags, gen,
                                  counter, err);
}
bool sweep_supported(int bl) { return bl == 6 || bl == 10 || bl == 24 || bl == 40; }
cpg_status bsr_matvec_raw(cpg_ctx *ctx, const cpg_bsr *A, const double *x, double *y) {
    return launch_rows(ctx, A->precision, A->bl, A->n_rows, nullptr, A->rowptr_d, A->colidx_d, A->vals, x, y,
                       MODE_MATVEC);
}
}  // namespace cpg

static void free_bsr(cpg_bsr *A) {
    if (A->owns_pattern) {
        dfree(A->rowptr_d);
        dfree(A->colidx_d);
    }
    dfree(A->vals);
}

static cpg_status bsr_alloc(cpg_ctx *ctx, cpg_bsr *A) {
    CPG_TRY(upload(ctx, &A->rowptr_d, A->rowptr));
    CPG_TRY(upload(ctx, &A->colidx_d, A->colidx));
    const size_t bytes = (size_t)A->nnzb * A->bl * A->bl * A->elem();
    cudaError_t e = cudaMalloc(&A->vals, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        A->vals = nullptr;
        return fail(ctx, CPG_ERR_OOM, "BSR values: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    CPG_CUDA(ctx, cudaMemsetAsync(A->vals, 0, bytes, ctx->stream));
    return CPG_OK;
}

template <class T>
__global__ void k_convert(int64_t n, const double *__restrict__ src, T *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (T)src[i];
}
template <class T>
__global__ void k_widen(int64_t n, const T *__restrict__ src, double *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = (double)src[i];
}

extern "C" {

cpg_status cpg_bsr_create(cpg_ctx *ctx, const cpg_equation *eq, int precision, cpg_bsr **out) {
    if (!ctx || !eq || !out || (precision != CPG_F64 && precision != CPG_F32)) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    cpg_bsr *A = new (std::nothrow) cpg_bsr();
    if (!A) return fail(ctx, CPG_ERR_OOM, "host allocation");
    A->ctx = ctx;
    A->n_rows = eq->n;
    A->bl = eq->bl;
    A->precision = precision;
    A->rowptr = eq->rowptr;
    A->colidx = eq->colidx;
    A->nnzb = (int64_t)eq->colidx.size();
    cpg_status s = bsr_alloc(ctx, A);
    if (s != CPG_OK) {
        free_bsr(A);
        delete A;
        return s;
    }
    *out = A;
    return CPG_OK;
}

cpg_status cpg_bsr_create_host(cpg_ctx *ctx, int n_rows, int bl, const int *rowptr, const int *colidx,
                               const double *values_host, int precision, cpg_bsr **out) {
    if (!ctx || !rowptr || !colidx || !out || n_rows <= 0 || bl <= 0 ||
        (precision != CPG_F64 && precision != CPG_F32))
        return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    for (int i = 0; i < n_rows; i++) {
        if (rowptr[i + 1] < rowptr[i]) return fail(ctx, CPG_ERR_INVALID_ARG, "rowptr must be non-decreasing");
        for (int k = rowptr[i]; k < rowptr[i + 1]; k++)
            if (colidx[k] < 0 || colidx[k] >= n_rows) return fail(ctx, CPG_ERR_INVALID_ARG, "column out of range");
    }
    if (rowptr[0] != 0) return fail(ctx, CPG_ERR_INVALID_ARG, "rowptr[0] must be 0");
    cpg_bsr *A = new (std::nothrow) cpg_bsr();
    if (!A) return fail(ctx, CPG_ERR_OOM, "host allocation");
    A->ctx = ctx;
    A->n_rows = n_rows;
    A->bl = bl;
    A->precision = precision;
    A->rowptr.assign(rowptr, rowptr + n_rows + 1);
    A->colidx.assign(colidx, colidx + rowptr[n_rows]);
    A->nnzb = rowptr[n_rows];
    cpg_status s = bsr_alloc(ctx, A);
    if (s == CPG_OK && values_host) s = cpg_bsr_upload(ctx, A, values_host);
    if (s != CPG_OK) {
        free_bsr(A);
        delete A;
        return s;
    }
    *out = A;
    return CPG_OK;
}

void cpg_bsr_destroy(cpg_bsr *A) {
    if (!A) return;
    // cudaFree synchronizes the device; the context may already be gone
    free_bsr(A);
    delete A;
}

cpg_status cpg_bsr_get_info(const cpg_bsr *A, int *n_rows, int *bl, int64_t *nnzb, int *precision) {
    if (!A) return CPG_ERR_INVALID_ARG;
    if (n_rows) *n_rows = A->n_rows;
    if (bl) *bl = A->bl;
    if (nnzb) *nnzb = A->nnzb;
    if (precision) *precision = A->precision;
    return CPG_OK;
}

cpg_status cpg_bsr_upload(cpg_ctx *ctx, cpg_bsr *A, const double *values_host) {
    if (!ctx || !A || !values_host) return CPG_ERR_INVALID_ARG;
    const int64_t n = A->nnzb * A->bl * A->bl;
    if (n == 0) return CPG_OK;
    if (A->precision == CPG_F64) {
        CPG_CUDA(ctx, cudaMemcpyAsync(A->vals, values_host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    } else {
        double *tmp;
        CPG_TRY(dmalloc(ctx, &tmp, (size_t)n));
        CPG_CUDA(ctx, cudaMemcpyAsync(tmp, values_host, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        k_convert<float><<<1024, 256, 0, ctx->stream>>>(n, tmp, (float *)A->vals);
        CPG_TRY(launched(ctx, "convert kernel"));
        CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        cudaFree(tmp);
    }
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CPG_OK;
}

cpg_status cpg_bsr_export(cpg_ctx *ctx, const cpg_bsr *A, int *rowptr, int *colidx, double *values_host) {
    if (!ctx || !A) return CPG_ERR_INVALID_ARG;
    if (rowptr) std::memcpy(rowptr, A->rowptr.data(), sizeof(int) * A->rowptr.size());
    if (colidx) std::memcpy(colidx, A->colidx.data(), sizeof(int) * A->colidx.size());
    if (values_host) {
        const int64_t n = A->nnzb * A->bl * A->bl;
        if (n == 0) return CPG_OK;
        if (A->precision == CPG_F64) {
            CPG_CUDA(ctx, cudaMemcpyAsync(values_host, A->vals, n * sizeof(double), cudaMemcpyDeviceToHost,
                                          ctx->stream));
        } else {
            double *tmp;
            CPG_TRY(dmalloc(ctx, &tmp, (size_t)n));
            k_widen<float><<<1024, 256, 0, ctx->stream>>>(n, (const float *)A->vals, tmp);
            CPG_TRY(launched(ctx, "widen kernel"));
            CPG_CUDA(ctx, cudaMemcpyAsync(values_host, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(tmp);
        }
        CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    }
    return CPG_OK;
}

cpg_status cpg_bsr_matvec(cpg_ctx *ctx, const cpg_bsr *A, const double *x, double *y) {
    if (!ctx || !A || !x || !y) return CPG_ERR_INVALID_ARG;
    if (x == y) return fail(ctx, CPG_ERR_INVALID_ARG, "matvec is out of place: x and y must differ");
    return bsr_matvec_raw(ctx, A, x, y);
}

}  // extern "C"
