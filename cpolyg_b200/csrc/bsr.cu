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
// Triangular sweeps either run sync-free, one launch per sweep (k_sweep_direct
// with rows streamed straight into registers, or k_sweep with a TMA ring), or
// one launch per level of the level schedule computed from the block pattern.
#include <algorithm>
#include <atomic>
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

// the same vector loads from shared memory (plain loads: the streaming
// cache hints above are global-memory instructions)
template <class T, int VEC>
struct SmemLoad;
template <>
struct SmemLoad<double, 2> {
    static __device__ __forceinline__ void ld(const double *p, double *v) {
        const double2 a = *reinterpret_cast<const double2 *>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
};
template <>
struct SmemLoad<float, 2> {
    static __device__ __forceinline__ void ld(const float *p, double *v) {
        const float2 a = *reinterpret_cast<const float2 *>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
};
template <>
struct SmemLoad<float, 4> {
    static __device__ __forceinline__ void ld(const float *p, double *v) {
        const float4 a = *reinterpret_cast<const float4 *>(p);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
};

constexpr int MAX_ROW_BLOCKS = 64;

constexpr int PREFETCH_ROWS = 50000;  // below this many rows a launch is latency-bound

// Bulk prefetch of a row's blocks into L2 (cp.async.bulk.prefetch.L2, no
// multicast), one block per lane of the calling warp: issued as soon as the
// row is known, so that the streaming loads that follow hit L2.  Only for
// block sizes whose blocks are whole multiples of 16 bytes (the bulk copy's
// granule); the row starts 16-byte aligned then too.
template <class T, int BL>
__device__ __forceinline__ void prefetch_row_l2(const T *vals, int k0, int nblk, int lane) {
    constexpr unsigned B = BL * BL * sizeof(T);
    if constexpr (B % 16 == 0) {
        for (int b = lane; b < nblk; b += 32)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(vals + (size_t)(k0 + b) * BL * BL),
                         "r"(B)
                         : "memory");
    }
}

template <class T, int BL, int VEC, int TPR>
__global__ void __launch_bounds__(TPR) k_rows(const int *__restrict__ rows, const int *__restrict__ rowptr,
                                              const int *__restrict__ col, const T *__restrict__ vals,
                                              const double *x, double *y, int mode, const int *skip,
                                              int prefetch, const double *addv) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    static_assert((TPR * VEC) % BL == 0, "stride must be a multiple of the block size");
    static_assert(BL % VEC == 0, "vector width must divide the block size");
    constexpr int S = TPR * VEC, G = S / BL, BL2 = BL * BL;
    __shared__ int scol[MAX_ROW_BLOCKS];
    __shared__ double red[G][BL];
    const int i = rows ? rows[blockIdx.x] : blockIdx.x;
    const int k0 = rowptr[i], nblk = rowptr[i + 1] - k0;
    const int tid = threadIdx.x;
    if (prefetch && tid < 32) prefetch_row_l2<T, BL>(vals, k0, nblk, tid);
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
        else if (addv) s = s + __ldg(addv + (size_t)i * BL + tid);
        yi[tid] = s;
    }
}

// generic block size: scalar loads, TPR = block size * groups
template <class T>
__global__ void __launch_bounds__(256) k_rows_dyn(int BL, int G, const int *__restrict__ rows,
                                                  const int *__restrict__ rowptr, const int *__restrict__ col,
                                                  const T *__restrict__ vals, const double *x, double *y, int mode,
                                                  const int *skip, const double *addv) {
    if (skip && *skip) return;
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
        else if (addv) s = s + __ldg(addv + (size_t)i * BL + tid);
        yi[tid] = s;
    }
}

// ---------------------------------------------------------------------------
// Sync-free triangular sweep: one launch for a whole forward or backward
// ILU(0) sweep, warp specialised around a TMA bulk-copy ring.
//
// Several CTAs per SM.  In each, a producer warp claims rows in level order
// from a global counter (a few at a time) and copies each row's contiguous
// value array, in chunks of BPC blocks, from HBM into a ring of R shared-
// memory stages with cp.async.bulk; an mbarrier per stage signals "full"
// when the bytes have landed and one per stage collects the consumer warps'
// "empty" arrivals.  The consumer warps take the stages in order.  At a
// row's first chunk they wait, one warp per block, until every row it reads
// has published its value (flags[j] == gen), and stage those x segments in
// shared memory; then every consumer thread streams its elements of each
// chunk exactly as k_rows does (same threads per row, same element
// sequence, same group reduction), so the result is bitwise that of the
// level form.  At the row's last chunk the groups are reduced, x_i is
// written through L2 and the row's flag is released.  The producer runs up
// to R chunks ahead, so copies overlap the waits, reductions and publishes.
//
// Progress: every CTA takes its rows in claim order and a row only waits on
// rows claimed before it, by CTAs that are running, so the earliest
// unfinished row can always proceed.  Every wait is bounded; once any wait
// gives up it sets *err, later dependency waits stop waiting (the result is
// then garbage and the solve reports CPG_ERR_TIMEOUT), and the ring keeps
// draining so the kernel ends.  Consumers leave the loop together, through a
// barrier that ORs "my ring wait gave up / no more rows" over all of them;
// a producer whose ring wait gave up waits (bounded) for the copies it still
// has in flight before it returns.
// ---------------------------------------------------------------------------
constexpr long long SWEEP_MAX_SPINS = 1LL << 22;  // dependency polls (>= 64 ns apart): >= 0.27 s
constexpr long long RING_MAX_SPINS = 1LL << 24;   // mbarrier polls, a backstop only

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait for the phase of parity `parity` (>= 1 s before it gives up,
// longer than a dependency wait can last); false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err) {
    long long spins = 0;
    while (!mbar_test(bar, parity)) {
        if (++spins > RING_MAX_SPINS) {
            atomicExch(err, 2);
            return false;
        }
        if (spins > 1024) __nanosleep(64);
    }
    return true;
}
// HBM -> shared bulk copy completing on an mbarrier (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ int lane_of(int tid) { return tid & 31; }
// Named barrier 1 over the first nthreads threads (whole warps).  The
// non-aligned form: callers reach it right after divergent code (one thread
// per element of a row), and the aligned form (bar.sync) requires every warp
// to arrive converged, which the compiler does not arrange for inline PTX.
__device__ __forceinline__ void consumers_sync(int nthreads) {
    asm volatile("barrier.sync 1, %0;" ::"r"(nthreads) : "memory");
}
// the same barrier, returning whether any participating thread passed pred != 0
__device__ __forceinline__ int consumers_sync_or(int nthreads, int pred) {
    int r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.s32 p, %1, 0;\n barrier.red.or.pred q, 1, %2, p;\n selp.s32 %0, 1, 0, q;\n}"
        : "=r"(r)
        : "r"(pred), "r"(nthreads)
        : "memory");
    return r;
}

// Per-(block size, precision) shape of the sweep: consumer threads CT and
// vector width VEC match the level form's threads per row (k_rows variant
// 0), and a chunk of BPC blocks is a whole number of passes of CT * VEC
// elements, so every thread sees the same element sequence as in k_rows.
// Shared memory stays near 40-50 KB so four or more CTAs share an SM.
constexpr int SWEEP_MAXB = SWEEP_MAX_ROW_BLOCKS;  // blocks per row the sync-free form accepts
template <class T, int BL>
struct SweepShape;
template <class T> struct SweepShape<T, 6> { static constexpr int VEC = 2, CT = 96, BPC = 16, R = 6; };
template <class T> struct SweepShape<T, 10> { static constexpr int VEC = 2, CT = 160, BPC = 16, R = sizeof(T) == 8 ? 3 : 6; };
template <> struct SweepShape<double, 24> { static constexpr int VEC = 2, CT = 192, BPC = 2, R = 4; };
template <> struct SweepShape<float, 24> { static constexpr int VEC = 4, CT = 96, BPC = 2, R = 6; };
template <> struct SweepShape<double, 40> { static constexpr int VEC = 2, CT = 160, BPC = 1, R = 3; };
template <> struct SweepShape<float, 40> { static constexpr int VEC = 4, CT = 160, BPC = 2, R = 3; };

struct ChunkMeta {
    int row;   // cell row, or -1: no more rows
    int blk0;  // index of the chunk's first block within the row (0: first chunk)
    int nb;    // blocks in the chunk
    int last;  // 1 on the row's last chunk
    int nblk;  // blocks in the row
    int cols[SWEEP_MAXB];  // the row's block columns (first chunk only)
};

template <class T, int BL>
struct SweepSmem {
    using Sh = SweepShape<T, BL>;
    static constexpr int BL2 = BL * BL, G = Sh::CT * Sh::VEC / BL;
    static constexpr size_t STAGE = (size_t)Sh::BPC * BL2 * sizeof(T);
    static constexpr size_t RING = STAGE * Sh::R;
    static constexpr size_t BARS = RING;  // full[R], empty[R]
    static constexpr size_t META = BARS + 16 * (size_t)Sh::R;
    static constexpr size_t XS = (META + sizeof(ChunkMeta) * Sh::R + 15) / 16 * 16;  // the row's x segments
    static constexpr size_t RED = XS + sizeof(double) * SWEEP_MAXB * BL;
    static constexpr size_t BYTES = RED + sizeof(double) * G * BL;
    static_assert(STAGE % 16 == 0, "bulk copies move multiples of 16 bytes");
    static_assert((Sh::CT * Sh::VEC) % BL == 0, "stride must be a multiple of the block size");
    static_assert(((size_t)Sh::BPC * BL2) % (Sh::CT * Sh::VEC) == 0, "a chunk is a whole number of passes");
    static_assert(BYTES <= 60 * 1024, "several CTAs per SM");
};

template <class T, int BL>
__global__ void __launch_bounds__(SweepShape<T, BL>::CT + 32)
    k_sweep(const int *__restrict__ order, int n, const int *__restrict__ rowptr, const int *__restrict__ col,
            const T *__restrict__ vals, double *x, int mode, int *flags, int gen, int *counter, int *err, const int *skip,
            const double *addv) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    using Sh = SweepShape<T, BL>;
    using L = SweepSmem<T, BL>;
    constexpr int CT = Sh::CT, VEC = Sh::VEC, BPC = Sh::BPC, R = Sh::R;
    constexpr int S = CT * VEC, G = S / BL, BL2 = BL * BL, NCW = CT / 32;
    extern __shared__ __align__(128) unsigned char sm[];
    T *ring = (T *)sm;
    uint64_t *full = (uint64_t *)(sm + L::BARS), *empty = full + R;
    ChunkMeta *meta = (ChunkMeta *)(sm + L::META);
    double(*xs)[BL] = (double(*)[BL])(sm + L::XS);
    double(*red)[BL] = (double(*)[BL])(sm + L::RED);
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int r = 0; r < R; r++) {
            mbar_init(full + r, 1);
            mbar_init(empty + r, NCW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (tid >= CT) {  // ---------------- producer warp ----------------
        // Rows are claimed CLAIM at a time; lane k < CLAIM fetches row k's
        // metadata, the lanes copy the row's block columns, lane 0 issues
        // the mbarrier operations and the copies.  The next claim's atomic
        // is in flight while the current batch is issued.
        constexpr int CLAIM = 4;
        const unsigned FULL = 0xffffffffu;
        const int lane = lane_of(tid);
        int stage = 0;
        uint32_t phase = 0;
        int pending[R];  // lane 0: parity of the fill in flight per stage, -1 none
#pragma unroll
        for (int r = 0; r < R; r++) pending[r] = -1;
        bool ok = true, done = false;
        int qn = (lane == 0) ? atomicAdd(counter, CLAIM) : 0;
        while (!done && ok) {
            const int q0 = __shfl_sync(FULL, qn, 0);
            if (lane == 0 && q0 < n) qn = atomicAdd(counter, CLAIM);
            int my_i = -1, my_k0 = 0, my_nb = 0;
            if (lane < CLAIM && q0 + lane < n) {
                my_i = order[q0 + lane];
                my_k0 = rowptr[my_i];
                my_nb = rowptr[my_i + 1] - my_k0;
            }
            for (int k = 0; k < CLAIM && ok && !done; k++) {
                const int i = __shfl_sync(FULL, my_i, k);
                const int k0 = __shfl_sync(FULL, my_k0, k), nblk_raw = __shfl_sync(FULL, my_nb, k);
                // the host admits no longer rows; a longer one is reported, not read
                const int nblk = nblk_raw > SWEEP_MAXB ? 0 : nblk_raw;
                if (lane == 0 && nblk_raw > SWEEP_MAXB) atomicExch(err, 3);
                done = i < 0;  // past the last row: this chunk is the stop marker
                int c0 = 0;
                do {  // a row without blocks still sends one (empty) chunk to publish its flag
                    const int w = lane == 0 ? (int)mbar_wait(empty + stage, phase ^ 1, err) : 0;
                    if (!(ok = __shfl_sync(FULL, w, 0) != 0)) break;
                    ChunkMeta &m = meta[stage];
                    const int nb = done ? 0 : min(BPC, nblk - c0);
                    if (c0 == 0)
                        for (int b = lane; b < nblk; b += 32) m.cols[b] = col[k0 + b];
                    __syncwarp();
                    if (lane == 0) {
                        m.row = i;
                        m.blk0 = c0;
                        m.nb = nb;
                        m.nblk = done ? 0 : nblk;
                        m.last = (c0 + nb >= nblk) ? 1 : 0;
                        if (nb > 0) {
                            const uint32_t bytes = (uint32_t)(nb * BL2 * sizeof(T));
                            mbar_arrive_tx(full + stage, bytes);
                            bulk_load(ring + (size_t)stage * BPC * BL2, vals + (size_t)(k0 + c0) * BL2, bytes,
                                      full + stage);
                        } else {
                            mbar_arrive(full + stage);
                        }
                        pending[stage] = (int)phase;
                    }
                    __syncwarp();
                    c0 += BPC;
                    if (++stage == R) {
                        stage = 0;
                        phase ^= 1;
                    }
                } while (c0 < nblk);
            }
        }
        if (!ok && lane == 0)  // consumers left early: let the copies in flight land before the CTA ends
            for (int r = 0; r < R; r++)
                if (pending[r] >= 0) mbar_wait(full + r, (uint32_t)pending[r], err);
        return;
    }

    // ---------------- consumer warps ----------------
    const int warp = tid >> 5, lane = tid & 31;
    const int e0 = tid * VEC;
    const int r0 = e0 % BL, g = e0 / BL;
    const double s0 = (mode == MODE_FORWARD) ? -1.0 : 1.0;
    const double sr = -1.0;
    const int first_dep = (mode == MODE_BACKWARD) ? 1 : 0;  // the backward row's block 0 is D^{-1}_i
    double acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) acc[v] = 0.0;
    int stage = 0;
    uint32_t phase = 0;
    for (;;) {
        // a thread whose ring wait gave up touches nothing of the stage; this
        // barrier takes every consumer out together on that or on the stop marker
        const bool landed = mbar_wait(full + stage, phase, err);
        const int i = landed ? meta[stage].row : -1;
        if (consumers_sync_or(CT, i < 0)) break;
        const ChunkMeta &m = meta[stage];
        const int blk0 = m.blk0, nb = m.nb, last = m.last;
        if (blk0 == 0) {
            // the row's dependencies and x segments, block b by warp b % NCW
            const int nblk = m.nblk;
            for (int b = warp; b < nblk; b += NCW) {
                const int j = m.cols[b];
                if (lane == 0 && b >= first_dep) {
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
                __syncwarp();
                // values published during this sweep: read through L2, not L1
                for (int c = lane; c < BL; c += 32) xs[b][c] = __ldcg(x + (size_t)j * BL + c);
            }
            consumers_sync(CT);
        }
        const T *base = ring + (size_t)stage * BPC * BL2;
        const int E = nb * BL2;
        int blk = e0 / BL2, within = e0 % BL2;
#pragma unroll 4
        for (int e = e0; e < E; e += S) {
            const int c = within / BL;
            double a[VEC];
            SmemLoad<T, VEC>::ld(base + e, a);
            const int gb = blk0 + blk;  // block index within the row
            const double xv = xs[gb][c] * (gb == 0 ? s0 : sr);
#pragma unroll
            for (int v = 0; v < VEC; v++) acc[v] += a[v] * xv;
            within += S;
            while (within >= BL2) {
                within -= BL2;
                blk++;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + stage);  // this warp is done with the stage
        if (++stage == R) {
            stage = 0;
            phase ^= 1;
        }
        if (last) {
#pragma unroll
            for (int v = 0; v < VEC; v++) {
                red[g][r0 + v] = acc[v];
                acc[v] = 0.0;
            }
            consumers_sync(CT);
            if (tid < BL) {
                double s = 0.0;
#pragma unroll
                for (int qq = 0; qq < G; qq++) s += red[qq][tid];
                double *xi = x + (size_t)i * BL;
                if (mode == MODE_FORWARD) s = __ldcg(xi + tid) + s;
                else if (addv) s = s + __ldg(addv + (size_t)i * BL + tid);
                __stcg(xi + tid, s);
            }
            consumers_sync(CT);  // also: nobody stages the next row's xs before this row is done
            if (tid == 0) {
                __threadfence();
                st_release(flags + i, gen);
            }
        }
    }
}

template <class T, int BL>
cpg_status launch_sweep_cfg(cpg_ctx *ctx, int nrows, const int *order, const int *rowptr, const int *col,
                            const T *vals, double *x, int mode, int *flags, int gen, int *counter, int *err,
                            const double *addv) {
    using L = SweepSmem<T, BL>;
    constexpr int threads = SweepShape<T, BL>::CT + 32;
    static std::atomic<int> per_sm[64];  // occupancy per device, computed once
    CPG_TRY(smem_limit_once(ctx, (const void *)k_sweep<T, BL>, (int)L::BYTES));
    const bool cacheable = ctx->device >= 0 && ctx->device < 64;
    int occ = cacheable ? per_sm[ctx->device].load() : 0;
    if (!occ) {
        CPG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sweep<T, BL>, threads, L::BYTES));
        if (cacheable) per_sm[ctx->device].store(occ);
    }
    const int grid = std::max(1, std::min(nrows, std::max(1, occ) * ctx->num_sms));
    CPG_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
    k_sweep<T, BL><<<grid, threads, L::BYTES, ctx->stream>>>(order, nrows, rowptr, col, vals, x, mode, flags, gen,
                                                            counter, err, ctx->skip_dev, addv);
    return launched(ctx, "sync-free sweep kernel");
}

// ---------------------------------------------------------------------------
// The same sweep without the ring: CTAs of the level form's size (k_rows
// variant 0) stream their row's values straight from HBM into registers, as
// k_rows does, and many of them share an SM.  A CTA claims its next row
// while the current one streams, waits (one thread per block) for the rows
// it reads, and publishes like k_sweep.  Same threads per row and element
// order as the level form, so the same bits; same progress argument and the
// same bounded waits.
// ---------------------------------------------------------------------------
// fill the SM with rows in flight: registers capped so that 1,920 threads
// (12 CTAs of 160) fit, as rows are latency bound
template <class T, int BL, int TPR>
__global__ void __launch_bounds__(TPR, (1920 / TPR > 0 ? 1920 / TPR : 1))
    k_sweep_direct(const int *__restrict__ order, int n, const int *__restrict__ rowptr,
                   const int *__restrict__ col, const T *__restrict__ vals, double *x, int mode, int *flags,
                   int gen, int *counter, int *err, const int *skip, int prefetch, const double *addv) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    constexpr int VEC = SweepShape<T, BL>::VEC;
    constexpr int S = TPR * VEC, G = S / BL, BL2 = BL * BL;
    constexpr int CLAIMER = TPR > 32 ? 32 : 0;  // warp 0 holds the dependency waits
    __shared__ int s_row[2];
    __shared__ int scol[SWEEP_MAXB];
    __shared__ double red[G][BL];
    const int tid = threadIdx.x;
    const int e0 = tid * VEC;
    const int r0 = e0 % BL, g = e0 / BL;
    const double s0 = (mode == MODE_FORWARD) ? -1.0 : 1.0;
    const double sr = -1.0;
    const int first_dep = (mode == MODE_BACKWARD) ? 1 : 0;  // the backward row's block 0 is D^{-1}_i
    if (tid == CLAIMER) s_row[0] = atomicAdd(counter, 1);
    __syncthreads();
    for (int cur = 0;; cur ^= 1) {
        const int q = s_row[cur];
        if (q >= n) break;
        // the next claim stays in flight while this row streams: its result
        // is stored to shared memory only after the streaming loop
        const int next = tid == CLAIMER ? atomicAdd(counter, 1) : 0;
        const int i = order[q];
        const int k0 = rowptr[i], nraw = rowptr[i + 1] - k0;
        const int nblk = nraw > SWEEP_MAXB ? 0 : nraw;  // the host admits no longer rows
        if (tid == 0 && nraw > SWEEP_MAXB) atomicExch(err, 3);
        // the row's values do not depend on the rows it waits for: on a
        // latency-bound sweep (few rows) they are fetched into L2 meanwhile
        if (prefetch && tid >= TPR - 32) prefetch_row_l2<T, BL>(vals, k0, nblk, tid - (TPR - 32));
        for (int b = tid; b < nblk; b += TPR) {
            const int j = col[k0 + b];
            scol[b] = j;
            if (b >= first_dep) {
                long long spins = 0;
                while (ld_acquire(flags + j) != gen) {
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
            // values published during this sweep: read through L2, not L1
            const double xv = __ldcg(x + (size_t)scol[blk] * BL + c) * (blk == 0 ? s0 : sr);
#pragma unroll
            for (int v = 0; v < VEC; v++) acc[v] += a[v] * xv;
            within += S;
            while (within >= BL2) {
                within -= BL2;
                blk++;
            }
        }
        if (tid == CLAIMER) s_row[cur ^ 1] = next;
#pragma unroll
        for (int v = 0; v < VEC; v++) red[g][r0 + v] = acc[v];
        __syncthreads();
        if (tid < BL) {
            double sum = 0.0;
#pragma unroll
            for (int qq = 0; qq < G; qq++) sum += red[qq][tid];
            double *xi = x + (size_t)i * BL;
            if (mode == MODE_FORWARD) sum = __ldcg(xi + tid) + sum;
            else if (addv) sum = sum + __ldg(addv + (size_t)i * BL + tid);
            __stcg(xi + tid, sum);
        }
        __syncthreads();  // the row's stores and the next claim are done
        if (tid == 0) {
            __threadfence();
            st_release(flags + i, gen);
        }
    }
}

template <class T, int BL, int TPR>
cpg_status launch_sweep_direct_cfg(cpg_ctx *ctx, int nrows, const int *order, const int *rowptr, const int *col,
                                   const T *vals, double *x, int mode, int *flags, int gen, int *counter,
                                   int *err, const double *addv) {
    static std::atomic<int> per_sm[64];  // occupancy per device, computed once
    const bool cacheable = ctx->device >= 0 && ctx->device < 64;
    int occ = cacheable ? per_sm[ctx->device].load() : 0;
    if (!occ) {
        CPG_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_sweep_direct<T, BL, TPR>, TPR, 0));
        if (cacheable) per_sm[ctx->device].store(occ);
    }
    const int grid = std::max(1, std::min(nrows, std::max(1, occ) * ctx->num_sms));
    CPG_CUDA(ctx, cudaMemsetAsync(counter, 0, sizeof(int), ctx->stream));
    k_sweep_direct<T, BL, TPR><<<grid, TPR, 0, ctx->stream>>>(order, nrows, rowptr, col, vals, x, mode, flags,
                                                             gen, counter, err, ctx->skip_dev,
                                                             nrows < PREFETCH_ROWS ? 1 : 0, addv);
    return launched(ctx, "sync-free sweep kernel (direct)");
}

// kind 0: TMA ring; kinds 1, 2, 3: direct loads with 1, 2 or 4 times the
// consumer threads per row (the level form's variants 0, 1, 2)
template <class T>
cpg_status launch_sweep_t(cpg_ctx *ctx, int bl, int nrows, const int *order, const int *rowptr, const int *col,
                          const T *vals, double *x, int mode, int *flags, int gen, int *counter, int *err,
                          int kind, const double *addv) {
    if (nrows <= 0) return CPG_OK;
#define CPG_SWEEP(BLV)                                                                                          \
    {                                                                                                           \
        constexpr int CT = SweepShape<T, BLV>::CT;                                                              \
        switch (kind) {                                                                                         \
            case 1:                                                                                             \
                return launch_sweep_direct_cfg<T, BLV, CT>(ctx, nrows, order, rowptr, col, vals, x, mode, flags, \
                                                           gen, counter, err, addv);                            \
            case 2:                                                                                             \
                return launch_sweep_direct_cfg<T, BLV, 2 * CT>(ctx, nrows, order, rowptr, col, vals, x, mode,    \
                                                               flags, gen, counter, err, addv);                 \
            case 3:                                                                                             \
                return launch_sweep_direct_cfg<T, BLV, 4 * CT>(ctx, nrows, order, rowptr, col, vals, x, mode,    \
                                                               flags, gen, counter, err, addv);                 \
            default:                                                                                            \
                return launch_sweep_cfg<T, BLV>(ctx, nrows, order, rowptr, col, vals, x, mode, flags, gen,       \
                                                counter, err, addv);                                            \
        }                                                                                                       \
    }
    switch (bl) {
        case 6: CPG_SWEEP(6);
        case 10: CPG_SWEEP(10);
        case 24: CPG_SWEEP(24);
        case 40: CPG_SWEEP(40);
        default: return CPG_ERR_UNSUPPORTED;
    }
#undef CPG_SWEEP
}

// ---------------------------------------------------------------------------
// Rows of the split form of P^{-1} A for an ILU(0) P (precond.cu): with
// A = (I + L) D + D U' + E, the product needs y = (U_A + E) x only, where
// y_i = E_i x_i + sum_{j > i} A_ij x_j.  The columns are those of the DU
// row (its first block is the row's own); E_i stands in for the D^{-1} slot
// and the other blocks are read from A at the positions u2a.  Threads per
// row and element order as k_rows.
// ---------------------------------------------------------------------------
template <int BL, int VEC, int TPR>
__global__ void __launch_bounds__(TPR) k_rows_split(const int *__restrict__ rowptr, const int *__restrict__ col,
                                                    const int *__restrict__ u2a, const double *__restrict__ vals,
                                                    const double *__restrict__ Eb, const double *x, double *y,
                                                    const int *skip, int prefetch) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    static_assert((TPR * VEC) % BL == 0, "stride must be a multiple of the block size");
    constexpr int S = TPR * VEC, G = S / BL, BL2 = BL * BL;
    constexpr unsigned BYTES = BL2 * sizeof(double);
    __shared__ int scol[SWEEP_MAXB];
    __shared__ const double *sptr[SWEEP_MAXB];
    __shared__ double red[G][BL];
    const int i = blockIdx.x;
    const int k0 = rowptr[i], nraw = rowptr[i + 1] - k0;
    const int nblk = nraw > SWEEP_MAXB ? SWEEP_MAXB : nraw;  // the host admits no longer rows
    const int tid = threadIdx.x;
    for (int q = tid; q < nblk; q += TPR) {
        const double *p = q == 0 ? Eb + (size_t)i * BL2 : vals + (size_t)u2a[k0 + q] * BL2;
        scol[q] = col[k0 + q];
        sptr[q] = p;
        if constexpr (BYTES % 16 == 0)
            if (prefetch)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(BYTES) : "memory");
    }
    __syncthreads();
    const int e0 = tid * VEC;
    const int r0 = e0 % BL, g = e0 / BL;
    double acc[VEC];
#pragma unroll
    for (int v = 0; v < VEC; v++) acc[v] = 0.0;
    const int E = nblk * BL2;
    int blk = e0 / BL2, within = e0 % BL2;
#pragma unroll 4
    for (int e = e0; e < E; e += S) {
        const int c = within / BL;
        double a[VEC];
        VecLoad<double, VEC>::ld(sptr[blk] + within, a);
        const double xv = __ldg(x + (size_t)scol[blk] * BL + c);
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
        y[(size_t)i * BL + tid] = s;
    }
}

cpg_status launch_split_v(cpg_ctx *ctx, int bl, int nrows, const int *rowptr, const int *col, const int *u2a,
                          const double *vals, const double *E, const double *x, double *y, int variant) {
    cudaStream_t s = ctx->stream;
    const int pf = nrows < PREFETCH_ROWS ? 1 : 0;
#define CPG_SPLIT3(BLV, T0, T1, T2)                                                                               \
    switch (variant) {                                                                                            \
        case 0: k_rows_split<BLV, 2, T0><<<nrows, T0, 0, s>>>(rowptr, col, u2a, vals, E, x, y, ctx->skip_dev, pf); break; \
        case 1: k_rows_split<BLV, 2, T1><<<nrows, T1, 0, s>>>(rowptr, col, u2a, vals, E, x, y, ctx->skip_dev, pf); break; \
        default: k_rows_split<BLV, 2, T2><<<nrows, T2, 0, s>>>(rowptr, col, u2a, vals, E, x, y, ctx->skip_dev, pf); break; \
    }
    switch (bl) {
        case 6: CPG_SPLIT3(6, 96, 192, 384) break;
        case 10: CPG_SPLIT3(10, 160, 320, 640) break;
        case 24: CPG_SPLIT3(24, 192, 384, 576) break;
        case 40: CPG_SPLIT3(40, 160, 320, 640) break;
        default: return fail(ctx, CPG_ERR_UNSUPPORTED, "block size of the split rows");
    }
#undef CPG_SPLIT3
    return launched(ctx, "split block-row kernel");
}

template <class T>
cpg_status launch_rows_t(cpg_ctx *ctx, int bl, int nrows, const int *rows, const int *rowptr, const int *col,
                         const T *vals, const double *x, double *y, int mode, int variant,
                         const double *addv) {
    if (nrows <= 0) return CPG_OK;
    cudaStream_t s = ctx->stream;
    constexpr bool F32 = std::is_same<T, float>::value;
    // L2 prefetch of each row where rows are latency-bound: FP32 values
    // (half the bytes per row for the same per-row work) and launches of few
    // rows; a full FP64 matvec streams at the copy bandwidth without it
    const int pf = (F32 || nrows < PREFETCH_ROWS) ? 1 : 0;
    // threads per row: variants 0/1/2 use about 8/16/32 column groups; the
    // matvec picks its variant by timing (autotune below), level sweeps take
    // the widest variant because they are latency bound
#define CPG_ROWS3(BLV, V, T0, T1, T2)                                                                    \
    switch (variant) {                                                                                   \
        case 0: k_rows<T, BLV, V, T0><<<nrows, T0, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break;  \
        case 1: k_rows<T, BLV, V, T1><<<nrows, T1, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break;  \
        default: k_rows<T, BLV, V, T2><<<nrows, T2, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break; \
    }
    switch (bl) {
        case 1: k_rows<T, 1, 1, 32><<<nrows, 32, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break;
        case 3: k_rows<T, 3, 1, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break;
        case 4: k_rows<T, 4, 2, 64><<<nrows, 64, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv); break;
        case 6: CPG_ROWS3(6, 2, 96, 192, 384) break;
        case 10: CPG_ROWS3(10, 2, 160, 320, 640) break;
        case 12:
            if constexpr (F32) k_rows<T, 12, 4, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv);
            else k_rows<T, 12, 2, 96><<<nrows, 96, 0, s>>>(rows, rowptr, col, vals, x, y, mode, ctx->skip_dev, pf, addv);
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
            k_rows_dyn<T><<<nrows, 256, sizeof(double) * bl * G, s>>>(bl, G, rows, rowptr, col, vals, x, y, mode,
                                                                     ctx->skip_dev, addv);
        }
    }
#undef CPG_ROWS3
    return launched(ctx, "block-row kernel");
}

cpg_status launch_rows_v(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                         const int *col, const void *vals, const double *x, double *y, int mode, int variant,
                         const double *addv = nullptr) {
    if (precision == CPG_F32)
        return launch_rows_t<float>(ctx, bl, nrows, rows, rowptr, col, (const float *)vals, x, y, mode, variant,
                                    addv);
    return launch_rows_t<double>(ctx, bl, nrows, rows, rowptr, col, (const double *)vals, x, y, mode, variant,
                                 addv);
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

// the split rows' own threads-per-row decision per block size, taken the
// same way on the first split product of the process
int g_tune_split[64];

int tuned_split_variant(cpg_ctx *ctx, int bl, int nrows, const int *rowptr, const int *col, const int *u2a,
                        const double *vals, const double *E, const double *x, double *y) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (g_tune_split[bl]) return g_tune_split[bl] - 1;
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
            ok = launch_split_v(ctx, bl, nrows, rowptr, col, u2a, vals, E, x, y, v) == CPG_OK;
        cudaEventRecord(e0, ctx->stream);
        for (int r = 0; r < 3 && ok; r++)
            ok = launch_split_v(ctx, bl, nrows, rowptr, col, u2a, vals, E, x, y, v) == CPG_OK;
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
    g_tune_split[bl] = best + 1;
    return best;
}

cpg_status launch_rows(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                       const int *col, const void *vals, const double *x, double *y, int mode) {
    // level sweeps: variant 0, the threads per row of the sync-free sweep's
    // consumers, so both forms sum in the same order
    int variant = 0;
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
cpg_status rows_op_v(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                     const int *col, const void *vals, const double *x, double *y, int mode, int variant,
                     const double *addv) {
    return launch_rows_v(ctx, precision, bl, nrows, rows, rowptr, col, vals, x, y, mode, variant, addv);
}
bool rows_tunable(int bl) { return tunable(bl); }
cpg_status sweep_op(cpg_ctx *ctx, int precision, int bl, int nrows, const int *order, const int *rowptr,
                    const int *col, const void *vals, double *x, int mode, int *flags, int gen, int *counter,
                    int *err, int kind, const double *addv) {
    if (precision == CPG_F32)
        return launch_sweep_t<float>(ctx, bl, nrows, order, rowptr, col, (const float *)vals, x, mode, flags, gen,
                                     counter, err, kind, addv);
    return launch_sweep_t<double>(ctx, bl, nrows, order, rowptr, col, (const double *)vals, x, mode, flags, gen,
                                  counter, err, kind, addv);
}
bool sweep_supported(int bl) { return bl == 6 || bl == 10 || bl == 24 || bl == 40; }
cpg_status bsr_matvec_raw(cpg_ctx *ctx, const cpg_bsr *A, const double *x, double *y) {
    return launch_rows(ctx, A->precision, A->bl, A->n_rows, nullptr, A->rowptr_d, A->colidx_d, A->vals, x, y,
                       MODE_MATVEC);
}
cpg_status split_rows_op(cpg_ctx *ctx, const cpg_bsr *A, const int *U_rowptr, const int *U_col, const int *u2a,
                         const double *E, const double *x, double *y) {
    if (A->precision != CPG_F64) return fail(ctx, CPG_ERR_UNSUPPORTED, "split rows need FP64 values");
    const int n = A->n_rows;
    if (n <= 0) return CPG_OK;
    const double *vals = (const double *)A->vals;
    const int v = tuned_split_variant(ctx, A->bl, n, U_rowptr, U_col, u2a, vals, E, x, y);
    return launch_split_v(ctx, A->bl, n, U_rowptr, U_col, u2a, vals, E, x, y, v);
}
// stamps come from one process-wide counter, so a matrix freed and another
// allocated at the same address never share one
std::atomic<uint64_t> g_bsr_version{0};
void bsr_touch(cpg_bsr *A) { A->version = ++g_bsr_version; }
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
    bsr_touch(A);
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
    bsr_touch(A);
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CPG_OK;
}

cpg_status cpg_bsr_stack(cpg_ctx *ctx, int k, const cpg_bsr *const *parts, cpg_bsr **out) {
    if (!ctx || k < 1 || !parts || !out) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    const int bl = parts[0]->bl, prec = parts[0]->precision;
    std::vector<int> rowptr(1, 0), col;
    int row0 = 0;
    for (int q = 0; q < k; q++) {
        const cpg_bsr *A = parts[q];
        if (!A || A->bl != bl || A->precision != prec)
            return fail(ctx, CPG_ERR_INVALID_ARG, "stacked matrices need one block size and precision");
        for (int i = 0; i < A->n_rows; i++) {
            for (int p = A->rowptr[i]; p < A->rowptr[i + 1]; p++) col.push_back(row0 + A->colidx[p]);
            rowptr.push_back((int)col.size());
        }
        row0 += A->n_rows;
    }
    cpg_bsr *S = nullptr;
    CPG_TRY(cpg_bsr_create_host(ctx, row0, bl, rowptr.data(), col.data(), nullptr, prec, &S));
    const size_t b2 = (size_t)bl * bl * S->elem();
    size_t at = 0;
    for (int q = 0; q < k; q++) {
        const size_t bytes = (size_t)parts[q]->nnzb * b2;
        const cudaError_t e = cudaMemcpyAsync((char *)S->vals + at, parts[q]->vals, bytes, cudaMemcpyDeviceToDevice,
                                              ctx->stream);
        if (e != cudaSuccess) {
            cpg_bsr_destroy(S);
            return cuda_fail(ctx, e, "stacking matrix values");
        }
        at += bytes;
    }
    bsr_touch(S);
    *out = S;
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
