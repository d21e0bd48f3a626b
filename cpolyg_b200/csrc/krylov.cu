// Krylov solvers and vector kernels: restarted GMRES with classical
// Gram-Schmidt (BlockMatrix::gmres, src/BlockMatrix.cpp:79-163), its flexible
// right-preconditioned variant (FGMRES), both also for a batch of independent
// systems, damped block Jacobi (BlockMatrix::jacobi, :51-77), and MeshFn
// arithmetic.
//
// The Krylov basis V lives on the device, column i at V + i*N.  One Arnoldi
// step is: matvec, preconditioner, h = V^T w (multi-dot), w -= V h fused with
// the partial sums of |w|^2, normalisation, and the Givens update of the
// least-squares problem, all on the device; the host reads the systems'
// state once per restart cycle.  Reductions use a fixed grid and a fixed
// combination order, so results are reproducible run to run.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.hpp"

using namespace cpg;

namespace {

constexpr int RED = 256;   // CTAs of a reduction (fixed for determinism)
constexpr int RT = 256;    // threads per reduction CTA

__device__ __forceinline__ double block_sum(double v, double *sh) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) s += sh[q];
    __syncthreads();
    return s;
}

// partial[l*RED + cta] = sum over this CTA's slice of V_l . w
__global__ void __launch_bounds__(RT) k_mdot(int64_t N, const double *__restrict__ V, const double *__restrict__ w,
                                             double *__restrict__ part) {
    __shared__ double sh[RT / 32];
    const int l = blockIdx.y;
    const double *v = V + (size_t)l * N;
    double s = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * RT + threadIdx.x; q < N; q += (int64_t)RED * RT) s += v[q] * w[q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[(size_t)l * RED + blockIdx.x] = s;
}
// out[l] = sum_cta partial[l*RED + cta]
__global__ void k_reduce_parts(int nv, const double *__restrict__ part, double *__restrict__ out) {
    const int l = blockIdx.x;
    __shared__ double sh[RT / 32];
    double s = 0.0;
    for (int q = threadIdx.x; q < RED; q += blockDim.x) s += part[(size_t)l * RED + q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[l] = s;
}
// partial sums of |x|^2
__global__ void __launch_bounds__(RT) k_sumsq(int64_t N, const double *__restrict__ x, double *__restrict__ part) {
    __shared__ double sh[RT / 32];
    double s = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * RT + threadIdx.x; q < N; q += (int64_t)RED * RT) s += x[q] * x[q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}
// out[0] = sqrt(sum parts) ; out[1] = 1 / out[0]
__global__ void k_norm_final(const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double sh[RT / 32];
    double s = 0.0;
    for (int q = threadIdx.x; q < RED; q += blockDim.x) s += part[q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        const double nr = sqrt(s);
        out[0] = nr;
        out[1] = 1. / nr;
    }
}
__global__ void k_axpby(int64_t N, double a, const double *__restrict__ x, double b, double *__restrict__ y) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = a * x[q] + b * y[q];
}
__global__ void k_copy(int64_t N, const double *__restrict__ x, double *__restrict__ y, const int *skip) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = x[q];
}
__global__ void k_fill(int64_t N, double v, double *__restrict__ y) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = v;
}
// Jacobi update x = (omega*Dinvb + x) - omega*t
__global__ void k_jacobi_update(int64_t N, double omega, const double *__restrict__ dinvb,
                                const double *__restrict__ t, double *__restrict__ x) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        x[q] = (omega * dinvb[q] + x[q]) - omega * t[q];
}

int grid_for(cpg_ctx *ctx, int64_t N) {
    const int64_t g = (N + 255) / 256;
    return (int)std::min<int64_t>(g, (int64_t)ctx->num_sms * 16);
}

// Krylov workspace from the context (grow-only)
cpg_status kws(cpg_ctx *ctx, size_t n, double **out) {
    if (n > ctx->kws_cap) {
        if (ctx->kws) {
            CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFree(ctx->kws);
            ctx->kws = nullptr;
            ctx->kws_cap = 0;
        }
        CPG_TRY(dmalloc(ctx, &ctx->kws, n));
        ctx->kws_cap = n;
    }
    *out = ctx->kws;
    return CPG_OK;
}

// device norm; result (norm, 1/norm) at out_dev[0..1]
cpg_status norm_dev(cpg_ctx *ctx, int64_t N, const double *x, double *part, double *out_dev) {
    k_sumsq<<<RED, RT, 0, ctx->stream>>>(N, x, part);
    CPG_TRY(launched(ctx, "sumsq kernel"));
    k_norm_final<<<1, RT, 0, ctx->stream>>>(part, out_dev);
    return launched(ctx, "norm kernel");
}

cpg_status read_host(cpg_ctx *ctx, const double *dev, int n, double *host) {
    double *hp;
    CPG_TRY(pinned(ctx, n, &hp));
    CPG_CUDA(ctx, cudaMemcpyAsync(hp, dev, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    std::memcpy(host, hp, n * sizeof(double));
    return CPG_OK;
}

}  // namespace

namespace cpg {

cpg_status vec_axpby(cpg_ctx *ctx, int64_t n, double a, const double *x, double b, double *y) {
    if (n <= 0) return CPG_OK;
    k_axpby<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(n, a, x, b, y);
    return launched(ctx, "axpby kernel");
}
cpg_status vec_copy(cpg_ctx *ctx, int64_t n, const double *x, double *y) {
    if (n <= 0) return CPG_OK;
    k_copy<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(n, x, y, ctx->skip_dev);
    return launched(ctx, "copy kernel");
}
cpg_status vec_fill(cpg_ctx *ctx, int64_t n, double v, double *y) {
    if (n <= 0) return CPG_OK;
    k_fill<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(n, v, y);
    return launched(ctx, "fill kernel");
}
cpg_status vec_dot(cpg_ctx *ctx, int64_t n, const double *x, const double *y, double *out_host) {
    double *part;
    CPG_TRY(scratch(ctx, RED + 8, &part));
    k_mdot<<<dim3(RED, 1), RT, 0, ctx->stream>>>(n, x, y, part);
    CPG_TRY(launched(ctx, "dot kernel"));
    k_reduce_parts<<<1, RT, 0, ctx->stream>>>(1, part, part + RED);
    CPG_TRY(launched(ctx, "dot reduce kernel"));
    return read_host(ctx, part + RED, 1, out_host);
}

}  // namespace cpg

// BSR operator / preconditioner pair
struct KrylovOp : LinOp {
    const cpg_bsr *A;
    const cpg_precond *P;
    bool split;  // P^{-1} A in split form (an FP64 ILU(0) of A's current values, rounding well below tol)
    KrylovOp(const cpg_bsr *a, const cpg_precond *p, double tol) : A(a), P(p), split(split_allowed(p, a, tol)) {}
    cpg_status apply(cpg_ctx *ctx, const double *x, double *y) const override { return bsr_matvec_raw(ctx, A, x, y); }
    cpg_status prec(cpg_ctx *ctx, double *x) const override { return precond_apply_raw(ctx, P, x); }
    cpg_status apply_prec(cpg_ctx *ctx, const double *x, double *y) const override {
        if (split) return split_apply_prec(ctx, A, P, x, y);
        return LinOp::apply_prec(ctx, x, y);
    }
};

namespace {
// ---------------------------------------------------------------------------
// Segmented GMRES: K independent systems stacked along the vector (a block
// diagonal operator, segment k = dofs [off[k], off[k+1])), each with its own
// Krylov scalars.  Every reduction runs per segment on a fixed grid (CPS CTAs
// a segment), so a system's result does not depend on what else is batched
// with it.  The Givens rotations, the least-squares update and the stopping
// test run on the device (one thread per system); once every system has
// converged, a device word makes the remaining launches of the cycle return
// at once.  The host enqueues a whole restart cycle and reads the systems'
// state once per cycle.  With K = 1 this is the reference's sequence
// (BlockMatrix.cpp:79-163) with the same sums in the same order.
// ---------------------------------------------------------------------------
constexpr int CPS = RED;  // CTAs per segment of a reduction

struct Seg {
    const int64_t *off;  // K + 1 dof offsets
    int K;
};
__device__ __forceinline__ bool skipped(const int *done) { return done && *done; }

// part[(l*K + seg)*CPS + cta] = this CTA's slice of V_l . w over the segment
__global__ void __launch_bounds__(RT) k_seg_mdot(Seg sg, const double *__restrict__ V, int64_t N,
                                                 const double *__restrict__ w, double *__restrict__ part,
                                                 const int *done) {
    if (skipped(done)) return;
    __shared__ double sh[RT / 32];
    const int l = blockIdx.y, seg = blockIdx.z;
    const int64_t a = sg.off[seg], b = sg.off[seg + 1];
    const double *v = V + (size_t)l * N;
    double s = 0.0;
    for (int64_t q = a + (int64_t)blockIdx.x * RT + threadIdx.x; q < b; q += (int64_t)CPS * RT) s += v[q] * w[q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[((size_t)l * sg.K + seg) * CPS + blockIdx.x] = s;
}
// out[seg*stride + l] = sum over the segment's CTAs (fixed order)
__global__ void k_seg_reduce(int K, const double *__restrict__ part, double *__restrict__ out, int stride,
                             const int *done) {
    if (skipped(done)) return;
    __shared__ double sh[RT / 32];
    const int l = blockIdx.x, seg = blockIdx.y;
    double s = 0.0;
    for (int q = threadIdx.x; q < CPS; q += blockDim.x) s += part[((size_t)l * K + seg) * CPS + q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[(size_t)seg * stride + l] = s;
}
// w -= sum_l h[l] V_l per segment (column order as dgemv 'N'); |w|^2 partials
__global__ void __launch_bounds__(RT) k_seg_cgs(Seg sg, int64_t N, int nv, const double *__restrict__ V,
                                                const double *__restrict__ h, int stride, double *__restrict__ w,
                                                double *__restrict__ part, const int *done) {
    if (skipped(done)) return;
    __shared__ double sh[RT / 32];
    __shared__ double sh_h[64];
    const int seg = blockIdx.y;
    for (int l = threadIdx.x; l < nv; l += RT) sh_h[l] = -h[(size_t)seg * stride + l];
    __syncthreads();
    const int64_t a = sg.off[seg], b = sg.off[seg + 1];
    constexpr int64_t STRIDE = (int64_t)CPS * RT;
    double s = 0.0;
    // two elements of the thread's sequence at a time (two independent
    // chains of loads in flight); each element, and the order in which the
    // thread sums their squares, is as for one element at a time
    for (int64_t q = a + (int64_t)blockIdx.x * RT + threadIdx.x; q < b; q += 2 * STRIDE) {
        const int64_t q2 = q + STRIDE;
        const bool two = q2 < b;
        double x = w[q], x2 = two ? w[q2] : 0.0;
        for (int l = 0; l < nv; l++) {
            const double hl = sh_h[l];
            x += hl * V[(size_t)l * N + q];
            if (two) x2 += hl * V[(size_t)l * N + q2];
        }
        w[q] = x;
        s += x * x;
        if (two) {
            w[q2] = x2;
            s += x2 * x2;
        }
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[(size_t)seg * CPS + blockIdx.x] = s;
}
// |x|^2 partials per segment
__global__ void __launch_bounds__(RT) k_seg_sumsq(Seg sg, const double *__restrict__ x, double *__restrict__ part,
                                                  const int *done) {
    if (skipped(done)) return;
    __shared__ double sh[RT / 32];
    const int seg = blockIdx.y;
    const int64_t a = sg.off[seg], b = sg.off[seg + 1];
    double s = 0.0;
    for (int64_t q = a + (int64_t)blockIdx.x * RT + threadIdx.x; q < b; q += (int64_t)CPS * RT) s += x[q] * x[q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[(size_t)seg * CPS + blockIdx.x] = s;
}
// out[seg*stride + idx] = sqrt(sum), out[... + idx + 1] = 1 / that
__global__ void k_seg_norm(const double *__restrict__ part, double *__restrict__ out, int stride, int idx,
                           const int *done) {
    if (skipped(done)) return;
    __shared__ double sh[RT / 32];
    const int seg = blockIdx.x;
    double s = 0.0;
    for (int q = threadIdx.x; q < CPS; q += blockDim.x) s += part[(size_t)seg * CPS + q];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) {
        const double nr = sqrt(s);
        out[(size_t)seg * stride + idx] = nr;
        out[(size_t)seg * stride + idx + 1] = 1. / nr;
    }
}
// y = x * sc[seg*stride + idx] over each segment
__global__ void k_seg_scale(Seg sg, const double *__restrict__ x, const double *__restrict__ sc, int stride, int idx,
                            double *__restrict__ y, const int *done) {
    if (skipped(done)) return;
    const int seg = blockIdx.y;
    const double f = sc[(size_t)seg * stride + idx];
    const int64_t a = sg.off[seg], b = sg.off[seg + 1];
    for (int64_t q = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < b; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = x[q] * f;
}
// x += sum_{l < nsteps[seg]} cy[seg][l] * B_l over each segment
__global__ void k_seg_combine(Seg sg, int64_t N, const double *__restrict__ B, const double *__restrict__ cy,
                              int cstride, const int *__restrict__ nsteps, double *__restrict__ x) {
    __shared__ double sc[64];
    const int seg = blockIdx.y, nv = nsteps[seg];
    if (nv <= 0) return;
    for (int l = threadIdx.x; l < nv; l += blockDim.x) sc[l] = cy[(size_t)seg * cstride + l];
    __syncthreads();
    const int64_t a = sg.off[seg], b = sg.off[seg + 1];
    for (int64_t q = a + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < b; q += (int64_t)gridDim.x * blockDim.x) {
        double v = x[q];
        for (int l = 0; l < nv; l++) v += sc[l] * B[(size_t)l * N + q];
        x[q] = v;
    }
}

// Krylov scalars of the K systems (device)
struct KState {
    double *hcol;   // K x HS: h column of the step, then |w|, 1/|w|; slot 0/1 of a restart: beta, 1/beta
    double *H;      // K x HP: packed upper triangle (Givens-rotated Hessenberg)
    double *c, *s;  // K x m
    double *y;      // K x (m+1)
    double *cy;     // K x (m+1): solution-update coefficients
    double *nrm2b;  // K x 2
    int *active;    // K: still iterating in this cycle
    int *nsteps;    // K: Arnoldi steps taken in this cycle
    int *finished;  // K: converged (stops for good)
    int *its;       // K: iterations as the reference counts them
    int *done;      // 1: no system active
    int *status;    // 1: a non-finite quantity (bit 0)
    int HS, HP, m;
};

// start of a cycle: y0 = beta, decide which systems iterate
__global__ void k_gmres_start(int K, KState st, double tol) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int seg = threadIdx.x; seg < K; seg += blockDim.x) {
        const double beta = st.hcol[(size_t)seg * st.HS];
        if (!isfinite(beta) || !isfinite(st.nrm2b[2 * seg])) atomicOr(st.status, 1);
        st.y[(size_t)seg * (st.m + 1)] = beta;
        st.nsteps[seg] = 0;
        const bool act = !st.finished[seg] && !(fabs(beta) < tol * st.nrm2b[2 * seg]);
        st.active[seg] = act ? 1 : 0;
        if (act) atomicOr(&any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) *st.done = any ? 0 : 1;
}

// step i: rotate the new Hessenberg column, new rotation, update y, test
__global__ void k_givens(int K, int i, KState st, double tol) {
    if (skipped(st.done)) return;
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int seg = threadIdx.x; seg < K; seg += blockDim.x) {
        if (!st.active[seg]) continue;
        const double *hb = st.hcol + (size_t)seg * st.HS;
        double *H = st.H + (size_t)seg * st.HP, *c = st.c + (size_t)seg * st.m, *s = st.s + (size_t)seg * st.m;
        double *y = st.y + (size_t)seg * (st.m + 1);
        int u = i * (i + 1) / 2;
        for (int l = 0; l <= i; l++) H[u + l] = hb[l];
        const double hnew = hb[i + 1];
        if (!isfinite(hnew)) atomicOr(st.status, 1);
        for (int k = 0; k < i; ++k) {
            const double tmp = __dsub_rn(__dmul_rn(c[k], H[u]), __dmul_rn(s[k], H[u + 1]));
            H[u + 1] = __dadd_rn(__dmul_rn(s[k], H[u]), __dmul_rn(c[k], H[u + 1]));
            H[u] = tmp;
            ++u;
        }
        const double rd = H[u];
        const double dd = __dsqrt_rn(__dadd_rn(__dmul_rn(rd, rd), __dmul_rn(hnew, hnew)));
        c[i] = __ddiv_rn(rd, dd);
        s[i] = __ddiv_rn(-hnew, dd);
        H[u] = dd;
        y[i + 1] = __dmul_rn(s[i], y[i]);
        y[i] = __dmul_rn(c[i], y[i]);
        st.nsteps[seg] = i + 1;
        const bool more = i + 1 < st.m && !(fabs(y[i + 1]) < tol * st.nrm2b[2 * seg]);
        st.active[seg] = more ? 1 : 0;
        if (more) atomicOr(&any, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0 && !any) *st.done = 1;
}

// end of a cycle: R y = g (packed upper triangle, dtpsv 'U','N','N'), the
// update coefficients, and whether each system has converged
__global__ void k_gmres_end(int K, int j, KState st, double tol, int flexible) {
    for (int seg = blockIdx.x * blockDim.x + threadIdx.x; seg < K; seg += gridDim.x * blockDim.x) {
        if (st.finished[seg]) {
            st.nsteps[seg] = 0;  // leaves x alone
            continue;
        }
        const int i = st.nsteps[seg];
        const double *H = st.H + (size_t)seg * st.HP;
        double *y = st.y + (size_t)seg * (st.m + 1), *cy = st.cy + (size_t)seg * (st.m + 1);
        for (int col = i - 1; col >= 0; col--) {
            const int kk = col * (col + 1) / 2;
            y[col] = __ddiv_rn(y[col], H[kk + col]);
            for (int row = 0; row < col; row++) y[row] = __dsub_rn(y[row], __dmul_rn(y[col], H[kk + row]));
        }
        for (int l = 0; l < i; l++) cy[l] = flexible ? y[l] : -y[l];
        st.its[seg] = st.m * j + i;
        const double r = fabs(y[i]);
        st.nrm2b[2 * seg + 1] = r;
        if (r < tol * st.nrm2b[2 * seg]) st.finished[seg] = 1;
    }
}

int grid_seg(int64_t N, int K) {
    const int64_t per = (N / std::max(1, K) + 255) / 256;
    return (int)std::max<int64_t>(1, std::min<int64_t>(per, 512));
}

cpg_status seg_norm(cpg_ctx *ctx, const Seg &sg, const double *x, double *part, double *out, int stride, int idx,
                    const int *done) {
    k_seg_sumsq<<<dim3(CPS, sg.K), RT, 0, ctx->stream>>>(sg, x, part, done);
    CPG_TRY(launched(ctx, "segmented sumsq kernel"));
    k_seg_norm<<<sg.K, RT, 0, ctx->stream>>>(part, out, stride, idx, done);
    return launched(ctx, "segmented norm kernel");
}

cpg_status gmres_seg_run(cpg_ctx *ctx, const LinOp &op, int K, const int64_t *off_host, const double *b, double *x,
                         int m, double tol, int maxit, int flexible, cpg_solve_stats *stats) {
    if (m < 1 || m > 62) return fail(ctx, CPG_ERR_INVALID_ARG, "GMRES restart must be 1..62");
    if (K < 1 || K > 1024) return fail(ctx, CPG_ERR_INVALID_ARG, "1..1024 systems per batched solve");
    const int64_t N = off_host[K];
    // workspace: V (m+1) N, r N, [Z m N]
    const size_t need = (size_t)(m + 2 + (flexible ? m : 0)) * N;
    double *ws;
    CPG_TRY(kws(ctx, need, &ws));
    double *V = ws, *r = ws + (size_t)(m + 1) * N, *Z = r + N;
    // scratch: partials, the systems' scalars, offsets and ints
    const int HS = m + 4, HP = m * (m + 1) / 2 + 1;
    const size_t n_part = (size_t)CPS * K * (m + 2);
    const size_t n_dbl = n_part + (size_t)K * (HS + HP + 2 * m + 2 * (m + 1) + 2);
    // after the doubles: K + 1 int64 offsets, then 4K + 2 ints
    double *sc;
    CPG_TRY(scratch(ctx, n_dbl + (size_t)(K + 1) + (size_t)(2 * K + 1) + 4, &sc));
    double *part = sc;
    KState st;
    st.m = m;
    st.HS = HS;
    st.HP = HP;
    st.hcol = part + n_part;
    st.H = st.hcol + (size_t)K * HS;
    st.c = st.H + (size_t)K * HP;
    st.s = st.c + (size_t)K * m;
    st.y = st.s + (size_t)K * m;
    st.cy = st.y + (size_t)K * (m + 1);
    st.nrm2b = st.cy + (size_t)K * (m + 1);
    int64_t *off_dev = (int64_t *)(st.nrm2b + 2 * (size_t)K);
    int *ints = (int *)(off_dev + K + 1);
    st.active = ints;
    st.nsteps = ints + K;
    st.finished = ints + 2 * K;
    st.its = ints + 3 * K;
    st.done = ints + 4 * K;
    st.status = ints + 4 * K + 1;
    CPG_CUDA(ctx, cudaMemcpyAsync(off_dev, off_host, sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, ctx->stream));
    CPG_CUDA(ctx, cudaMemsetAsync(ints, 0, sizeof(int) * (4 * K + 2), ctx->stream));
    const Seg sg{off_dev, K};
    const dim3 vgrid(grid_seg(N, K), K);

    // nrm2b: |P^{-1} b| (left) or |b| (flexible), per system
    CPG_TRY(vec_copy(ctx, N, b, r));
    if (!flexible) CPG_TRY(op.prec(ctx, r));
    CPG_TRY(seg_norm(ctx, sg, r, part, st.nrm2b, 2, 0, nullptr));
    if (maxit % m > 0) maxit = (maxit / m + 1) * m;
    const int cycles = maxit / m;
    int j;
    cpg_status rc = CPG_OK;
    for (j = 0; j < cycles && rc == CPG_OK; j++) {
        // r = P^{-1}(A x - b)   or   r = b - A x ; beta, V_0 = r / beta
        CPG_TRY(op.apply(ctx, x, r));
        if (!flexible) {
            CPG_TRY(vec_axpby(ctx, N, -1.0, b, 1.0, r));
            CPG_TRY(op.prec(ctx, r));
        } else {
            CPG_TRY(vec_axpby(ctx, N, 1.0, b, -1.0, r));
        }
        CPG_TRY(seg_norm(ctx, sg, r, part, st.hcol, HS, 0, nullptr));
        k_seg_scale<<<vgrid, 256, 0, ctx->stream>>>(sg, r, st.hcol, HS, 1, V, nullptr);
        CPG_TRY(launched(ctx, "segmented scale kernel"));
        k_gmres_start<<<1, 1024, 0, ctx->stream>>>(K, st, tol);
        CPG_TRY(launched(ctx, "gmres start kernel"));
        // the cycle, with no host synchronisation: once every system has
        // converged the remaining launches return at once
        ctx->skip_dev = st.done;
        for (int i = 0; i < m && rc == CPG_OK; i++) {
            double *vi = V + (size_t)N * i, *vi1 = V + (size_t)N * (i + 1);
            if (!flexible) {
                rc = op.apply_prec(ctx, vi, vi1);
            } else {
                double *zi = Z + (size_t)N * i;
                rc = vec_copy(ctx, N, vi, zi);
                if (rc == CPG_OK) rc = op.prec(ctx, zi);
                if (rc == CPG_OK) rc = op.apply(ctx, zi, vi1);
            }
            if (rc != CPG_OK) break;
            // h = V^T w ; w -= V h ; |w| ; w /= |w| ; Givens
            k_seg_mdot<<<dim3(CPS, i + 1, K), RT, 0, ctx->stream>>>(sg, V, N, vi1, part, st.done);
            rc = launched(ctx, "segmented multi-dot kernel");
            if (rc == CPG_OK) {
                k_seg_reduce<<<dim3(i + 1, K), RT, 0, ctx->stream>>>(K, part, st.hcol, HS, st.done);
                rc = launched(ctx, "segmented multi-dot reduce kernel");
            }
            if (rc == CPG_OK) {
                k_seg_cgs<<<dim3(CPS, K), RT, 0, ctx->stream>>>(sg, N, i + 1, V, st.hcol, HS, vi1, part, st.done);
                rc = launched(ctx, "segmented gram-schmidt kernel");
            }
            if (rc == CPG_OK) {
                k_seg_norm<<<K, RT, 0, ctx->stream>>>(part, st.hcol, HS, i + 1, st.done);
                rc = launched(ctx, "segmented norm kernel");
            }
            if (rc == CPG_OK) {
                k_seg_scale<<<vgrid, 256, 0, ctx->stream>>>(sg, vi1, st.hcol, HS, i + 2, vi1, st.done);
                rc = launched(ctx, "segmented scale kernel");
            }
            if (rc == CPG_OK) {
                k_givens<<<1, 1024, 0, ctx->stream>>>(K, i, st, tol);
                rc = launched(ctx, "givens kernel");
            }
        }
        ctx->skip_dev = nullptr;
        if (rc != CPG_OK) break;
        k_gmres_end<<<(K + 255) / 256, 256, 0, ctx->stream>>>(K, j, st, tol, flexible);
        CPG_TRY(launched(ctx, "gmres end kernel"));
        k_seg_combine<<<vgrid, 256, 0, ctx->stream>>>(sg, N, flexible ? Z : V, st.cy, m + 1, st.nsteps, x);
        CPG_TRY(launched(ctx, "solution update kernel"));
        // one read-back per cycle: which systems have converged, and status
        double *hbuf;
        CPG_TRY(pinned(ctx, (size_t)(K + 2) / 2 + 1, &hbuf));
        int *hp = reinterpret_cast<int *>(hbuf);  // K + 1 ints
        CPG_CUDA(ctx, cudaMemcpyAsync(hp, st.finished, sizeof(int) * K, cudaMemcpyDeviceToHost, ctx->stream));
        CPG_CUDA(ctx, cudaMemcpyAsync(hp + K, st.status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        if (hp[K]) return fail(ctx, CPG_ERR_NONFINITE, "non-finite GMRES quantity (right-hand side, residual or "
                                                       "Arnoldi vector)");
        bool all = true;
        for (int k = 0; k < K; k++) all = all && hp[k];
        if (all) break;
    }
    if (rc != CPG_OK) return rc;
    // iteration counts and residuals as the reference reports them
    // (BlockMatrix.cpp:157-158): its = m*j + i, |y_i| / |P^{-1} b|
    std::vector<int> its(K), finh(K);
    std::vector<double> nb(2 * (size_t)K);
    CPG_CUDA(ctx, cudaMemcpyAsync(its.data(), st.its, sizeof(int) * K, cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaMemcpyAsync(finh.data(), st.finished, sizeof(int) * K, cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaMemcpyAsync(nb.data(), st.nrm2b, sizeof(double) * 2 * K, cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < K && stats; k++) {
        const double res = nb[2 * k] > 0 ? nb[2 * k + 1] / nb[2 * k] : 0.0;
        stats[k].iterations = finh[k] ? its[k] : m * cycles + m;
        stats[k].residual = res;
        stats[k].converged = res < tol ? 1 : 0;
    }
    return CPG_OK;
}
}  // namespace

namespace cpg {
// one status check per solve: a triangular sweep whose bounded wait ran out
// turns the whole solve into CPG_ERR_TIMEOUT
cpg_status gmres_op(cpg_ctx *ctx, const LinOp &op, int64_t N, const double *b, double *x, int m, double tol,
                    int maxit, int flexible, cpg_solve_stats *stats) {
    const int64_t off[2] = {0, N};
    return check_sweep_error(ctx, gmres_seg_run(ctx, op, 1, off, b, x, m, tol, maxit, flexible, stats));
}
}  // namespace cpg

extern "C" {

cpg_status cpg_gmres(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, const double *b, double *x, int m,
                     double tol, int maxit, int flexible, cpg_solve_stats *stats) {
    if (!ctx || !A || !b || !x || maxit < 1) return CPG_ERR_INVALID_ARG;
    if (P && (P->n != A->n_rows || P->bl != A->bl)) return fail(ctx, CPG_ERR_INVALID_ARG, "preconditioner size");
    KrylovOp op(A, P, tol);
    return gmres_op(ctx, op, (int64_t)A->n_rows * A->bl, b, x, m, tol, maxit, flexible, stats);
}

cpg_status cpg_gmres_batched(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, int nsys, const int *seg_rows,
                             const double *b, double *x, int m, double tol, int maxit, int flexible,
                             cpg_solve_stats *stats) {
    if (!ctx || !A || !b || !x || !seg_rows || maxit < 1 || nsys < 1) return CPG_ERR_INVALID_ARG;
    if (P && (P->n != A->n_rows || P->bl != A->bl)) return fail(ctx, CPG_ERR_INVALID_ARG, "preconditioner size");
    if (seg_rows[0] != 0 || seg_rows[nsys] != A->n_rows)
        return fail(ctx, CPG_ERR_INVALID_ARG, "system row ranges must start at 0 and end at the matrix's rows");
    std::vector<int64_t> off(nsys + 1);
    for (int k = 0; k <= nsys; k++) {
        if (k > 0 && seg_rows[k] <= seg_rows[k - 1])
            return fail(ctx, CPG_ERR_INVALID_ARG, "system row ranges must be increasing and non-empty");
        off[k] = (int64_t)seg_rows[k] * A->bl;
    }
    // the systems must be independent: every block of a row lies in the row's system
    for (int k = 0; k < nsys; k++)
        for (int i = seg_rows[k]; i < seg_rows[k + 1]; i++)
            for (int q = A->rowptr[i]; q < A->rowptr[i + 1]; q++)
                if (A->colidx[q] < seg_rows[k] || A->colidx[q] >= seg_rows[k + 1])
                    return fail(ctx, CPG_ERR_INVALID_ARG,
                                "block (" + std::to_string(i) + ", " + std::to_string(A->colidx[q]) +
                                    ") couples two systems");
    KrylovOp op(A, P, tol);
    return check_sweep_error(ctx, gmres_seg_run(ctx, op, nsys, off.data(), b, x, m, tol, maxit, flexible, stats));
}

}  // extern "C"

namespace {
cpg_status jacobi_run(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, const double *b, double *x,
                      double tol, int maxit, cpg_solve_stats *stats) {
    const int64_t N = (int64_t)A->n_rows * A->bl;
    double *ws;
    CPG_TRY(kws(ctx, 3 * (size_t)N, &ws));
    double *dinvb = ws, *t = ws + N, *r = ws + 2 * N;
    double *sc;
    CPG_TRY(scratch(ctx, RED + 8, &sc));
    const double omega = 1.0;
    CPG_TRY(vec_copy(ctx, N, b, dinvb));
    CPG_TRY(precond_apply_raw(ctx, P, dinvb));
    int mm;
    double nr = 0.0;
    for (mm = 0; mm < maxit; mm++) {
        CPG_TRY(bsr_matvec_raw(ctx, A, x, t));
        CPG_TRY(vec_copy(ctx, N, t, r));
        CPG_TRY(vec_axpby(ctx, N, -1.0, b, 1.0, r));
        CPG_TRY(norm_dev(ctx, N, r, sc, sc + RED));
        CPG_TRY(read_host(ctx, sc + RED, 1, &nr));
        if (!std::isfinite(nr)) return fail(ctx, CPG_ERR_NONFINITE, "non-finite Jacobi residual");
        if (nr < tol) break;
        CPG_TRY(precond_apply_raw(ctx, P, t));
        k_jacobi_update<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, omega, dinvb, t, x);
        CPG_TRY(launched(ctx, "jacobi update kernel"));
    }
    if (stats) {
        stats->iterations = mm;
        stats->residual = nr;
        stats->converged = nr < tol ? 1 : 0;
    }
    return CPG_OK;
}
}  // namespace

extern "C" {

cpg_status cpg_jacobi_solve(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, const double *b, double *x,
                            double tol, int maxit, cpg_solve_stats *stats) {
    if (!ctx || !A || !P || !b || !x) return CPG_ERR_INVALID_ARG;
    return check_sweep_error(ctx, jacobi_run(ctx, A, P, b, x, tol, maxit, stats));
}

cpg_status cpg_axpby(cpg_ctx *ctx, int64_t n, double a, const double *x, double b, double *y) {
    if (!ctx || !x || !y || n < 0) return CPG_ERR_INVALID_ARG;
    return vec_axpby(ctx, n, a, x, b, y);
}

}  // extern "C"
