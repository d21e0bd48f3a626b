// Krylov solvers and vector kernels: restarted GMRES with classical
// Gram-Schmidt (BlockMatrix::gmres, src/BlockMatrix.cpp:79-163), its flexible
// right-preconditioned variant (FGMRES), damped block Jacobi
// (BlockMatrix::jacobi, :51-77), and MeshFn arithmetic.
//
// The Krylov basis V lives on the device, column i at V + i*N.  One Arnoldi
// step is: matvec, preconditioner, h = V^T w (multi-dot), w -= V h fused with
// the partial sums of |w|^2, normalisation; the host reads h and |w| once per
// step for the Givens rotations (a few doubles), exactly the reference's
// sequence.  Reductions use a fixed grid and a fixed combination order, so
// results are reproducible run to run.
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
// w -= sum_l h[l] V_l (column order as dgemv 'N'); partial sums of |w|^2
__global__ void __launch_bounds__(RT) k_cgs_update(int64_t N, int nv, const double *__restrict__ V,
                                                   const double *__restrict__ h, double *__restrict__ w,
                                                   double *__restrict__ part) {
    __shared__ double sh[RT / 32];
    __shared__ double sh_h[64];
    for (int l = threadIdx.x; l < nv; l += RT) sh_h[l] = -h[l];
    __syncthreads();
    double s = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * RT + threadIdx.x; q < N; q += (int64_t)RED * RT) {
        double x = w[q];
        for (int l = 0; l < nv; l++) x += sh_h[l] * V[(size_t)l * N + q];
        w[q] = x;
        s += x * x;
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
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
// y = x * (*scale)
__global__ void k_scale_dev(int64_t N, const double *__restrict__ x, const double *__restrict__ scale,
                            double *__restrict__ y) {
    const double a = *scale;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = x[q] * a;
}
// x += sum_l c[l] V_l
__global__ void k_combine_basis(int64_t N, int nv, const double *__restrict__ V, const double *__restrict__ c,
                                double *__restrict__ x) {
    __shared__ double sc[64];
    for (int l = threadIdx.x; l < nv; l += blockDim.x) sc[l] = c[l];
    __syncthreads();
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        double v = x[q];
        for (int l = 0; l < nv; l++) v += sc[l] * V[(size_t)l * N + q];
        x[q] = v;
    }
}
__global__ void k_axpby(int64_t N, double a, const double *__restrict__ x, double b, double *__restrict__ y) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        y[q] = a * x[q] + b * y[q];
}
__global__ void k_copy(int64_t N, const double *__restrict__ x, double *__restrict__ y) {
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
    k_copy<<<grid_for(ctx, n), 256, 0, ctx->stream>>>(n, x, y);
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
    KrylovOp(const cpg_bsr *a, const cpg_precond *p) : A(a), P(p) {}
    cpg_status apply(cpg_ctx *ctx, const double *x, double *y) const override { return bsr_matvec_raw(ctx, A, x, y); }
    cpg_status prec(cpg_ctx *ctx, double *x) const override { return precond_apply_raw(ctx, P, x); }
};

namespace {
cpg_status gmres_run(cpg_ctx *ctx, const LinOp &op, int64_t N, const double *b, double *x, int m, double tol,
                     int maxit, int flexible, cpg_solve_stats *stats) {
    if (m < 1 || m > 62) return fail(ctx, CPG_ERR_INVALID_ARG, "GMRES restart must be 1..62");
    // workspace: V (m+1) N, r N, [Z m N]
    const size_t need = (size_t)(m + 2 + (flexible ? m : 0)) * N;
    double *ws;
    CPG_TRY(kws(ctx, need, &ws));
    double *V = ws, *r = ws + (size_t)(m + 1) * N, *Z = r + N;
    // small device vectors: parts (RED * (m+1)), hdev (m+2), nrm (2), ydev (m+1)
    double *sc;
    CPG_TRY(scratch(ctx, (size_t)RED * (m + 2) + 4 * (m + 4), &sc));
    double *part = sc, *hdev = sc + (size_t)RED * (m + 2), *nrm = hdev + (m + 4), *ydev = nrm + (m + 4);
    std::vector<double> h((size_t)m * (m + 1) / 2 + 1, 0.0), y(m + 1, 0.0), c(m, 0.0), s(m, 0.0), hb(m + 2);
    double beta, hnew, rd, dd, nrm2b, tmp2[2];
    int i = 0, j, uki, u0i;

    // nrm2b: |P^{-1} b| (left) or |b| (flexible)
    CPG_TRY(vec_copy(ctx, N, b, r));
    if (!flexible) CPG_TRY(op.prec(ctx, r));
    CPG_TRY(norm_dev(ctx, N, r, part, nrm));
    CPG_TRY(read_host(ctx, nrm, 2, tmp2));
    nrm2b = tmp2[0];
    if (!std::isfinite(nrm2b)) return fail(ctx, CPG_ERR_NONFINITE, "non-finite right-hand side");
    if (maxit % m > 0) maxit = (maxit / m + 1) * m;
    const int cycles = maxit / m;
    for (j = 0; j < cycles; j++) {
        // r = P^{-1}(A x - b)   or   r = b - A x
        CPG_TRY(op.apply(ctx, x, r));
        if (!flexible) {
            CPG_TRY(vec_axpby(ctx, N, -1.0, b, 1.0, r));
            CPG_TRY(op.prec(ctx, r));
        } else {
            CPG_TRY(vec_axpby(ctx, N, 1.0, b, -1.0, r));
        }
        CPG_TRY(norm_dev(ctx, N, r, part, nrm));
        k_scale_dev<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, r, nrm + 1, V);
        CPG_TRY(launched(ctx, "scale kernel"));
        CPG_TRY(read_host(ctx, nrm, 1, &beta));
        if (!std::isfinite(beta)) return fail(ctx, CPG_ERR_NONFINITE, "non-finite GMRES residual");
        y[0] = beta;
        uki = 0;
        for (i = 0; i < m; i++) {
            if (std::fabs(y[i]) < tol * nrm2b) break;
            double *vi = V + (size_t)N * i, *vi1 = V + (size_t)N * (i + 1);
            u0i = uki;
            if (!flexible) {
                CPG_TRY(op.apply(ctx, vi, vi1));
                CPG_TRY(op.prec(ctx, vi1));
            } else {
                double *zi = Z + (size_t)N * i;
                CPG_TRY(vec_copy(ctx, N, vi, zi));
                CPG_TRY(op.prec(ctx, zi));
                CPG_TRY(op.apply(ctx, zi, vi1));
            }
            // h = V^T w ; w -= V h ; |w|
            k_mdot<<<dim3(RED, i + 1), RT, 0, ctx->stream>>>(N, V, vi1, part);
            CPG_TRY(launched(ctx, "multi-dot kernel"));
            k_reduce_parts<<<i + 1, RT, 0, ctx->stream>>>(i + 1, part, hdev);
            CPG_TRY(launched(ctx, "multi-dot reduce kernel"));
            k_cgs_update<<<RED, RT, 0, ctx->stream>>>(N, i + 1, V, hdev, vi1, part);
            CPG_TRY(launched(ctx, "gram-schmidt kernel"));
            k_norm_final<<<1, RT, 0, ctx->stream>>>(part, hdev + i + 1);
            CPG_TRY(launched(ctx, "norm kernel"));
            k_scale_dev<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, vi1, hdev + i + 2, vi1);
            CPG_TRY(launched(ctx, "scale kernel"));
            CPG_TRY(read_host(ctx, hdev, i + 2, hb.data()));
            for (int l = 0; l <= i; l++) h[u0i + l] = hb[l];
            hnew = hb[i + 1];
            if (!std::isfinite(hnew)) return fail(ctx, CPG_ERR_NONFINITE, "non-finite Arnoldi vector");
            for (int k = 0; k < i; ++k) {
                const double tmp = c[k] * h[uki] - s[k] * h[uki + 1];
                h[uki + 1] = s[k] * h[uki] + c[k] * h[uki + 1];
                h[uki] = tmp;
                ++uki;
            }
            rd = h[uki];
            dd = std::sqrt(rd * rd + hnew * hnew);
            c[i] = rd / dd;
            s[i] = -hnew / dd;
            h[uki] = dd;
            ++uki;
            y[i + 1] = s[i] * y[i];
            y[i] = c[i] * y[i];
        }
        // R y = g (packed upper triangle, dtpsv 'U','N','N')
        for (int col = i - 1; col >= 0; col--) {
            const int kk = col * (col + 1) / 2;
            y[col] /= h[kk + col];
            for (int row = 0; row < col; row++) y[row] -= y[col] * h[kk + row];
        }
        if (i > 0) {
            std::vector<double> cy(i);
            for (int l = 0; l < i; l++) cy[l] = flexible ? y[l] : -y[l];
            double *hp;
            CPG_TRY(pinned(ctx, i, &hp));
            std::memcpy(hp, cy.data(), sizeof(double) * i);
            CPG_CUDA(ctx, cudaMemcpyAsync(ydev, hp, sizeof(double) * i, cudaMemcpyHostToDevice, ctx->stream));
            k_combine_basis<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, i, flexible ? Z : V, ydev, x);
            CPG_TRY(launched(ctx, "solution update kernel"));
            CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        }
        if (std::fabs(y[i]) < tol * nrm2b) break;
    }
    // iteration count and residual as the reference reports them
    // (BlockMatrix.cpp:157-158)
    const int its = m * j + i;
    const double res = nrm2b > 0 ? std::fabs(y[i]) / nrm2b : 0.0;
    if (stats) {
        stats->iterations = its;
        stats->residual = res;
        stats->converged = res < tol ? 1 : 0;
    }
    return CPG_OK;
}
}  // namespace

namespace cpg {
// one status check per solve: a triangular sweep whose bounded wait ran out
// turns the whole solve into CPG_ERR_TIMEOUT
cpg_status gmres_op(cpg_ctx *ctx, const LinOp &op, int64_t N, const double *b, double *x, int m, double tol,
                    int maxit, int flexible, cpg_solve_stats *stats) {
    return check_sweep_error(ctx, gmres_run(ctx, op, N, b, x, m, tol, maxit, flexible, stats));
}
}  // namespace cpg

extern "C" {

cpg_status cpg_gmres(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, const double *b, double *x, int m,
                     double tol, int maxit, int flexible, cpg_solve_stats *stats) {
    if (!ctx || !A || !b || !x || maxit < 1) return CPG_ERR_INVALID_ARG;
    if (P && (P->n != A->n_rows || P->bl != A->bl)) return fail(ctx, CPG_ERR_INVALID_ARG, "preconditioner size");
    KrylovOp op(A, P);
    return gmres_op(ctx, op, (int64_t)A->n_rows * A->bl, b, x, m, tol, maxit, flexible, stats);
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
