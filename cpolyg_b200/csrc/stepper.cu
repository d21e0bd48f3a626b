// Time integration (src/TimeIntegration.cpp): ForwardEuler, RK2, RK4,
// BackwardEuler, DIRK (3 and 5 stages) and Radau IIA IRK (2 and 3 stages,
// IRK::advance and IRK::newAdvance).  Host control flow over the C ABI; the
// per-element stage arithmetic runs in the kernels below, written in the
// reference's evaluation order.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "internal.hpp"

using namespace cpg;

namespace {

// out = ((u + a0 k0) + a1 k1) + ...   (MeshFn += scalar * MeshFn chains)
struct Comb {
    const double *k[8];
    double a[8];
    int nk;
};
// skip: a Krylov solve's converged word (null outside a solve's cycle)
__global__ void k_combine(int64_t N, const double *__restrict__ u, Comb c, double *__restrict__ out,
                          const int *skip) {
    if (skip && *skip) return;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        double v = u ? u[q] : 0.0;
        for (int j = 0; j < c.nk; j++) v = v + c.a[j] * c.k[j][q];
        out[q] = v;
    }
}
// RK4 (TimeIntegration.cpp:14-22): u + (k1 + 2*k2 + 2*k3 + k4)/6
__global__ void k_rk4_final(int64_t N, const double *__restrict__ k1, const double *__restrict__ k2,
                            const double *__restrict__ k3, const double *__restrict__ k4, double *__restrict__ u) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        u[q] = u[q] + (((k1[q] + 2 * k2[q]) + 2 * k3[q]) + k4[q]) * (1.0 / 6.0);
}
// RK2: u + 0.5*(k1 + k2)
__global__ void k_rk2_final(int64_t N, const double *__restrict__ k1, const double *__restrict__ k2,
                            double *__restrict__ u) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x)
        u[q] = u[q] + 0.5 * (k1[q] + k2[q]);
}

// stage-coupled BSR assembly (BlockMatrix::blockBlockMatrix,
// BlockMatrix.cpp:228-258): out = (J[src]*s1)*s2 + M_r*mc on mass blocks
struct CoupledMap {
    const int *src;      // source block in the stacked stage Jacobians, -1 = none
    const double *s1, *s2, *mc;
    const int *mrow;     // cell whose mass block is added, -1 = none
};
template <class T>
__global__ void k_build_coupled(int64_t nblk, int nb, int nc, CoupledMap mp, const T *__restrict__ Jst,
                                const double *__restrict__ mass, T *__restrict__ out) {
    const int bl = nb * nc;
    const int64_t b2 = (int64_t)bl * bl;
    for (int64_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const int src = mp.src[blk], mr = mp.mrow[blk];
        const double s1 = mp.s1[blk], s2 = mp.s2[blk], mc = mp.mc[blk];
        for (int e = threadIdx.x; e < b2; e += blockDim.x) {
            double v = src >= 0 ? ((double)Jst[(size_t)src * b2 + e] * s1) * s2 : 0.0;
            if (mr >= 0) {
                const int r = e % bl, c = e / bl;
                if (r / nb == c / nb) v = v + mass[(size_t)mr * nb * nb + (c % nb) * nb + (r % nb)] * mc;
            }
            out[blk * b2 + e] = (T)v;
        }
    }
}

// cell-coupled stage blocks for CPG_PC_STAGE_BJACOBI:
// P_K(i,j) = delta_ij M_K - dt A(i,j) J_i,KK  as an (s*bl)^2 block per cell
template <class T>
__global__ void k_build_stage_blocks(int n, int s, int nb, int nc, const T *__restrict__ Jst, int64_t nnzb,
                                     const int *__restrict__ rowptr, const double *__restrict__ Acoef, double dt,
                                     const double *__restrict__ mass, T *__restrict__ out) {
    const int bl = nb * nc, S = s * bl;
    const int cell = blockIdx.x;
    if (cell >= n) return;
    const int64_t b2 = (int64_t)bl * bl;
    T *P = out + (size_t)cell * S * S;
    for (int e = threadIdx.x; e < S * S; e += blockDim.x) {
        const int R = e % S, C = e / S;
        const int i = R / bl, j = C / bl, r = R % bl, c = C % bl;
        const double jv = (double)Jst[((size_t)i * nnzb + rowptr[cell]) * b2 + (size_t)c * bl + r];
        double v = (jv * -dt) * Acoef[i * s + j];
        if (i == j && r / nb == c / nb) v = v + mass[(size_t)cell * nb * nb + (c % nb) * nb + (r % nb)];
        P[e] = (T)v;
    }
}
// stage-major [stage][cell][bl] <-> cell-major [cell][stage][bl]
__global__ void k_stage_perm(int n, int s, int bl, const double *__restrict__ in, double *__restrict__ out,
                             int to_cell, const int *skip) {
    if (skip && *skip) return;
    const int64_t N = (int64_t)n * s * bl;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < N; q += (int64_t)gridDim.x * blockDim.x) {
        // q indexes the stage-major vector
        const int64_t stage = q / ((int64_t)n * bl), rem = q % ((int64_t)n * bl);
        const int64_t cell = rem / bl, r = rem % bl;
        const int64_t qc = (cell * s + stage) * bl + r;
        if (to_cell) out[qc] = in[q];
        else out[q] = in[qc];
    }
}

int grid_for(cpg_ctx *ctx, int64_t N) {
    return (int)std::min<int64_t>((N + 255) / 256, (int64_t)ctx->num_sms * 16);
}

void tableau(int kind, int &s, std::vector<double> &A, std::vector<double> &Ainv, std::vector<double> &b,
             std::vector<double> &c) {
    const double r6 = std::sqrt(6.0);
    Ainv.clear();
    switch (kind) {
        case CPG_STEP_BACKWARD_EULER:
            s = 1;
            A = {1.0};
            b = {1.0};
            c = {1.0};
            break;
        case CPG_STEP_DIRK3: {  // TimeIntegration.cpp:70-77
            const double alpha = 0.435866521508459;
            s = 3;
            A = {(1 + alpha) / 2.0, 0, 0, -alpha / 2.0, (1 + alpha) / 2.0, 0, 1 + alpha, -(1 + 2 * alpha),
                 (1 + alpha) / 2.0};
            b = {1.0 / 6.0 / (alpha * alpha), 1 - 1.0 / 3.0 / (alpha * alpha), 1.0 / 6.0 / (alpha * alpha)};
            c = {(1 + alpha) / 2.0, 1.0 / 2.0, (1 - alpha) / 2.0};
            break;
        }
        case CPG_STEP_SDIRK3: {
            // Alexander's L-stable SDIRK of order 3 (SIAM J. Numer. Anal. 14,
            // 1977): gamma solves g^3 - 3g^2 + 3g/2 - 1/6 = 0 in (1/6, 1/2);
            // the last row of A is b
            const double g = 0.435866521508459, t2 = (1 + g) / 2.0;
            const double b1 = -(6 * g * g - 16 * g + 1) / 4.0, b2 = (6 * g * g - 20 * g + 5) / 4.0;
            s = 3;
            A = {g, 0, 0, t2 - g, g, 0, b1, b2, g};
            b = {b1, b2, g};
            c = {g, t2, 1.0};
            break;
        }
        case CPG_STEP_DIRK5: {  // Cooper and Sayfy, TimeIntegration.cpp:78-88
            const double g = (6 - r6) / 10.0;
            s = 5;
            A = {g, 0, 0, 0, 0,
                 (-6 + 5 * r6) / 14.0, g, 0, 0, 0,
                 (888 + 607 * r6) / 2850.0, (126 - 161 * r6) / 1425.0, g, 0, 0,
                 (3153 - 3082 * r6) / 14250.0, (3213 + 1148 * r6) / 28500.0, (-267 + 88 * r6) / 500.0, g, 0,
                 (-32583 + 14638 * r6) / 71250.0, (-17199 + 364 * r6) / 142500.0, (1329 - 544 * r6) / 2500.0,
                 (-96 + 131 * r6) / 625.0, g};
            b = {0, 0, 1 / 9.0, (16 - r6) / 36.0, (16 + r6) / 36.0};
            c = {g, (6 + 9 * r6) / 35.0, 1, (4 - r6) / 10.0, (4 + r6) / 10.0};
            break;
        }
        case CPG_STEP_IRK2:
        case CPG_STEP_IRK2_INV:  // TimeIntegration.cpp:155-161
            s = 2;
            A = {5 / 12.0, -1 / 12.0, 3 / 4.0, 1 / 4.0};
            Ainv = {3 / 2.0, 1 / 2.0, -9 / 2.0, 5 / 2.0};
            b = {3 / 4.0, 1 / 4.0};
            c = {1 / 3.0, 1};
            break;
        default: {  // IRK3, TimeIntegration.cpp:163-184
            s = 3;
            A = {(88 - 7 * r6) / 360.0, (296 - 169 * r6) / 1800.0, (-2 + 3 * r6) / 225.0,
                 (296 + 169 * r6) / 1800.0, (88 + 7 * r6) / 360.0, (-2 - 3 * r6) / 225.0,
                 (16 - r6) / 36.0, (16 + r6) / 36.0, 1 / 9.0};
            Ainv = {60 * (1 / 30.0 + 1.0 / (20 * r6)), 60 * (-1 / 50.0 + 29.0 / (300 * r6)),
                    60 * (1 / 150.0 - std::sqrt(2 / 3.0) / 75.0),
                    60 * (-1 / 50.0 - 29.0 / (300 * r6)), 60 * (1 / 30.0 - 1.0 / (20 * r6)),
                    60.0 * (1 / 150.0 + std::sqrt(2 / 3.0) / 75.0),
                    60 * (-1 / 60.0 + (2 * std::sqrt(2 / 3.0)) / 15.0),
                    60 * (-1 / 60.0 - (2 * std::sqrt(2 / 3.0)) / 15.0), 5};
            b = {(16 - r6) / 36.0, (16 + r6) / 36.0, 1 / 9.0};
            c = {(4 - r6) / 10.0, (4 + r6) / 10.0, 1};
        }
    }
}

bool is_irk(int kind) { return kind >= CPG_STEP_IRK2 && kind <= CPG_STEP_IRK3_INV; }
bool is_inv(int kind) { return kind == CPG_STEP_IRK2_INV || kind == CPG_STEP_IRK3_INV; }

}  // namespace

struct cpg_stepper {
    cpg_ctx *ctx = nullptr;
    cpg_equation *eq = nullptr;
    cpg_stepper_desc d{};
    int s = 0;
    std::vector<double> A, Ainv, b, c;
    int64_t N = 0;
    double *work = nullptr;  // device work vectors
    double *k = nullptr, *cu = nullptr, *rhs = nullptr, *r = nullptr, *dk = nullptr, *w = nullptr, *big = nullptr,
           *big2 = nullptr, *tmp = nullptr;
    // DIRK / BE
    cpg_bsr *J = nullptr;
    cpg_precond *P = nullptr;
    // IRK
    void *Jstack = nullptr;                 // s * nnzb blocks
    std::vector<cpg_bsr *> Jview;           // per-stage views into Jstack
    cpg_bsr *full = nullptr, *fullpc = nullptr;  // coupled stage-major matrices
    int *map_src = nullptr, *map_mrow = nullptr, *pmap_src = nullptr, *pmap_mrow = nullptr;
    double *map_s1 = nullptr, *map_s2 = nullptr, *map_mc = nullptr, *pmap_s1 = nullptr, *pmap_s2 = nullptr,
           *pmap_mc = nullptr;
    cpg_bsr *stage_blocks = nullptr;        // CPG_PC_STAGE_BJACOBI blocks
    double *Acoef_d = nullptr;
    double *udev = nullptr;                 // device copy for cpg_step_host
    // explicit steps replayed as a CUDA graph (keyed on the field and dt)
    cudaGraphExec_t gexec = nullptr;
    const double *g_u = nullptr;
    double g_dt = 0.0;
    uint64_t g_launches = 0;
    bool g_off = false;
};

namespace {

void free_stepper(cpg_stepper *S) {
    if (S->J) cpg_bsr_destroy(S->J);
    if (S->P) cpg_precond_destroy(S->P);
    if (S->full) cpg_bsr_destroy(S->full);
    if (S->fullpc) cpg_bsr_destroy(S->fullpc);
    if (S->stage_blocks) cpg_bsr_destroy(S->stage_blocks);
    for (cpg_bsr *v : S->Jview) {
        v->vals = nullptr;  // views do not own storage
        v->rowptr_d = v->colidx_d = nullptr;
        delete v;
    }
    if (S->gexec) cudaGraphExecDestroy(S->gexec);
    void *ptrs[] = {S->work, S->Jstack, S->map_src, S->map_mrow, S->pmap_src, S->pmap_mrow, S->map_s1, S->map_s2,
                    S->map_mc, S->pmap_s1, S->pmap_s2, S->pmap_mc, S->Acoef_d, S->udev};
    for (void *p : ptrs) dfree(p);
}

// build the stage-major coupled matrix pattern and gather map
// (newAdvance: off-diagonal stage pairs hold mass blocks only; the
// preconditioner matrix holds stage-diagonal pairs only)
cpg_status build_coupled(cpg_stepper *S, bool inverted, bool pc_only, cpg_bsr **out, int **m_src, int **m_mrow,
                         double **m_s1, double **m_s2, double **m_mc) {
    cpg_ctx *ctx = S->ctx;
    const cpg_equation *eq = S->eq;
    const int n = eq->n, s = S->s;
    const int64_t nnzb = (int64_t)eq->colidx.size();
    std::vector<int> rowptr(1, 0), col, src, mrow;
    std::vector<double> s1, s2, mc;
    for (int i = 0; i < s; i++)
        for (int r = 0; r < n; r++) {
            for (int j = 0; j < s; j++) {
                if (pc_only && j != i) continue;
                const bool jblocks = !inverted || i == j;
                if (jblocks) {
                    for (int k = eq->rowptr[r]; k < eq->rowptr[r + 1]; k++) {
                        col.push_back(j * n + eq->colidx[k]);
                        src.push_back((int)(i * nnzb + k));
                        const bool dg = (i == j) && eq->colidx[k] == r;
                        mrow.push_back(dg ? r : -1);
                        if (!inverted) {
                            s1.push_back(0.0);  // filled per step (-dt)
                            s2.push_back(S->A[i * s + j]);
                            mc.push_back(1.0);
                        } else {
                            s1.push_back(0.0);
                            s2.push_back(1.0);
                            mc.push_back(S->Ainv[i * s + i]);
                        }
                    }
                } else {
                    col.push_back(j * n + r);
                    src.push_back(-1);
                    mrow.push_back(r);
                    s1.push_back(0.0);
                    s2.push_back(0.0);
                    mc.push_back(S->Ainv[i * s + j]);
                }
            }
            rowptr.push_back((int)col.size());
        }
    cpg_bsr *B = nullptr;
    CPG_TRY(cpg_bsr_create_host(ctx, n * s, eq->bl, rowptr.data(), col.data(), nullptr, S->d.matrix_precision, &B));
    *out = B;
    CPG_TRY(upload(ctx, m_src, src));
    CPG_TRY(upload(ctx, m_mrow, mrow));
    CPG_TRY(upload(ctx, m_s1, s1));
    CPG_TRY(upload(ctx, m_s2, s2));
    CPG_TRY(upload(ctx, m_mc, mc));
    return CPG_OK;
}

cpg_status fill_coupled(cpg_stepper *S, cpg_bsr *B, int *src, int *mrow, double *s1, double *s2, double *mc,
                        double dt) {
    cpg_ctx *ctx = S->ctx;
    // s1 = -dt for every J-sourced block
    std::vector<double> h(B->nnzb, -dt);
    CPG_CUDA(ctx, cudaMemcpyAsync(s1, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, ctx->stream));
    CoupledMap mp{src, s1, s2, mc, mrow};
    const int grid = (int)std::min<int64_t>(B->nnzb, (int64_t)ctx->num_sms * 32);
    if (B->precision == CPG_F32)
        k_build_coupled<float><<<grid, 256, 0, ctx->stream>>>(B->nnzb, S->eq->nb, S->eq->nc, mp,
                                                              (const float *)S->Jstack, S->eq->mass, (float *)B->vals);
    else
        k_build_coupled<double><<<grid, 256, 0, ctx->stream>>>(B->nnzb, S->eq->nb, S->eq->nc, mp,
                                                               (const double *)S->Jstack, S->eq->mass,
                                                               (double *)B->vals);
    bsr_touch(B);
    CPG_TRY(launched(ctx, "coupled matrix kernel"));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // h is pageable and short-lived
    return CPG_OK;
}

// Kronecker-form stage operator: y_i = M x_i - dt J_i (sum_j A_ij x_j),
// preconditioned by the cell-coupled stage blocks
struct StageOp : LinOp {
    cpg_stepper *S;
    double dt;
    cpg_status apply(cpg_ctx *ctx, const double *x, double *y) const override {
        const int s = S->s;
        const int64_t N = S->N;
        for (int i = 0; i < s; i++) {
            Comb cb{};
            cb.nk = s;
            for (int j = 0; j < s; j++) {
                cb.k[j] = x + j * N;
                cb.a[j] = S->A[i * s + j];
            }
            k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, nullptr, cb, S->tmp, ctx->skip_dev);
            CPG_TRY(launched(ctx, "stage combine kernel"));
            CPG_TRY(bsr_matvec_raw(ctx, S->Jview[i], S->tmp, S->dk));
            CPG_TRY(mass_apply_axpy(ctx, S->eq, x + i * N, 1.0, S->dk, -dt, y + i * N));
        }
        return CPG_OK;
    }
    cpg_status prec(cpg_ctx *ctx, double *x) const override {
        const int n = S->eq->n, s = S->s, bl = S->eq->bl;
        const int64_t NS = S->N * s;
        k_stage_perm<<<grid_for(ctx, NS), 256, 0, ctx->stream>>>(n, s, bl, x, S->big2, 1, ctx->skip_dev);
        CPG_TRY(launched(ctx, "stage permute kernel"));
        CPG_TRY(precond_apply_raw(ctx, S->P, S->big2));
        k_stage_perm<<<grid_for(ctx, NS), 256, 0, ctx->stream>>>(n, s, bl, S->big2, x, 0, ctx->skip_dev);
        return launched(ctx, "stage permute kernel");
    }
};

// storage precision of the preconditioner's factors
int pc_precision(const cpg_stepper *S) { return S->d.pc_f32 ? CPG_F32 : S->d.matrix_precision; }

cpg_status newton_norm(cpg_stepper *S, const double *r, double *out) {
    double l2[4];
    CPG_TRY(cpg_l2norm(S->ctx, S->eq, r, l2));
    double mx = l2[0];
    for (int c = 1; c < S->eq->nc; c++) mx = std::max(mx, l2[c]);
    *out = mx;
    return CPG_OK;
}

// k = dt * M^{-1} assemble(u, t)
cpg_status rk_stage(cpg_stepper *S, const double *u, double t, double dt, double *k) {
    CPG_TRY(assemble_raw(S->ctx, S->eq, u, t, S->rhs));
    return mass_solve_scaled(S->ctx, S->eq, S->rhs, dt, k);
}

cpg_status combine(cpg_stepper *S, const double *u, std::initializer_list<std::pair<const double *, double>> terms,
                   double *out) {
    Comb cb{};
    cb.nk = 0;
    for (auto &t : terms) {
        cb.k[cb.nk] = t.first;
        cb.a[cb.nk] = t.second;
        cb.nk++;
    }
    k_combine<<<grid_for(S->ctx, S->N), 256, 0, S->ctx->stream>>>(S->N, u, cb, out, S->ctx->skip_dev);
    return launched(S->ctx, "combine kernel");
}

cpg_status explicit_step(cpg_stepper *S, double *u, double dt, double t) {
    cpg_ctx *ctx = S->ctx;
    const int64_t N = S->N;
    double *k1 = S->k, *k2 = S->k + N, *k3 = S->k + 2 * N, *k4 = S->k + 3 * N;
    if (S->d.kind == CPG_STEP_FORWARD_EULER) {  // TimeIntegration.cpp:10-12
        CPG_TRY(rk_stage(S, u, t, dt, k1));
        return combine(S, u, {{k1, 1.0}}, u);
    }
    if (S->d.kind == CPG_STEP_RK2) {  // :24-29
        CPG_TRY(rk_stage(S, u, t, dt, k1));
        CPG_TRY(combine(S, u, {{k1, 0.5}}, S->cu));
        CPG_TRY(rk_stage(S, S->cu, t + 0.5 * dt, dt, k2));
        k_rk2_final<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, k1, k2, u);
        return launched(ctx, "rk2 kernel");
    }
    // RK4 :14-22
    CPG_TRY(rk_stage(S, u, t, dt, k1));
    CPG_TRY(combine(S, u, {{k1, 0.5}}, S->cu));
    CPG_TRY(rk_stage(S, S->cu, t + 0.5 * dt, dt, k2));
    CPG_TRY(combine(S, u, {{k2, 0.5}}, S->cu));
    CPG_TRY(rk_stage(S, S->cu, t + 0.5 * dt, dt, k3));
    CPG_TRY(combine(S, u, {{k3, 1.0}}, S->cu));
    CPG_TRY(rk_stage(S, S->cu, t + dt, dt, k4));
    k_rk4_final<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, k1, k2, k3, k4, u);
    return launched(ctx, "rk4 kernel");
}

// An explicit step is a fixed sequence of kernel launches with no host
// synchronisation, so it is captured once as a CUDA graph and replayed: one
// launch per step instead of 13 (RK4), which is what small meshes in a
// serving mix pay for.  The graph bakes in the field pointer, dt and the
// stage times, so it is used only when no face reads a time-dependent
// boundary field, on a context with its own stream, and is re-captured when
// the field or dt changes.  CPG_GRAPHS=0 turns it off.
cpg_status explicit_step_graph(cpg_stepper *S, double *u, double dt, double t) {
    cpg_ctx *ctx = S->ctx;
    static const bool off_env = [] {
        const char *e = std::getenv("CPG_GRAPHS");
        return e && std::strcmp(e, "0") == 0;
    }();
    if (S->g_off || off_env || ctx->stream == nullptr || S->eq->time_dependent_bc) return explicit_step(S, u, dt, t);
    if (!S->gexec || S->g_u != u || S->g_dt != dt) {
        if (S->gexec) {
            cudaGraphExecDestroy(S->gexec);
            S->gexec = nullptr;
        }
        const uint64_t before = ctx->launches;
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            (void)cudaGetLastError();
            S->g_off = true;
            return explicit_step(S, u, dt, t);
        }
        const cpg_status st = explicit_step(S, u, dt, t);
        const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
        const bool ok = st == CPG_OK && ec == cudaSuccess && graph &&
                        cudaGraphInstantiate(&S->gexec, graph, 0) == cudaSuccess;
        if (graph) cudaGraphDestroy(graph);
        const uint64_t captured = ctx->launches - before;  // kernels the graph holds
        ctx->launches = before;
        if (!ok) {  // capture refused: run this and later steps directly
            (void)cudaGetLastError();
            S->gexec = nullptr;
            S->g_off = true;
            return explicit_step(S, u, dt, t);
        }
        S->g_launches = captured;
        S->g_u = u;
        S->g_dt = dt;
    }
    CPG_CUDA(ctx, cudaGraphLaunch(S->gexec, ctx->stream));
    ctx->launches += S->g_launches;
    return CPG_OK;
}

// DIRK::advance (TimeIntegration.cpp:93-151); BackwardEuler is the one-stage
// tableau (:31-66)
cpg_status dirk_step(cpg_stepper *S, double *u, double dt, double t, cpg_step_stats *st) {
    cpg_ctx *ctx = S->ctx;
    const int64_t N = S->N;
    const int s = S->s;
    CPG_TRY(vec_fill(ctx, N * s, 0.0, S->k));
    st->converged = 1;
    for (int stage = 0; stage < s; stage++) {
        double *ks = S->k + stage * N;
        const double ts = t + dt * S->c[stage];
        int iter;
        int since_build = 0;
        double upd_rel = INFINITY;  // last Newton update relative to the stage vector
        for (iter = 0; iter < S->d.newton_maxit; iter++) {
            Comb cb{};
            cb.nk = stage + 1;
            for (int j = 0; j <= stage; j++) {
                cb.k[j] = S->k + j * N;
                cb.a[j] = S->A[stage * s + j];
            }
            k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, u, cb, S->cu, ctx->skip_dev);
            CPG_TRY(launched(ctx, "stage combine kernel"));
            CPG_TRY(assemble_raw(ctx, S->eq, S->cu, ts, S->rhs));
            CPG_TRY(mass_apply_axpy(ctx, S->eq, ks, 1.0, S->rhs, -dt, S->r));  // r = M k - dt rhs
            double nr;
            // a non-physical state names its cell before its NaN norm fails
            const cpg_status ns = newton_norm(S, S->r, &nr);
            CPG_TRY(check_state(ctx, "DIRK stage " + std::to_string(stage) + ", Newton iteration " +
                                         std::to_string(iter) + ", t = " + std::to_string(ts)));
            CPG_TRY(ns);
            st->last_newton_residual = nr;
            if (nr < S->d.newton_tol && (S->d.newton_rtol <= 0 || upd_rel < S->d.newton_rtol)) break;
            st->newton_iterations++;
            const bool rebuild = S->d.reuse_jacobian <= 0 || iter == 0 || since_build >= S->d.reuse_jacobian;
            if (rebuild) {
                CPG_TRY(cpg_jacobian(ctx, S->eq, S->cu, ts, -dt * S->A[stage * s + stage], 1, S->J));
                if (S->P) {
                    CPG_TRY(cpg_precond_refactor(ctx, S->P, S->J));
                } else {
                    CPG_TRY(cpg_precond_create(ctx, S->J, S->d.pc_kind, pc_precision(S), &S->P));
                }
                since_build = 0;
            }
            since_build++;
            CPG_TRY(vec_fill(ctx, N, 0.0, S->dk));
            cpg_solve_stats ls{};
            CPG_TRY(cpg_gmres(ctx, S->J, S->P, S->r, S->dk, S->d.gmres_m, S->d.gmres_tol, S->d.gmres_maxit,
                              S->d.flexible, &ls));
            st->gmres_iterations += ls.iterations;
            st->linear_solves++;
            CPG_TRY(vec_axpby(ctx, N, -1.0, S->dk, 1.0, ks));  // k -= dk
            if (S->d.newton_rtol > 0) {
                double nd, nk;
                CPG_TRY(newton_norm(S, S->dk, &nd));
                CPG_TRY(newton_norm(S, ks, &nk));
                upd_rel = nk > 0 ? nd / nk : 0.0;
            }
        }
        if (iter == S->d.newton_maxit) st->converged = 0;
    }
    Comb cb{};
    cb.nk = s;
    for (int i = 0; i < s; i++) {
        cb.k[i] = S->k + i * N;
        cb.a[i] = S->b[i];
    }
    k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, u, cb, u, ctx->skip_dev);
    return launched(ctx, "stage combine kernel");
}

// IRK::advance (:188-281) and IRK::newAdvance (:283-395)
cpg_status irk_step(cpg_stepper *S, double *u, double dt, double t, cpg_step_stats *st) {
    cpg_ctx *ctx = S->ctx;
    const int64_t N = S->N;
    const int s = S->s;
    const bool inv = is_inv(S->d.kind);
    const bool kron = S->d.pc_kind == CPG_PC_STAGE_BJACOBI;
    double *K = S->k;      // k (advance) or w (newAdvance), stage-major s*N
    double *R = S->big;    // stacked residual
    double *sol = S->w;    // bigK / bigU, kept across Newton iterations
    CPG_TRY(vec_fill(ctx, N * s, 0.0, K));
    CPG_TRY(vec_fill(ctx, N * s, 0.0, sol));
    st->converged = 1;
    int iter;
    double upd_rel = INFINITY;  // last Newton update relative to the stage vectors
    for (iter = 0; iter < S->d.newton_maxit; iter++) {
        double rNorm = 0.0;
        if (inv) {
            // k_i = sum_j Ainv(i,j) w_j  (into S->dk-sized temporaries of R)
            for (int i = 0; i < s; i++) {
                Comb cb{};
                cb.nk = s;
                for (int j = 0; j < s; j++) {
                    cb.k[j] = K + j * N;
                    cb.a[j] = S->Ainv[i * s + j];
                }
                k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, nullptr, cb, S->tmp, ctx->skip_dev);
                CPG_TRY(launched(ctx, "stage combine kernel"));
                CPG_TRY(combine(S, u, {{K + i * N, 1.0}}, S->cu));  // u + w_i
                CPG_TRY(assemble_raw(ctx, S->eq, S->cu, t + dt * S->c[i], S->rhs));
                CPG_TRY(mass_apply_axpy(ctx, S->eq, S->tmp, 1.0, S->rhs, -dt, R + i * N));
                double nr;
                const cpg_status ns = newton_norm(S, R + i * N, &nr);
                CPG_TRY(check_state(ctx, "implicit RK stage " + std::to_string(i) + ", Newton iteration " +
                                             std::to_string(iter) + ", t = " + std::to_string(t)));
                CPG_TRY(ns);
                rNorm += nr * nr;
            }
        } else {
            for (int i = 0; i < s; i++) {
                Comb cb{};
                cb.nk = s;
                for (int j = 0; j < s; j++) {
                    cb.k[j] = K + j * N;
                    cb.a[j] = S->A[i * s + j];
                }
                k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, u, cb, S->cu, ctx->skip_dev);
                CPG_TRY(launched(ctx, "stage combine kernel"));
                CPG_TRY(assemble_raw(ctx, S->eq, S->cu, t + dt * S->c[i], S->rhs));
                CPG_TRY(mass_apply_axpy(ctx, S->eq, K + i * N, 1.0, S->rhs, -dt, R + i * N));
                double nr;
                const cpg_status ns = newton_norm(S, R + i * N, &nr);
                CPG_TRY(check_state(ctx, "implicit RK stage " + std::to_string(i) + ", Newton iteration " +
                                             std::to_string(iter) + ", t = " + std::to_string(t)));
                CPG_TRY(ns);
                rNorm += nr * nr;
            }
        }
        rNorm = std::sqrt(rNorm);
        st->last_newton_residual = rNorm;
        if (rNorm < S->d.newton_tol && (S->d.newton_rtol <= 0 || upd_rel < S->d.newton_rtol)) break;
        st->newton_iterations++;
        // modified Newton: with reuse_jacobian = r > 0 the stage Jacobians,
        // the coupled matrix and its factorisation are rebuilt every r-th
        // iteration only (the reference rebuilds every iteration)
        const bool rebuild = S->d.reuse_jacobian <= 0 || iter == 0 || iter % S->d.reuse_jacobian == 0;
        // stage Jacobians at the stage states
        for (int i = 0; i < s && rebuild; i++) {
            if (inv) CPG_TRY(combine(S, u, {{K + i * N, 1.0}}, S->cu));
            else {
                Comb cb{};
                cb.nk = s;
                for (int j = 0; j < s; j++) {
                    cb.k[j] = K + j * N;
                    cb.a[j] = S->A[i * s + j];
                }
                k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, u, cb, S->cu, ctx->skip_dev);
                CPG_TRY(launched(ctx, "stage combine kernel"));
            }
            CPG_TRY(cpg_jacobian(ctx, S->eq, S->cu, t + dt * S->c[i], 1.0, 0, S->Jview[i]));
        }
        cpg_solve_stats ls{};
        if (kron && rebuild) {
            const int grid = S->eq->n;
            const int64_t nnzb = (int64_t)S->eq->colidx.size();
            if (S->d.matrix_precision == CPG_F32)
                k_build_stage_blocks<float><<<grid, 256, 0, ctx->stream>>>(
                    S->eq->n, s, S->eq->nb, S->eq->nc, (const float *)S->Jstack, nnzb, S->eq->rowptr_d, S->Acoef_d, dt,
                    S->eq->mass, (float *)S->stage_blocks->vals);
            else
                k_build_stage_blocks<double><<<grid, 256, 0, ctx->stream>>>(
                    S->eq->n, s, S->eq->nb, S->eq->nc, (const double *)S->Jstack, nnzb, S->eq->rowptr_d,
                    S->Acoef_d, dt, S->eq->mass, (double *)S->stage_blocks->vals);
            bsr_touch(S->stage_blocks);
            CPG_TRY(launched(ctx, "stage block kernel"));
            if (S->P) CPG_TRY(cpg_precond_refactor(ctx, S->P, S->stage_blocks));
            else CPG_TRY(cpg_precond_create(ctx, S->stage_blocks, CPG_PC_BJACOBI, pc_precision(S), &S->P));
        } else if (!kron && rebuild) {
            CPG_TRY(fill_coupled(S, S->full, S->map_src, S->map_mrow, S->map_s1, S->map_s2, S->map_mc, dt));
            cpg_bsr *pcm = S->full;
            if (inv) {
                CPG_TRY(fill_coupled(S, S->fullpc, S->pmap_src, S->pmap_mrow, S->pmap_s1, S->pmap_s2, S->pmap_mc, dt));
                pcm = S->fullpc;
            }
            if (S->P) CPG_TRY(cpg_precond_refactor(ctx, S->P, pcm));
            else CPG_TRY(cpg_precond_create(ctx, pcm, S->d.pc_kind, pc_precision(S), &S->P));
        }
        if (kron) {
            StageOp op;
            op.S = S;
            op.dt = dt;
            CPG_TRY(gmres_op(ctx, op, N * s, R, sol, S->d.gmres_m, S->d.gmres_tol, S->d.gmres_maxit, S->d.flexible,
                             &ls));
        } else {
            CPG_TRY(cpg_gmres(ctx, S->full, S->P, R, sol, S->d.gmres_m, S->d.gmres_tol, S->d.gmres_maxit,
                              S->d.flexible, &ls));
        }
        st->gmres_iterations += ls.iterations;
        st->linear_solves++;
        CPG_TRY(vec_axpby(ctx, N * s, -1.0, sol, 1.0, K));  // k (or w) -= solution
        if (S->d.newton_rtol > 0) {
            double nd2 = 0.0, nk2 = 0.0;
            for (int i = 0; i < s; i++) {
                double nd, nk;
                CPG_TRY(newton_norm(S, sol + i * N, &nd));
                CPG_TRY(newton_norm(S, K + i * N, &nk));
                nd2 += nd * nd;
                nk2 += nk * nk;
            }
            upd_rel = nk2 > 0 ? std::sqrt(nd2 / nk2) : 0.0;
        }
    }
    if (iter == S->d.newton_maxit) st->converged = 0;
    Comb cb{};
    cb.nk = s;
    for (int i = 0; i < s; i++) {
        cb.k[i] = K + i * N;
        if (inv) {  // b^T Ainv
            double bt = 0;
            for (int j = 0; j < s; j++) bt += S->b[j] * S->Ainv[j * s + i];
            cb.a[i] = bt;
        } else {
            cb.a[i] = S->b[i];
        }
    }
    k_combine<<<grid_for(ctx, N), 256, 0, ctx->stream>>>(N, u, cb, u, ctx->skip_dev);
    return launched(ctx, "stage combine kernel");
}

}  // namespace

extern "C" {

cpg_status cpg_stepper_create(cpg_ctx *ctx, cpg_equation *eq, const cpg_stepper_desc *d, cpg_stepper **out) {
    if (!ctx || !eq || !d || !out) return CPG_ERR_INVALID_ARG;
    if (d->kind < CPG_STEP_FORWARD_EULER || d->kind > CPG_STEP_SDIRK3)
        return fail(ctx, CPG_ERR_INVALID_ARG, "unknown stepper kind");
    *out = nullptr;
    cpg_stepper *S = new (std::nothrow) cpg_stepper();
    if (!S) return fail(ctx, CPG_ERR_OOM, "host allocation");
    S->ctx = ctx;
    S->eq = eq;
    S->d = *d;
    if (S->d.gmres_m <= 0) S->d.gmres_m = 20;
    if (S->d.gmres_tol <= 0) S->d.gmres_tol = 1e-14;
    if (S->d.gmres_maxit <= 0) S->d.gmres_maxit = is_irk(d->kind) ? 20000 : 90000;
    if (S->d.newton_tol <= 0) S->d.newton_tol = 5e-13;
    if (S->d.newton_maxit <= 0) S->d.newton_maxit = 100;
    S->N = (int64_t)eq->n * eq->bl;
    const bool implicit = d->kind >= CPG_STEP_BACKWARD_EULER;
    if (implicit) tableau(d->kind, S->s, S->A, S->Ainv, S->b, S->c);
    if (d->pc_kind == CPG_PC_STAGE_BJACOBI && !is_irk(d->kind)) {
        delete S;
        return fail(ctx, CPG_ERR_INVALID_ARG, "stage block Jacobi is for implicit RK (IRK) steppers");
    }
    const int64_t N = S->N;
    const int s = std::max(S->s, 1);
    // work: k (max(4, s) N) | cu | rhs | r | dk | tmp | w (s N) | big (s N) | big2 (s N)
    const int nk = std::max(4, s);
    const int64_t words = N * (nk + 5) + (is_irk(d->kind) ? 3 * N * s : 0);
    cpg_status st = dmalloc(ctx, &S->work, (size_t)words);
    if (st == CPG_OK) {
        double *p = S->work;
        S->k = p;
        p += N * nk;
        S->cu = p;
        p += N;
        S->rhs = p;
        p += N;
        S->r = p;
        p += N;
        S->dk = p;
        p += N;
        S->tmp = p;
        p += N;
        if (is_irk(d->kind)) {
            S->w = p;
            p += N * s;
            S->big = p;
            p += N * s;
            S->big2 = p;
            p += N * s;
        }
    }
    if (st == CPG_OK && implicit && !is_irk(d->kind)) st = cpg_bsr_create(ctx, eq, d->matrix_precision, &S->J);
    if (st == CPG_OK && is_irk(d->kind)) {
        const int64_t nnzb = (int64_t)eq->colidx.size();
        const size_t elem = d->matrix_precision == CPG_F32 ? sizeof(float) : sizeof(double);
        const size_t bytes = (size_t)s * nnzb * eq->bl * eq->bl * elem;
        if (cudaMalloc(&S->Jstack, bytes) != cudaSuccess) {
            (void)cudaGetLastError();
            S->Jstack = nullptr;
            st = fail(ctx, CPG_ERR_OOM, "stage Jacobians: " + std::to_string(bytes) + " bytes");
        }
        for (int i = 0; st == CPG_OK && i < s; i++) {
            cpg_bsr *v = new cpg_bsr();
            v->ctx = ctx;
            v->n_rows = eq->n;
            v->bl = eq->bl;
            v->precision = d->matrix_precision;
            v->nnzb = nnzb;
            v->rowptr = eq->rowptr;
            v->colidx = eq->colidx;
            v->rowptr_d = eq->rowptr_d;
            v->colidx_d = eq->colidx_d;
            v->owns_pattern = false;
            v->vals = (char *)S->Jstack + (size_t)i * nnzb * eq->bl * eq->bl * elem;
            S->Jview.push_back(v);
        }
        if (st == CPG_OK && d->pc_kind == CPG_PC_STAGE_BJACOBI) {
            std::vector<int> rp(eq->n + 1), cl(eq->n);
            for (int i = 0; i <= eq->n; i++) rp[i] = i;
            for (int i = 0; i < eq->n; i++) cl[i] = i;
            st = cpg_bsr_create_host(ctx, eq->n, s * eq->bl, rp.data(), cl.data(), nullptr, d->matrix_precision,
                                     &S->stage_blocks);
            if (st == CPG_OK) st = upload(ctx, &S->Acoef_d, S->A);
        } else if (st == CPG_OK) {
            const bool inv = is_inv(d->kind);
            st = build_coupled(S, inv, false, &S->full, &S->map_src, &S->map_mrow, &S->map_s1, &S->map_s2,
                               &S->map_mc);
            if (st == CPG_OK && inv)
                st = build_coupled(S, inv, true, &S->fullpc, &S->pmap_src, &S->pmap_mrow, &S->pmap_s1, &S->pmap_s2,
                                   &S->pmap_mc);
        }
    }
    if (st != CPG_OK) {
        free_stepper(S);
        delete S;
        return st;
    }
    *out = S;
    return CPG_OK;
}

void cpg_stepper_destroy(cpg_stepper *S) {
    if (!S) return;
    // cudaFree synchronizes the device; the context may already be gone
    free_stepper(S);
    delete S;
}

cpg_status cpg_step(cpg_ctx *ctx, cpg_stepper *S, double *u, double dt, double t, cpg_step_stats *stats) {
    if (!ctx || !S || !u) return CPG_ERR_INVALID_ARG;
    cpg_step_stats st{};
    st.converged = 1;
    cpg_status rc;
    if (S->d.kind <= CPG_STEP_RK4) rc = explicit_step_graph(S, u, dt, t);
    else if (is_irk(S->d.kind)) rc = irk_step(S, u, dt, t, &st);
    else rc = dirk_step(S, u, dt, t, &st);
    if (stats) *stats = st;
    if (rc != CPG_OK) return rc;
    if (!st.converged) return fail(ctx, CPG_ERR_NOT_CONVERGED, "Newton iteration limit reached");
    return CPG_OK;
}

cpg_status cpg_step_host(cpg_ctx *ctx, cpg_stepper *S, double *u_host, double dt, double t, cpg_step_stats *stats) {
    if (!ctx || !S || !u_host) return CPG_ERR_INVALID_ARG;
    if (!S->udev) CPG_TRY(dmalloc(ctx, &S->udev, (size_t)S->N));
    double *dev = S->udev;
    cpg_status rc = CPG_OK;
    cudaError_t e = cudaMemcpyAsync(dev, u_host, S->N * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "host to device copy");
    if (rc == CPG_OK) rc = cpg_step(ctx, S, dev, dt, t, stats);
    if (rc == CPG_OK || rc == CPG_ERR_NOT_CONVERGED) {
        e = cudaMemcpyAsync(u_host, dev, S->N * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "device to host copy");
    }
    cudaStreamSynchronize(ctx->stream);
    // explicit steps launch without a host check; the state word is read here
    if (rc == CPG_OK) rc = check_state(ctx, "step from t = " + std::to_string(t));
    return rc;
}

}  // extern "C"
