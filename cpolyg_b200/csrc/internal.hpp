// Internal object layouts shared by the translation units of the library.
#pragma once
#include <vector>

#include "common.cuh"
#include "mesh.hpp"
#include "physics.cuh"

const cpg::Mesh &cpg_mesh_ref(const cpg_mesh *m);

namespace cpg {

// device view of the quadrature geometry (structure of arrays)
struct Geo {
    int n;
    const double4 *bb;        // x0, y0, w, h
    const int *vq_ptr;        // n+1, volume qp range of each cell
    const double *vx, *vy, *vxi, *veta, *vw;
    const int *f_ptr;         // n+1, faces (= polygon edges) of each cell
    const int *f_nbr;         // neighbour cell or boundary code
    const int *f_blk;         // BSR block of the neighbour (or -1)
    const double *f_nx, *f_ny;
    const double *qx, *qy, *qxi, *qeta, *qxin, *qetan, *qw;  // face qp f*nqf+q
};

}  // namespace cpg

struct cpg_equation {
    cpg_ctx *ctx = nullptr;
    int physics = 0, degree = 1, nb = 3, nc = 1, bl = 3, n = 0, nqf = 2;
    double gamma = 1.4, beta[2] = {1, 1};
    cpg::BCParams bc{};
    int n_vqp = 0, n_faces = 0;
    // device geometry
    double4 *bb = nullptr;
    int *vq_ptr = nullptr, *f_ptr = nullptr, *f_nbr = nullptr, *f_blk = nullptr;
    double *vx = nullptr, *vy = nullptr, *vxi = nullptr, *veta = nullptr, *vw = nullptr;
    double *f_nx = nullptr, *f_ny = nullptr;
    double *qx = nullptr, *qy = nullptr, *qxi = nullptr, *qeta = nullptr, *qxin = nullptr, *qetan = nullptr,
           *qw = nullptr;
    double *mass = nullptr, *mass_inv = nullptr;  // n * nb * nb, column-major
    double *interp_pinv = nullptr;                // nb x (p+1)^2
    std::vector<double> gl_nodes;                 // p+1 ascending
    // Jacobian pattern (host and device)
    std::vector<int> rowptr, colidx;
    int *rowptr_d = nullptr, *colidx_d = nullptr;
    int levels_lower = 0, levels_upper = 0;
    int exact_jacobian = 0;
    int time_dependent_bc = 0;  // some face reads a boundary field at time t

    cpg::Geo geo() const {
        return cpg::Geo{n, bb, vq_ptr, vx, vy, vxi, veta, vw, f_ptr, f_nbr, f_blk, f_nx, f_ny,
                        qx, qy, qxi, qeta, qxin, qetan, qw};
    }
};

struct cpg_bsr {
    cpg_ctx *ctx = nullptr;
    int n_rows = 0, bl = 0, precision = CPG_F64;
    int64_t nnzb = 0;
    std::vector<int> rowptr, colidx;   // host copies of the pattern
    int *rowptr_d = nullptr, *colidx_d = nullptr;
    void *vals = nullptr;              // double or float, nnzb * bl * bl
    bool owns_pattern = true;
    // process-unique stamp of the values, renewed by every write through the
    // library (cpg::bsr_touch); a factorisation records the stamp it read
    uint64_t version = 0;
    size_t elem() const { return precision == CPG_F32 ? sizeof(float) : sizeof(double); }
};

struct cpg_precond {
    cpg_ctx *ctx = nullptr;
    int kind = CPG_PC_NONE, precision = CPG_F64, n = 0, bl = 0;
    // level schedule
    std::vector<int> lptr, lrows, uptr, urows;
    int *lrows_d = nullptr, *urows_d = nullptr;
    // strictly lower factor L (reference BlockILU0::L)
    std::vector<int> L_rowptr, L_col;
    int *L_rowptr_d = nullptr, *L_col_d = nullptr;
    void *L_vals = nullptr;
    // [D^{-1}_i, U_i*] rows (reference DD and DU, D^{-1} first)
    std::vector<int> U_rowptr, U_col;
    int *U_rowptr_d = nullptr, *U_col_d = nullptr;
    void *U_vals = nullptr;
    // FP64 pivot inverses used during factorisation
    double *dinv64 = nullptr;   // only for FP32 storage (FP64 storage reads U_vals)
    int *dinv_idx_d = nullptr;  // block index of D^{-1}_i in its FP64 array
    // per-row factor work lists (lower neighbours ascending):
    //   A block (j,i), A block (i,j), L block (j,i), U block (i,j)
    std::vector<int> lp_ptr;
    int *lp_ptr_d = nullptr, *lp_i_d = nullptr, *lp_aji_d = nullptr, *lp_aij_d = nullptr, *lp_l_d = nullptr, *lp_u_d = nullptr;
    int *diag_a_d = nullptr;    // A block index of (i,i)
    // sync-free sweeps (one launch per triangular solve): per-row publish
    // flags and the generation counter that makes earlier values stale
    bool syncfree = false;
    int *row_flags_d = nullptr;
    mutable int generation = 0;
    // triangular sweep form: 0 = not decided (the first application times
    // the candidates), 1 = sync-free with a TMA ring, 2 = level sweeps with
    // the sync-free forms' threads per row (bitwise the same result as 1 and
    // 4), 3 = level sweeps with the widest rows, 4 / 5 / 6 = sync-free with
    // direct loads and 1 / 2 / 4 times those threads per row
    mutable int sweep_mode = 2;
    double *tune_tmp = nullptr;  // scratch vector for timing the forms (undecided classes only)
    int n_cand = 0, cand[6] = {0, 0, 0, 0, 0, 0};
    int form_key = -1;  // process-wide key of the decision (block size, precision, size class)
    int64_t nnzL = 0, nnzU = 0;
    // split form of M^{-1} A (FP64 ILU(0) only): E_i = A_ii - Ahat_ii per
    // row, the A position of every upper block of a DU row (u2a, -1 at the
    // D^{-1} slot), and the matrix and value stamp the factors were built
    // from; the split form applies only to that matrix with that stamp
    double *E_vals = nullptr;
    int *u2a_d = nullptr;
    bool split_capable = false;
    const cpg_bsr *split_src = nullptr;
    uint64_t split_version = 0;
    // largest cond_inf of a pivot block in the last factorisation (device
    // word as the bits of a non-negative double, and its host copy)
    unsigned long long *cond_d = nullptr;
    double pivot_cond = 0.0;
    size_t elem() const { return precision == CPG_F32 ? sizeof(float) : sizeof(double); }
};

namespace cpg {
// linear operator + preconditioner seen by the Krylov solvers
struct LinOp {
    virtual cpg_status apply(cpg_ctx *ctx, const double *x, double *y) const = 0;  // y = A x
    virtual cpg_status prec(cpg_ctx *ctx, double *x) const = 0;                    // x = P^{-1} x
    // y = P^{-1} A x (x and y distinct)
    virtual cpg_status apply_prec(cpg_ctx *ctx, const double *x, double *y) const {
        const cpg_status st = apply(ctx, x, y);
        return st == CPG_OK ? prec(ctx, y) : st;
    }
    virtual ~LinOp() {}
};
// renews A's value stamp after a write to its values (bsr.cu)
void bsr_touch(cpg_bsr *A);
cpg_status gmres_op(cpg_ctx *ctx, const LinOp &op, int64_t N, const double *b, double *x, int m, double tol,
                    int maxit, int flexible, cpg_solve_stats *stats);
// residual kernel alone, without the state check of cpg_assemble (equation.cu)
cpg_status assemble_raw(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double t, double *b);
// mass helpers (equation.cu)
cpg_status mass_apply_axpy(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double alpha, const double *z,
                           double beta, double *y);
cpg_status mass_solve_scaled(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double alpha, double *y);
// launch helpers implemented in bsr.cu / krylov.cu and used across units
cpg_status bsr_matvec_raw(cpg_ctx *ctx, const cpg_bsr *A, const double *x, double *y);
// sync-free triangular sweep over the rows in `order` (bsr.cu)
// block-row kernel with an explicit threads-per-row variant (bsr.cu)
// addv (or null): added to every row's result of a backward sweep
cpg_status rows_op_v(cpg_ctx *ctx, int precision, int bl, int nrows, const int *rows, const int *rowptr,
                     const int *col, const void *vals, const double *x, double *y, int mode, int variant,
                     const double *addv = nullptr);
bool rows_tunable(int bl);
cpg_status sweep_op(cpg_ctx *ctx, int precision, int bl, int nrows, const int *order, const int *rowptr,
                    const int *col, const void *vals, double *x, int mode, int *flags, int gen, int *counter,
                    int *err, int kind = 0, const double *addv = nullptr);
// y_i = E_i x_i + sum_{j > i} A_ij x_j over the DU rows' columns, with the
// A positions u2a and the row blocks E (FP64 values; bsr.cu)
cpg_status split_rows_op(cpg_ctx *ctx, const cpg_bsr *A, const int *U_rowptr, const int *U_col, const int *u2a,
                         const double *E, const double *x, double *y);
bool sweep_supported(int bl);
constexpr int SWEEP_MAX_ROW_BLOCKS = 16;  // longest L or DU row the sync-free sweep takes
// x = P^{-1} x without the host-side check of the sweep status word, for
// callers that check once per solve (precond.cu)
cpg_status precond_apply_raw(cpg_ctx *ctx, const cpg_precond *P, double *x, const double *addv = nullptr);
// P is an FP64 ILU(0) factored from A's current values (precond.cu)
bool split_ready(const cpg_precond *P, const cpg_bsr *A);
// ... and the split form's rounding stays well below tol
bool split_allowed(const cpg_precond *P, const cpg_bsr *A, double tol);
// y = P^{-1} A x in split form (the caller checked split_allowed)
cpg_status split_apply_prec(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P, const double *x, double *y);
// reads and clears the sweep status word; a bounded wait that ran out turns
// `st` into CPG_ERR_TIMEOUT (precond.cu)
cpg_status check_sweep_error(cpg_ctx *ctx, cpg_status st);
cpg_status vec_axpby(cpg_ctx *ctx, int64_t n, double a, const double *x, double b, double *y);
cpg_status vec_copy(cpg_ctx *ctx, int64_t n, const double *x, double *y);
cpg_status vec_fill(cpg_ctx *ctx, int64_t n, double v, double *y);
// dot products / norms with deterministic reductions; results to host
cpg_status vec_dot(cpg_ctx *ctx, int64_t n, const double *x, const double *y, double *out_host);
}  // namespace cpg
