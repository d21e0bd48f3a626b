// cpolyg.hpp -- C++ interface with the reference's class names and call
// shapes (src/PolyMesh.h, src/Equation.h, src/MassMatrix.h,
// src/BlockMatrix.h, src/Jacobian.h, src/Preconditioners.h,
// src/TimeIntegration.h), header-only over the C ABI of cpolyg.h.
//
// Differences from the reference, all deliberate:
//   * MeshFn owns device memory (cudaMalloc) instead of an arma::cube; its
//     flat layout k + nb*c + bl*i is the reference's.
//   * Physics is selected by Equation's factory functions (Advection,
//     ConstantAdvection, Euler) instead of virtual overrides; the device
//     kernels are compiled per physics.
//   * Errors throw cpolyg::Error carrying the cpg_status.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cpolyg.h"

namespace cpolyg {

struct Error : std::runtime_error {
    cpg_status status;
    Error(cpg_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

inline void check(cpg_status s, const cpg_ctx *ctx = nullptr) {
    if (s != CPG_OK) throw Error(s, ctx ? cpg_last_error(ctx) : "cpolyg error");
}

// device context (one per host thread)
class Context {
  public:
    explicit Context(int device = 0, cudaStream_t stream = nullptr) { check(cpg_ctx_create(device, stream, &h_)); }
    ~Context() { cpg_ctx_destroy(h_); }
    Context(const Context &) = delete;
    Context &operator=(const Context &) = delete;
    cpg_ctx *get() const { return h_; }
    void check(cpg_status s) const { cpolyg::check(s, h_); }

  private:
    cpg_ctx *h_ = nullptr;
};

// PolyMesh (src/PolyMesh.h:13-55)
class PolyMesh {
  public:
    PolyMesh(std::vector<std::array<double, 2>> pts, double width = 1, double height = 1, bool periodic = false,
             const int *side_codes = nullptr) {
        check(cpg_mesh_voronoi(&pts[0][0], (int)pts.size(), width, height, periodic, side_codes, &h_));
        cpg_mesh_get_info(h_, &info_);
        np = info_.n_cells;
    }
    ~PolyMesh() { cpg_mesh_destroy(h_); }
    PolyMesh(const PolyMesh &) = delete;
    PolyMesh &operator=(const PolyMesh &) = delete;
    cpg_mesh *get() const { return h_; }
    int np = 0;

  private:
    cpg_mesh *h_ = nullptr;
    cpg_mesh_info info_{};
};

// MeshFn (src/MeshFn.h): coefficients of a field, device resident
class MeshFn {
  public:
    MeshFn() = default;
    MeshFn(const Context &ctx, int np, int deg, int nc) : ctx_(&ctx), np_(np), deg(deg), nc(nc) {
        n_ = (size_t)np * nc * (deg + 1) * (deg + 2) / 2;
        if (cudaMalloc(&d_, n_ * sizeof(double)) != cudaSuccess) throw Error(CPG_ERR_OOM, "MeshFn allocation");
        cudaMemset(d_, 0, n_ * sizeof(double));
    }
    MeshFn(const MeshFn &o) : MeshFn(*o.ctx_, o.np_, o.deg, o.nc) {
        cudaMemcpyAsync(d_, o.d_, n_ * sizeof(double), cudaMemcpyDeviceToDevice, stream());
    }
    MeshFn &operator=(MeshFn o) {
        swap(o);
        return *this;
    }
    ~MeshFn() {
        if (d_) cudaFree(d_);
    }
    void swap(MeshFn &o) {
        std::swap(ctx_, o.ctx_);
        std::swap(np_, o.np_);
        std::swap(deg, o.deg);
        std::swap(nc, o.nc);
        std::swap(n_, o.n_);
        std::swap(d_, o.d_);
    }
    double *data() const { return d_; }
    size_t size() const { return n_; }
    // MeshFn::operator+=, -=, *, + (MeshFn.cpp:209-247) on the device
    MeshFn &operator+=(const MeshFn &o) {
        ctx_->check(cpg_axpby(ctx_->get(), (int64_t)n_, 1.0, o.d_, 1.0, d_));
        return *this;
    }
    MeshFn &operator-=(const MeshFn &o) {
        ctx_->check(cpg_axpby(ctx_->get(), (int64_t)n_, -1.0, o.d_, 1.0, d_));
        return *this;
    }
    MeshFn operator*(double s) const {
        MeshFn r(*ctx_, np_, deg, nc);
        ctx_->check(cpg_axpby(ctx_->get(), (int64_t)n_, s, d_, 0.0, r.d_));
        return r;
    }
    MeshFn operator+(const MeshFn &o) const {
        MeshFn r(*this);
        r += o;
        return r;
    }
    MeshFn operator-(const MeshFn &o) const {
        MeshFn r(*this);
        r -= o;
        return r;
    }
    void upload(const std::vector<double> &h) {
        cudaMemcpyAsync(d_, h.data(), n_ * sizeof(double), cudaMemcpyHostToDevice, stream());
        cudaStreamSynchronize(stream());
    }
    std::vector<double> download() const {
        std::vector<double> h(n_);
        cudaMemcpyAsync(h.data(), d_, n_ * sizeof(double), cudaMemcpyDeviceToHost, stream());
        cudaStreamSynchronize(stream());
        return h;
    }
    const Context &context() const { return *ctx_; }
    int np() const { return np_; }
    int deg = 0, nc = 1;

  private:
    cudaStream_t stream() const { return nullptr; }
    const Context *ctx_ = nullptr;
    int np_ = 0;
    size_t n_ = 0;
    double *d_ = nullptr;
};

class Jacobian;

// BlockMatrix (src/BlockMatrix.h:10-77)
class BlockMatrix {
  public:
    BlockMatrix(const Context &ctx, cpg_bsr *h) : ctx_(&ctx), h_(h) {
        int64_t nnzb;
        cpg_bsr_get_info(h_, &n_rows, &bl, &nnzb, &precision);
        nb = (int)nnzb;
    }
    BlockMatrix(const Context &ctx, const std::vector<int> &rowBlock, const std::vector<int> &colIndices, int a_bl,
                const std::vector<double> &blocks, int prec = CPG_F64)
        : ctx_(&ctx) {
        ctx.check(cpg_bsr_create_host(ctx.get(), (int)rowBlock.size() - 1, a_bl, rowBlock.data(), colIndices.data(),
                                      blocks.empty() ? nullptr : blocks.data(), prec, &h_));
        int64_t nnzb;
        cpg_bsr_get_info(h_, &n_rows, &bl, &nnzb, &precision);
        nb = (int)nnzb;
    }
    virtual ~BlockMatrix() { cpg_bsr_destroy(h_); }
    BlockMatrix(const BlockMatrix &) = delete;
    BlockMatrix &operator=(const BlockMatrix &) = delete;

    // y = A x (BlockMatrix::matvec, out of place on the device)
    void matvec(const double *x_dev, double *y_dev) const { ctx_->check(cpg_bsr_matvec(ctx_->get(), h_, x_dev, y_dev)); }
    // BlockMatrix::gmres: tol and maxIt in/out as in the reference
    void gmres(const double *b_dev, double *x_dev, int m, double &tol, int &maxIt, const cpg_precond *pc,
               bool flexible = false) const {
        cpg_solve_stats st{};
        ctx_->check(cpg_gmres(ctx_->get(), h_, pc, b_dev, x_dev, m, tol, maxIt, flexible, &st));
        tol = st.residual;
        maxIt = st.iterations;
    }
    void jacobi(const double *b_dev, double *x_dev, double &tol, int &maxIt, const cpg_precond *pc) const {
        cpg_solve_stats st{};
        ctx_->check(cpg_jacobi_solve(ctx_->get(), h_, pc, b_dev, x_dev, tol, maxIt, &st));
        tol = st.residual;
        maxIt = st.iterations;
    }
    cpg_bsr *get() const { return h_; }
    int n_rows = 0, bl = 0, nb = 0, precision = CPG_F64;

  protected:
    const Context *ctx_;
    cpg_bsr *h_ = nullptr;
};

// Jacobian (src/Jacobian.h): the mesh-pattern BlockMatrix
class Jacobian : public BlockMatrix {
  public:
    using BlockMatrix::BlockMatrix;
};

// Preconditioner (src/Preconditioners.h:10-56)
class Preconditioner {
  public:
    virtual ~Preconditioner() { cpg_precond_destroy(h_); }
    // Preconditioner::solve(double *x): x <- P^{-1} x, device pointer
    virtual void solve(double *x_dev) { ctx_->check(cpg_precond_apply(ctx_->get(), h_, x_dev)); }
    // y <- P^{-1} A x (A.matvec then solve, as a GMRES step does; the split
    // form when this is an FP64 ILU(0) of A's current values whose rounding
    // stays below `accuracy`)
    virtual void applyOperator(const BlockMatrix &A, const double *x_dev, double *y_dev, double accuracy = 0.0) {
        ctx_->check(cpg_precond_apply_op(ctx_->get(), h_, A.get(), x_dev, y_dev, accuracy));
    }
    const cpg_precond *get() const { return h_; }

  protected:
    Preconditioner(const BlockMatrix &A, const Context &ctx, int kind, int prec) : ctx_(&ctx) {
        ctx.check(cpg_precond_create(ctx.get(), A.get(), kind, prec, &h_));
    }
    Preconditioner() = default;
    const Context *ctx_ = nullptr;
    cpg_precond *h_ = nullptr;
};
struct NoPreconditioner : Preconditioner {
    void solve(double *) override {}
    void applyOperator(const BlockMatrix &A, const double *x_dev, double *y_dev, double = 0.0) override {
        A.matvec(x_dev, y_dev);
    }
};
struct BlockJacobi : Preconditioner {
    BlockJacobi(const BlockMatrix &M, const Context &ctx, int prec = CPG_F64)
        : Preconditioner(M, ctx, CPG_PC_BJACOBI, prec) {}
};
struct BlockILU0 : Preconditioner {
    BlockILU0(const BlockMatrix &A, const Context &ctx, int prec = CPG_F64)
        : Preconditioner(A, ctx, CPG_PC_ILU0, prec) {}
};

// Equation (src/Equation.h:8-67) with MassMatrix operations
class Equation {
  public:
    Equation(const Context &ctx, const PolyMesh &msh, const cpg_equation_desc &d) : ctx_(&ctx) {
        ctx.check(cpg_equation_create(ctx.get(), msh.get(), &d, &h_));
        cpg_equation_get_info(h_, &info_);
        nc = info_.nc;
        deg = d.degree;
        np = info_.n_cells;
    }
    virtual ~Equation() { cpg_equation_destroy(h_); }
    Equation(const Equation &) = delete;
    Equation &operator=(const Equation &) = delete;

    // Equation::assemble (Equation.cpp:152-191)
    MeshFn assemble(const MeshFn &u, double t) {
        MeshFn b(*ctx_, np, deg, nc);
        ctx_->check(cpg_assemble(ctx_->get(), h_, u.data(), t, b.data()));
        return b;
    }
    // Equation::jacobian (Equation.cpp:193-279)
    std::unique_ptr<Jacobian> jacobian(const MeshFn &u, double t, int prec = CPG_F64) {
        cpg_bsr *J;
        ctx_->check(cpg_bsr_create(ctx_->get(), h_, prec, &J));
        std::unique_ptr<Jacobian> out(new Jacobian(*ctx_, J));
        ctx_->check(cpg_jacobian(ctx_->get(), h_, u.data(), t, 1.0, 0, J));
        return out;
    }
    // MassMatrix::matvec / solve (MassMatrix.cpp:96-135)
    MeshFn massMatvec(const MeshFn &x) {
        MeshFn y(*ctx_, np, deg, nc);
        ctx_->check(cpg_mass_apply(ctx_->get(), h_, x.data(), y.data()));
        return y;
    }
    MeshFn massSolve(const MeshFn &x) {
        MeshFn y(*ctx_, np, deg, nc);
        ctx_->check(cpg_mass_solve(ctx_->get(), h_, x.data(), y.data()));
        return y;
    }
    // MeshFn::L2Norm (MeshFn.cpp:299-312)
    std::vector<double> L2Norm(const MeshFn &u) {
        std::vector<double> out(4);
        ctx_->check(cpg_l2norm(ctx_->get(), h_, u.data(), out.data()));
        out.resize(nc);
        return out;
    }
    // MeshFn::interp of an analytic field (MeshFn.cpp:56-145)
    MeshFn interp(int kind, const std::vector<double> &params, double t = 0) {
        MeshFn u(*ctx_, np, deg, nc);
        std::vector<double> p(params);
        p.resize(8, 0.0);
        ctx_->check(cpg_interp(ctx_->get(), h_, kind, p.data(), t, u.data()));
        return u;
    }
    cpg_equation *get() const { return h_; }
    const Context &context() const { return *ctx_; }
    int nc = 1, deg = 1, np = 0;

  protected:
    const Context *ctx_;
    cpg_equation *h_ = nullptr;
    cpg_equation_info info_{};
};

inline cpg_equation_desc advection_desc(int deg, double bx, double by, bool rotating) {
    cpg_equation_desc d{};
    d.physics = rotating ? CPG_ADVECTION_ROTATING : CPG_ADVECTION_CONST;
    d.degree = deg;
    d.beta[0] = bx;
    d.beta[1] = by;
    return d;
}
// eqns/Advection.h
struct Advection : Equation {
    Advection(const Context &c, const PolyMesh &m, int deg) : Equation(c, m, advection_desc(deg, 0, 0, true)) {}
};
struct ConstantAdvection : Equation {
    ConstantAdvection(const Context &c, const PolyMesh &m, int deg, double bx, double by)
        : Equation(c, m, advection_desc(deg, bx, by, false)) {}
};
// eqns/Euler.h
struct Euler : Equation {
    static cpg_equation_desc desc(int deg, double g, int dkind, const std::vector<double> &dp, bool exact) {
        cpg_equation_desc d{};
        d.physics = CPG_EULER;
        d.degree = deg;
        d.gamma = g;
        d.dirichlet_kind = dkind;
        d.exact_jacobian = exact ? 1 : 0;
        for (size_t q = 0; q < dp.size() && q < 8; q++) d.dirichlet_params[q] = dp[q];
        return d;
    }
    // exact_jacobian = false keeps the reference's Jacobian entries
    Euler(const Context &c, const PolyMesh &m, int deg, double g, int dkind = CPG_INIT_CONSTANT,
          const std::vector<double> &dp = {}, bool exact_jacobian = false)
        : Equation(c, m, desc(deg, g, dkind, dp, exact_jacobian)) {}
};

// TimeStepper (src/TimeIntegration.h:10-83)
class TimeStepper {
  public:
    TimeStepper(Equation &eqn, const cpg_stepper_desc &d) : eqn_(eqn) {
        eqn.context().check(cpg_stepper_create(eqn.context().get(), eqn.get(), &d, &h_));
    }
    virtual ~TimeStepper() { cpg_stepper_destroy(h_); }
    TimeStepper(const TimeStepper &) = delete;
    TimeStepper &operator=(const TimeStepper &) = delete;
    // TimeStepper::advance: returns the new state (value semantics)
    MeshFn advance(const MeshFn &u, double dt, double t = 0) {
        MeshFn out(u);
        eqn_.context().check(cpg_step(eqn_.context().get(), h_, out.data(), dt, t, &stats));
        return out;
    }
    cpg_step_stats stats{};

  protected:
    static cpg_stepper_desc desc(int kind, int pc = CPG_PC_ILU0) {
        cpg_stepper_desc d{};
        d.kind = kind;
        d.pc_kind = pc;
        d.matrix_precision = CPG_F64;
        d.gmres_m = 20;
        d.gmres_tol = 1e-14;
        d.newton_tol = 5e-13;
        d.newton_maxit = 100;
        return d;
    }
    Equation &eqn_;
    cpg_stepper *h_ = nullptr;
};
struct ForwardEuler : TimeStepper {
    explicit ForwardEuler(Equation &e) : TimeStepper(e, desc(CPG_STEP_FORWARD_EULER)) {}
};
struct RK2 : TimeStepper {
    explicit RK2(Equation &e) : TimeStepper(e, desc(CPG_STEP_RK2)) {}
};
struct RK4 : TimeStepper {
    explicit RK4(Equation &e) : TimeStepper(e, desc(CPG_STEP_RK4)) {}
};
struct BackwardEuler : TimeStepper {
    explicit BackwardEuler(Equation &e) : TimeStepper(e, desc(CPG_STEP_BACKWARD_EULER)) {}
};
struct DIRK : TimeStepper {
    DIRK(int nStages, Equation &e) : TimeStepper(e, desc(nStages == 5 ? CPG_STEP_DIRK5 : CPG_STEP_DIRK3)) {}
    DIRK(Equation &e, const cpg_stepper_desc &d) : TimeStepper(e, d) {}
};
struct IRK : TimeStepper {
    IRK(int nStages, Equation &e, bool inverted = false)
        : TimeStepper(e, desc(nStages == 3 ? (inverted ? CPG_STEP_IRK3_INV : CPG_STEP_IRK3)
                                           : (inverted ? CPG_STEP_IRK2_INV : CPG_STEP_IRK2))) {}
    IRK(Equation &e, const cpg_stepper_desc &d) : TimeStepper(e, d) {}
};

}  // namespace cpolyg
