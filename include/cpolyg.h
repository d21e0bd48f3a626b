/*
 * cpolyg.h -- C ABI of the B200 (sm_100a) implementation of the polygonal
 * discontinuous Galerkin hot path of cpolyg:
 *
 *   residual (Equation::assemble) -> block Jacobian (Equation::jacobian)
 *   -> BSR matvec (BlockMatrix::matvec) -> block ILU(0) / block Jacobi
 *   (Preconditioners) -> restarted GMRES (BlockMatrix::gmres)
 *   -> RK / DIRK / IRK stage updates (TimeIntegration).
 *
 * Every function returns a cpg_status; on failure cpg_last_error(ctx) holds a
 * one-line description.  Signatures carry only plain C types: pointers to
 * device memory are marked `_dev`, pointers to host memory `_host`.
 *
 * Field layout ("MeshFn" order, identical to the reference's
 * arma::cube(nb, nc, n) flattening, src/MeshFn.h:6-9): coefficient k of
 * component c of cell i lives at  k + nb*c + nb*nc*i,  nb = (p+1)(p+2)/2.
 *
 * Block layout: BSR with n_rows block rows of bl x bl blocks, bl = nb*nc,
 * blocks stored contiguously, each block column-major (element (r, c) at
 * c*bl + r), exactly as the reference's arma::mat blocks
 * (src/BlockMatrix.h:12-24).  Row i of a Jacobian holds the diagonal block
 * first, then one block per polygon edge that has a neighbour, in edge order
 * (src/Jacobian.cpp:7-47).
 *
 * All device work of a context is issued on the context's stream.  A context
 * is not thread safe; use one context per host thread.
 */
#ifndef CPOLYG_H
#define CPOLYG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* status codes                                                              */
/* ------------------------------------------------------------------------ */
typedef enum {
    CPG_OK = 0,
    CPG_ERR_INVALID_ARG = 1,
    CPG_ERR_OOM = 2,
    CPG_ERR_SINGULAR_BLOCK = 3, /* a pivot block could not be inverted      */
    CPG_ERR_NONFINITE = 4,      /* NaN/Inf in a residual or iterate         */
    CPG_ERR_NOT_CONVERGED = 5,  /* GMRES or Newton hit its iteration limit  */
    CPG_ERR_TIMEOUT = 6,        /* a bounded device wait ran out            */
    CPG_ERR_CUDA = 7,           /* a CUDA runtime call failed               */
    CPG_ERR_MESH = 8,           /* inconsistent or too coarse mesh          */
    CPG_ERR_UNSUPPORTED = 9,    /* degree / block size not compiled in     */
    CPG_ERR_NONPHYSICAL = 10    /* Euler state with density or pressure
                                   <= 0 (or not finite) at a quadrature
                                   point; cpg_last_error names the cell     */
} cpg_status;

/* physics, replaces the four pure virtuals of Equation (src/Equation.h:46-51)
 * with compile-time device functors selected by this code                    */
typedef enum {
    CPG_ADVECTION_CONST = 0,    /* ConstantAdvection (eqns/Advection.h:24-42) */
    CPG_ADVECTION_ROTATING = 1, /* Advection, beta = (2y-1, -2x+1)
                                   (eqns/Advection.cpp:8-16)                  */
    CPG_EULER = 2               /* Euler, Rusanov flux (eqns/Euler.cpp)       */
} cpg_physics;

/* boundary codes stored in the edge-neighbour table for exterior edges      */
typedef enum {
    CPG_BC_DIRICHLET = -1,  /* value from the problem's boundary state /
                               exact solution (BoundaryConditions.cpp:11-13)  */
    CPG_BC_WALL = -2,       /* slip wall: normal momentum reflected          */
    CPG_BC_OUTFLOW = -3,    /* extrapolation: u+ = u-                         */
    CPG_BC_INFLOW = -4      /* fixed free-stream state                        */
} cpg_bc_code;

/* initial data / exact solutions evaluated by cpg_interp and used as
 * Dirichlet states                                                           */
typedef enum {
    CPG_INIT_CONSTANT = 0,     /* params[0..nc-1] = state                     */
    CPG_INIT_GAUSSIAN = 1,     /* scalar: exp(-a((x-x0-bx t)^2+(y-y0-by t)^2)),
                                  params = {a, x0, y0, bx, by, Lx, Ly}: the
                                  centre moves with (bx, by); Lx, Ly > 0 take
                                  the nearest periodic image (the exact
                                  solution of constant advection)             */
    CPG_INIT_VORTEX = 2,       /* isentropic vortex, params =
                                  {beta, x0, y0, uinf, vinf, gamma, Lx, Ly}   */
    CPG_INIT_DENSITY_BUMP = 3  /* Euler: rho = 1 + A exp(-r^2/w^2), uniform
                                  u = M*c, p = 1/gamma, params =
                                  {A, w, x0, y0, mach, gamma}                 */
} cpg_init_kind;

/* matrix storage precision */
typedef enum { CPG_F64 = 0, CPG_F32 = 1 } cpg_precision;

/* preconditioner kinds (src/Preconditioners.h:10-56) */
typedef enum {
    CPG_PC_NONE = 0,     /* NoPreconditioner                                 */
    CPG_PC_BJACOBI = 1,  /* BlockJacobi                                      */
    CPG_PC_ILU0 = 2,     /* BlockILU0                                        */
    CPG_PC_STAGE_BJACOBI = 3  /* implicit RK only: block Jacobi on the
                                 (stages*bl)^2 cell-coupled stage blocks,
                                 with the stage operator applied in
                                 Kronecker form (never assembled)            */
} cpg_pc_kind;

/* time steppers (src/TimeIntegration.h) */
typedef enum {
    CPG_STEP_FORWARD_EULER = 0,
    CPG_STEP_RK2 = 1,
    CPG_STEP_RK4 = 2,
    CPG_STEP_BACKWARD_EULER = 3,
    CPG_STEP_DIRK3 = 4,
    CPG_STEP_DIRK5 = 5,
    CPG_STEP_IRK2 = 6,        /* Radau IIA, 2 stages, IRK::advance           */
    CPG_STEP_IRK3 = 7,        /* Radau IIA, 3 stages, IRK::advance           */
    CPG_STEP_IRK2_INV = 8,    /* IRK::newAdvance, 2 stages                   */
    CPG_STEP_IRK3_INV = 9,    /* IRK::newAdvance, 3 stages                   */
    CPG_STEP_SDIRK3 = 10      /* DIRK::advance with Alexander's L-stable
                                 3-stage SDIRK of order 3 (gamma =
                                 0.435866521508459, stiffly accurate).  The
                                 reference's getDIRK(3) (TimeIntegration.cpp:
                                 70-77, CPG_STEP_DIRK3 here) combines this
                                 gamma with Crouzeix's tableau: order 2 and
                                 not A-stable (|R(-inf)| = 1.78), so stiff DG
                                 modes grow at large time steps.             */
} cpg_step_kind;

typedef struct cpg_ctx cpg_ctx;
typedef struct cpg_mesh cpg_mesh;
typedef struct cpg_equation cpg_equation;
typedef struct cpg_bsr cpg_bsr;
typedef struct cpg_precond cpg_precond;
typedef struct cpg_stepper cpg_stepper;

/* ------------------------------------------------------------------------ */
/* context                                                                   */
/* ------------------------------------------------------------------------ */
/* stream: a cudaStream_t (NULL = legacy default stream).                     */
cpg_status cpg_ctx_create(int device, void *stream, cpg_ctx **out);
void cpg_ctx_destroy(cpg_ctx *ctx);
const char *cpg_last_error(const cpg_ctx *ctx);
/* Waits for the context's stream, then reads the device status words that
 * deferred calls left: a sweep whose bounded wait ran out (CPG_ERR_TIMEOUT),
 * a residual that met a non-physical state (CPG_ERR_NONPHYSICAL).          */
cpg_status cpg_ctx_sync(cpg_ctx *ctx);
/* on != 0: cpg_precond_apply and cpg_assemble launch their kernels and
 * return without synchronizing to read their status words (which they do
 * by default), so that back-to-back calls stay asynchronous; the words are
 * read by the next cpg_ctx_sync.  No counterpart in the reference (its calls
 * are synchronous CPU code).                                                */
cpg_status cpg_ctx_set_deferred_checks(cpg_ctx *ctx, int on);
/* number of kernels this library launched on ctx since creation */
uint64_t cpg_ctx_launch_count(const cpg_ctx *ctx);
/* library version string, e.g. "cpolyg_b200 0.1 sm_100a" */
const char *cpg_version(void);

/* ------------------------------------------------------------------------ */
/* host mesh (replaces PolyMesh, src/PolyMesh.h:13-55; stays on the host)    */
/* ------------------------------------------------------------------------ */
/* Seeds: std::mt19937_64(seed), x = (g()>>11)*2^-53 * width, then y.        */
cpg_status cpg_seeds_uniform(uint64_t seed, int n, double width, double height,
                             double *xy_host);
/* Voronoi cells of the seeds on [0,width]x[0,height] (PolyMesh(pts,w,h),
 * src/PolyMesh.cpp:162-218).  periodic != 0 wraps both directions;
 * otherwise side_codes[4] (bottom, right, top, left; NULL = all
 * CPG_BC_DIRICHLET) label exterior edges.  Cell i is the cell of seed i.    */
cpg_status cpg_mesh_voronoi(const double *xy_host, int n, double width,
                            double height, int periodic, const int *side_codes,
                            cpg_mesh **out);
/* Mesh from explicit convex polygons (generators of src/Meshes.cpp):
 * cell_ptr[n+1], poly_xy[2*cell_ptr[n]] vertex coordinates per cell.        */
cpg_status cpg_mesh_from_polygons(int n, const int *cell_ptr,
                                  const double *poly_xy, double width,
                                  double height, int periodic,
                                  const int *side_codes, cpg_mesh **out);
/* Replace the sub-triangulation that the volume quadrature integrates on
 * (Quadrature::polygonIntegral over Triangulation's triangles,
 * src/Quadrature.cpp:13-57, src/Triangulation.cpp:11-101).  By default
 * each polygon is split into the fan from its vertex centroid; a caller may
 * pass the reference's own Triangle "zQq" triangles instead.  tri_ptr[n+1]
 * (at least one triangle per cell), tri_xy[6*tri_ptr[n]] = (x0,y0,x1,y1,
 * x2,y2) per triangle in the cell's frame (the coordinates cpg_mesh_export
 * returns).  The triangles of a cell must cover its polygon: their areas
 * must add up to the polygon's (1e-9 relative) and their vertices lie in its
 * bounding box, else CPG_ERR_MESH.  Equations created afterwards use them. */
cpg_status cpg_mesh_set_subtriangles(cpg_mesh *m, const int *tri_ptr,
                                     const double *tri_xy);
void cpg_mesh_destroy(cpg_mesh *m);

typedef struct {
    int n_cells;
    int n_verts;     /* distinct (canonical) vertices                       */
    int n_edges;     /* sum of polygon sizes = cell_ptr[n]                   */
    int n_tris;      /* sub-triangles for volume quadrature                  */
    int periodic;
    double width, height;
} cpg_mesh_info;
cpg_status cpg_mesh_get_info(const cpg_mesh *m, cpg_mesh_info *info);
/* Copy mesh arrays out (any pointer may be NULL):
 *   cell_ptr[n+1], poly_xy[2*E] (cell-frame vertex coordinates),
 *   vert_id[E] (canonical vertex id), edge_nbr[E] (neighbour cell or
 *   boundary code of edge e = (vertex e, vertex e+1)), edge_shift[2*E]
 *   (point x on edge e maps to x+shift in the neighbour's frame),
 *   bb[4*n] (x0, y0, w, h), tri_ptr[n+1], tri_xy[6*T].                      */
cpg_status cpg_mesh_export(const cpg_mesh *m, int *cell_ptr, double *poly_xy,
                           int *vert_id, int *edge_nbr, double *edge_shift,
                           double *bb, int *tri_ptr, double *tri_xy);
/* Host only.  Jacobian block pattern of the mesh (Jacobian ctor,
 * src/Jacobian.cpp:7-47): rowptr[n+1], colidx[nnzb]; pass colidx = NULL to
 * query nnzb first.                                                         */
cpg_status cpg_mesh_pattern(const cpg_mesh *m, int *rowptr, int *colidx,
                            int64_t *nnzb);
/* Host only.  ILU(0) level schedule of a block pattern, the dependency
 * order of BlockILU0's factor and triangular sweeps
 * (src/Preconditioners.cpp:49-158): lower_ptr[n_lower+1] / lower_rows[n]
 * (forward), upper_ptr[n_upper+1] / upper_rows[n] (backward).  Pointers may
 * be NULL to query the level counts.                                        */
cpg_status cpg_pattern_levels(int n, const int *rowptr, const int *colidx,
                              int *n_lower, int *lower_ptr, int *lower_rows,
                              int *n_upper, int *upper_ptr, int *upper_rows);

/* ------------------------------------------------------------------------ */
/* equation: device geometry + physics (replaces Equation, Equation.h:8-67,  */
/* MassMatrix, MassMatrix.h:11-27, BoundaryConditions)                       */
/* ------------------------------------------------------------------------ */
typedef struct {
    int physics;          /* cpg_physics                                    */
    int degree;           /* p, 1..3                                        */
    double gamma;         /* Euler ratio of specific heats                  */
    double beta[2];       /* constant advection velocity                    */
    int dirichlet_kind;   /* cpg_init_kind used for CPG_BC_DIRICHLET        */
    double dirichlet_params[8];
    double inflow_state[4];  /* state for CPG_BC_INFLOW                     */
    int exact_jacobian;   /* 0: the reference's Euler Jacobian (entry (3,1)
                             of A_x is H-(g-1)(u^2+v^2), Euler.cpp:154-163;
                             neighbour blocks use the own state,
                             Euler.cpp:168-179); 1: exact derivatives.  The
                             residual, and so the converged solution, is the
                             same; only Newton's convergence rate differs.  */
} cpg_equation_desc;

cpg_status cpg_equation_create(cpg_ctx *ctx, const cpg_mesh *m,
                               const cpg_equation_desc *desc,
                               cpg_equation **out);
void cpg_equation_destroy(cpg_equation *eq);

typedef struct {
    int n_cells, nb, nc, bl;
    int64_t n_dof;        /* n_cells * bl                                   */
    int64_t nnzb;         /* blocks of the Jacobian pattern                 */
    int n_vqp, n_faces, nqf;   /* volume qp, faces, qp per face            */
    int levels_lower, levels_upper;  /* ILU(0) level counts                 */
} cpg_equation_info;
cpg_status cpg_equation_get_info(const cpg_equation *eq,
                                 cpg_equation_info *info);

/* Equation::assemble (src/Equation.cpp:152-191): b = volume - boundary.    */
cpg_status cpg_assemble(cpg_ctx *ctx, const cpg_equation *eq,
                        const double *u_dev, double t, double *b_dev);

/* MassMatrix::matvec / solve (src/MassMatrix.cpp:96-135), out of place.     */
cpg_status cpg_mass_apply(cpg_ctx *ctx, const cpg_equation *eq,
                          const double *x_dev, double *y_dev);
cpg_status cpg_mass_solve(cpg_ctx *ctx, const cpg_equation *eq,
                          const double *x_dev, double *y_dev);
/* MeshFn::L2Norm (src/MeshFn.cpp:299-312): per-component sqrt(u_c^T M u_c),
 * out_host[nc].                                                             */
cpg_status cpg_l2norm(cpg_ctx *ctx, const cpg_equation *eq,
                      const double *u_dev, double *out_host);
/* No counterpart in the reference.  Same result as cpg_l2norm, for callers
 * that may not allocate device or pinned host memory during the call:
 * applications that give every byte of device memory to their own pool, or
 * that admit work against a fixed memory budget (as cpolyg_b200.serve does),
 * cannot let a norm grow a scratch buffer inside their Newton loop.  The
 * partial sums live in a static device array of 1028 doubles (8224 bytes)
 * that every GPU loading this library holds until the process exits; it
 * serves equations with at most 4 components and rejects anything larger
 * with CPG_ERR_INVALID_ARG.  The context's device must be current.  The first
 * call on a device looks up the array's device address (set-up); make that
 * first call before any stream capture.  Calls share the array: calls that
 * overlap on the GPU (several contexts or streams at once) race and must be
 * serialized by the caller.                                                 */
cpg_status cpg_l2norm_noalloc(cpg_ctx *ctx, const cpg_equation *eq,
                              const double *u_dev, double *out_host);
/* MeshFn::L2Error (src/MeshFn.cpp:283-296): per-component
 * sqrt(sum_K int_K (u_h - exact)^2) with the degree-2p rule on the cells'
 * quadrature points, exact = the analytic field (init_kind, params) at
 * time t; out_host[nc].                                                     */
cpg_status cpg_l2error(cpg_ctx *ctx, const cpg_equation *eq, const double *u_dev, int init_kind,
                       const double *params, double t, double *out_host);
/* MeshFn::interp (src/MeshFn.cpp:56-145): least-squares projection on the
 * (p+1)^2 Gauss grid of each bounding box of an analytic field.             */
cpg_status cpg_interp(cpg_ctx *ctx, const cpg_equation *eq, int init_kind,
                      const double *params, double t, double *u_dev);
/* mass blocks (nb x nb per cell, column-major) to host, for checks          */
cpg_status cpg_mass_export(cpg_ctx *ctx, const cpg_equation *eq,
                           double *mass_host);

/* ------------------------------------------------------------------------ */
/* block sparse matrices (BlockMatrix, src/BlockMatrix.h; Jacobian)           */
/* ------------------------------------------------------------------------ */
/* BSR with the Jacobian pattern of eq (Jacobian ctor, Jacobian.cpp:7-47).   */
cpg_status cpg_bsr_create(cpg_ctx *ctx, const cpg_equation *eq,
                          int precision, cpg_bsr **out);
/* generic BSR from host arrays (values may be NULL = zeros)                 */
cpg_status cpg_bsr_create_host(cpg_ctx *ctx, int n_rows, int bl,
                               const int *rowptr, const int *colidx,
                               const double *values_host, int precision,
                               cpg_bsr **out);
void cpg_bsr_destroy(cpg_bsr *A);
cpg_status cpg_bsr_get_info(const cpg_bsr *A, int *n_rows, int *bl,
                            int64_t *nnzb, int *precision);
cpg_status cpg_bsr_export(cpg_ctx *ctx, const cpg_bsr *A, int *rowptr,
                          int *colidx, double *values_host);
cpg_status cpg_bsr_upload(cpg_ctx *ctx, cpg_bsr *A, const double *values_host);
/* k matrices of one block size and precision stacked block-diagonally into
 * a new matrix (rows and columns of part q offset by the rows of the parts
 * before it); for batched solves.  No counterpart in the reference.         */
cpg_status cpg_bsr_stack(cpg_ctx *ctx, int k, const cpg_bsr *const *parts,
                         cpg_bsr **out);

/* Equation::jacobian (Equation.cpp:193-279) fused with
 * BlockMatrix::operator*= (BlockMatrix.cpp:297-308) and
 * Jacobian::operator+=(MassMatrix) (Jacobian.cpp:99-110):
 *   J <- scale * dF/du  (+ M on the diagonal blocks when add_mass != 0).    */
cpg_status cpg_jacobian(cpg_ctx *ctx, const cpg_equation *eq,
                        const double *u_dev, double t, double scale,
                        int add_mass, cpg_bsr *J);

/* BlockMatrix::matvec (BlockMatrix.cpp:28-49), out of place: y = A x.      */
cpg_status cpg_bsr_matvec(cpg_ctx *ctx, const cpg_bsr *A, const double *x_dev,
                          double *y_dev);

/* ------------------------------------------------------------------------ */
/* preconditioners (src/Preconditioners.h:10-56)                             */
/* ------------------------------------------------------------------------ */
/* factor A into a new preconditioner (BlockILU0 / BlockJacobi ctors);
 * precision = storage of the factors (pivot blocks are inverted in FP64).  */
cpg_status cpg_precond_create(cpg_ctx *ctx, const cpg_bsr *A, int kind,
                              int precision, cpg_precond **out);
/* refactor with new values of the same pattern, reusing storage            */
cpg_status cpg_precond_refactor(cpg_ctx *ctx, cpg_precond *P, const cpg_bsr *A);
/* Preconditioner::solve(double *x): x <- P^{-1} x in place                  */
cpg_status cpg_precond_apply(cpg_ctx *ctx, const cpg_precond *P, double *x_dev);
/* y <- P^{-1} A x: the preconditioned operator of a left-preconditioned
 * Krylov step, `matvec(vi1); pc.solve(vi1)` in BlockMatrix::gmres
 * (src/BlockMatrix.cpp:121-122).  x and y distinct.  When P is an FP64
 * ILU(0) factored from A's current values (cpg_precond_split_ready), it can
 * be computed in split form: with A = (I + L) D + D U' + E, where
 * E_i = A_ii - Ahat_ii,
 *   P^{-1} A x = (I + U')^{-1} [x + D^{-1} (I + L)^{-1} (U_A + E) x],
 * which streams A's upper blocks and E instead of all of A.  Its rounding is
 * that of A perturbed by about eps * cond(D_i) relative, so it is taken only
 * when 0.25 * eps * cpg_precond_pivot_cond(P) <= accuracy (0: never);
 * otherwise the call is cpg_bsr_matvec followed by cpg_precond_apply.
 * cpg_gmres and cpg_gmres_batched decide the same way, with their tolerance
 * as the accuracy, in every Arnoldi step of the left-preconditioned form.  */
cpg_status cpg_precond_apply_op(cpg_ctx *ctx, const cpg_precond *P, const cpg_bsr *A, const double *x_dev,
                                double *y_dev, double accuracy);
/* 1 when cpg_precond_apply_op(P, A) takes the split form: P is an FP64
 * ILU(0) whose last factorisation read A's current values (any write to A's
 * values through this library since then, or another matrix, gives 0).
 * CPG_SPLIT_OPERATOR=0 at preconditioner creation turns the form off.      */
int cpg_precond_split_ready(const cpg_precond *P, const cpg_bsr *A);
/* largest cond_inf(Ahat_ii) = |Ahat_ii|_inf |Ahat_ii^{-1}|_inf over the pivot
 * blocks of the last factorisation (0 before one, or for no preconditioner) */
double cpg_precond_pivot_cond(const cpg_precond *P);
void cpg_precond_destroy(cpg_precond *P);
/* Triangular sweep form of an ILU(0) preconditioner: 1 = sync-free (one
 * launch per sweep), 2 = one launch per level with the sync-free form's
 * threads per row (bitwise the same result as 1), 3 = one launch per level
 * with the widest rows (another summation order), 4 / 5 / 6 = sync-free
 * with direct loads and 1 / 2 / 4 times form 1's threads per row (4 sums
 * as 1), 0 = not decided yet: the
 * first application times the candidates on a scratch copy of its vector,
 * then applies the fastest, and the decision holds for every ILU(0)
 * preconditioner of the process with the same block size, precision and
 * size class.  CPG_ILU_SWEEP=syncfree, =syncfree_direct, =levels,
 * =levels_wide or =form<N> in the environment when the preconditioner is
 * created forces a form.  No counterpart in the reference (its sweeps are sequential
 * loops, Preconditioners.cpp:125-158).                                      */
int cpg_precond_sweep_form(const cpg_precond *P);
/* Failure-detection check of the sync-free sweeps: runs, for each of the
 * two sync-free kernels (TMA ring, direct loads), a one-row sweep whose
 * dependency is never published, so the row's bounded wait runs out (a few
 * seconds each); returns CPG_ERR_TIMEOUT when both reported it, and leaves
 * the context usable.  No counterpart in the reference.                     */
cpg_status cpg_debug_sweep_timeout(cpg_ctx *ctx);
/* ILU(0) level schedule (row lists by level), for checks:
 *   lower_ptr[levels_lower+1], lower_rows[n], upper_ptr[...], upper_rows[n] */
cpg_status cpg_precond_levels(const cpg_precond *P, int *n_lower,
                              int *lower_ptr, int *lower_rows, int *n_upper,
                              int *upper_ptr, int *upper_rows);
/* factors to host (ILU: DD inverse blocks [n], L [nnzL], DU [nnzU] in the
 * reference's BlockMatrix order; Jacobi: inverse diagonal blocks [n])       */
cpg_status cpg_precond_export(cpg_ctx *ctx, const cpg_precond *P,
                              double *dinv_host, int *l_rowptr, int *l_col,
                              double *l_host, int *u_rowptr, int *u_col,
                              double *u_host);

/* ------------------------------------------------------------------------ */
/* Krylov (BlockMatrix::gmres, BlockMatrix.cpp:79-163; jacobi :51-77)        */
/* ------------------------------------------------------------------------ */
typedef struct {
    int iterations;       /* maxIt on output                                 */
    double residual;      /* tol on output: |y_i| / ||P^{-1} b||            */
    int converged;
} cpg_solve_stats;

/* Left-preconditioned restarted GMRES(m) with classical Gram-Schmidt as in
 * the reference when flexible == 0; right-preconditioned flexible GMRES(m)
 * (FGMRES) when flexible != 0.  P may be NULL (NoPreconditioner).  x holds
 * the initial guess on input.                                               */
cpg_status cpg_gmres(cpg_ctx *ctx, const cpg_bsr *A, const cpg_precond *P,
                     const double *b_dev, double *x_dev, int m, double tol,
                     int maxit, int flexible, cpg_solve_stats *stats);
/* No counterpart in the reference (its GMRES solves one system).  nsys
 * independent systems solved together: A is block diagonal, system k owning
 * block rows [seg_rows[k], seg_rows[k+1]) (host array, nsys + 1 entries;
 * cpg_bsr_stack builds such an A from separate matrices), P is A's
 * preconditioner (for a block-diagonal A, ILU(0) and block Jacobi factor each
 * system on its own), b and x stacked the same way.  Every system has its
 * own Krylov basis coefficients, rotations and stopping test, with the same
 * iterates as cpg_gmres on that system alone; one launch sequence serves all
 * of them.  stats: nsys entries.  Rejects an A that couples two systems.    */
cpg_status cpg_gmres_batched(cpg_ctx *ctx, const cpg_bsr *A,
                             const cpg_precond *P, int nsys,
                             const int *seg_rows_host, const double *b_dev,
                             double *x_dev, int m, double tol, int maxit,
                             int flexible, cpg_solve_stats *stats);
/* damped block-Jacobi iteration, omega = 1 (BlockMatrix::jacobi)           */
cpg_status cpg_jacobi_solve(cpg_ctx *ctx, const cpg_bsr *A,
                            const cpg_precond *P, const double *b_dev,
                            double *x_dev, double tol, int maxit,
                            cpg_solve_stats *stats);

/* ------------------------------------------------------------------------ */
/* vector helpers on fields (MeshFn arithmetic, MeshFn.cpp:209-247)          */
/* ------------------------------------------------------------------------ */
/* y <- a*x + b*y over n doubles */
cpg_status cpg_axpby(cpg_ctx *ctx, int64_t n, double a, const double *x_dev,
                     double b, double *y_dev);

/* ------------------------------------------------------------------------ */
/* time steppers (TimeStepper::advance, src/TimeIntegration.h:16)            */
/* ------------------------------------------------------------------------ */
typedef struct {
    int kind;                /* cpg_step_kind                               */
    int pc_kind;             /* cpg_pc_kind for implicit steppers           */
    int matrix_precision;    /* cpg_precision of Jacobian + factors         */
    int gmres_m;             /* restart length (reference: 20)              */
    double gmres_tol;        /* relative tolerance (reference: 1e-14)       */
    int gmres_maxit;         /* reference: 90000 (DIRK), 20000 (IRK)        */
    int flexible;            /* 1 = FGMRES (right preconditioned)           */
    double newton_tol;       /* reference: 5e-13                            */
    int newton_maxit;        /* reference: 100                              */
    int reuse_jacobian;      /* 0 = rebuild J and P every Newton iteration
                                as the reference; k > 0 = rebuild every k   */
    double newton_rtol;      /* 0 = the reference's stopping rule alone; r >
                                0 = also require the last Newton update to
                                be below r relative to the stage vector (in
                                the same L2 norm): the reference's residual
                                norm weights the weak-form residual by the
                                mass matrix and can pass while an inexact
                                (FP32-Jacobian) Newton iteration is still
                                converging                                  */
    int pc_f32;              /* 1 = store the preconditioner's factors in
                                FP32 even when the matrix is FP64 (FP64
                                operator, FP32 preconditioner); 0 = same
                                precision as the matrix                     */
} cpg_stepper_desc;

typedef struct {
    int newton_iterations;   /* summed over stages                          */
    int gmres_iterations;    /* summed over all linear solves               */
    int linear_solves;
    double last_newton_residual;
    int converged;
} cpg_step_stats;

cpg_status cpg_stepper_create(cpg_ctx *ctx, cpg_equation *eq,
                              const cpg_stepper_desc *desc, cpg_stepper **out);
void cpg_stepper_destroy(cpg_stepper *s);
/* u_dev <- advance(u_dev, dt, t) */
cpg_status cpg_step(cpg_ctx *ctx, cpg_stepper *s, double *u_dev, double dt,
                    double t, cpg_step_stats *stats);
/* same, with u in host memory; copies in and out on the context stream
 * (the reference's value-semantics MeshFn advance at the host boundary)    */
cpg_status cpg_step_host(cpg_ctx *ctx, cpg_stepper *s, double *u_host,
                         double dt, double t, cpg_step_stats *stats);

/* ------------------------------------------------------------------------ */
/* gnuplot text output (visual cross-checks; host files)                    */
/* ------------------------------------------------------------------------ */
/* PolyMesh::gnuplot (src/PolyMesh.cpp:221-241): per cell "# polygon number
 * i", its vertices with the first repeated, a blank line.  Coordinates are
 * the cell's own frame, so periodic cells are not cut at the domain edge.   */
cpg_status cpg_mesh_write_gnuplot(const cpg_mesh *m, const char *path);
/* MeshFn::gnuplot (src/MeshFn.cpp:161-207): one line "x y u_0 .. u_nc-1" per
 * point of the 3-point triangle rule on every sub-triangle of every cell;
 * the field is evaluated on the device.  m must be the equation's mesh.    */
cpg_status cpg_field_write_gnuplot(cpg_ctx *ctx, const cpg_equation *eq,
                                   const cpg_mesh *m, const double *u_dev,
                                   const char *path);
/* BlockMatrix::spy (src/BlockMatrix.cpp:318-349): one line "row col value"
 * per entry with |value| > 1e-10.                                            */
cpg_status cpg_bsr_write_spy(cpg_ctx *ctx, const cpg_bsr *A, const char *path);

#ifdef __cplusplus
}
#endif
#endif /* CPOLYG_H */
