// Equation: quadrature geometry on the device, DG residual (Equation::assemble),
// block Jacobian (Equation::jacobian) fused with the Newton-matrix update
// B = scale*J + M, mass matrix apply/solve, L2 norms and the projection of
// analytic fields (MeshFn::interp).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>

#include "internal.hpp"
#include "quadrature.hpp"

using namespace cpg;

namespace {

constexpr int nqf_of(int p) { return (2 * p <= 2) ? 2 : ((2 * p <= 4) ? 4 : 6); }

// ---------------------------------------------------------------------------
// residual: one warp per cell.  Lanes stride over the cell's volume qp and
// face qp; each lane accumulates all nb*nc test-function sums; a butterfly
// reduction combines the lanes.  Flux evaluations are done once per qp and
// contracted against every test function (the reference recomputes them per
// test function, Equation.cpp:176-187).
// ---------------------------------------------------------------------------
// A state that is not admissible (Euler: density or pressure <= 0, or not
// finite) at any of the cell's quadrature points records the cell in
// *nonphys (cell + 1, first writer wins) for the host to report.
template <class Phys, int P>
__global__ void __launch_bounds__(128) k_residual(Geo g, Phys ph, BCParams bc, const double *__restrict__ u,
                                                  double t, double *__restrict__ b, int *__restrict__ nonphys) {
    constexpr int NB = nbasis<P>(), NC = Phys::NC, BL = NB * NC, NQF = nqf_of(P);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cell = blockIdx.x * (blockDim.x >> 5) + wid;
    __shared__ double sU[4][BL];
    if (cell >= g.n) return;
    double *U = sU[wid];
    for (int r = lane; r < BL; r += 32) U[r] = u[(size_t)cell * BL + r];
    __syncwarp();
    const double4 box = g.bb[cell];
    const double sx = 2.0 / box.z, sy = 2.0 / box.w;
    double acc[BL];
#pragma unroll
    for (int r = 0; r < BL; r++) acc[r] = 0.0;
    bool bad = false;

    const int q1 = g.vq_ptr[cell + 1];
    for (int q = g.vq_ptr[cell] + lane; q < q1; q += 32) {
        double psi[NB], dx[NB], dy[NB];
        basis_grad<P>(g.vxi[q], g.veta[q], sx, sy, psi, dx, dy);
        double uu[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NB; k++) s += U[c * NB + k] * psi[k];
            uu[c] = s;
        }
        bad |= !ph.admissible(uu);
        double Fx[NC], Fy[NC];
        ph.flux(uu, g.vx[q], g.vy[q], Fx, Fy);
        const double w = g.vw[q];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const double fx = w * Fx[c], fy = w * Fy[c];
#pragma unroll
            for (int k = 0; k < NB; k++) acc[c * NB + k] += fx * dx[k] + fy * dy[k];
        }
    }
    const int f0 = g.f_ptr[cell], nf = g.f_ptr[cell + 1] - f0;
    for (int j = lane; j < nf * NQF; j += 32) {
        const int f = f0 + j / NQF;
        const int fq = f0 * NQF + j;
        double psi[NB];
        basis<P>(g.qxi[fq], g.qeta[fq], psi);
        double um[NC], up[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < NB; k++) s += U[c * NB + k] * psi[k];
            um[c] = s;
        }
        bad |= !ph.admissible(um);
        const int nbr = g.f_nbr[f];
        const double nx = g.f_nx[f], ny = g.f_ny[f], x = g.qx[fq], y = g.qy[fq];
        if (nbr >= 0) {
            double psin[NB];
            basis<P>(g.qxin[fq], g.qetan[fq], psin);
            const double *Un = u + (size_t)nbr * BL;
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) s += __ldg(Un + c * NB + k) * psin[k];
                up[c] = s;
            }
        } else {
            boundary_state(ph, bc, nbr, um, x, y, t, nx, ny, up);
        }
        double F[NC];
        ph.numflux(um, up, x, y, nx, ny, F);
        const double w = g.qw[fq];
#pragma unroll
        for (int c = 0; c < NC; c++) {
            const double fw = w * F[c];
#pragma unroll
            for (int k = 0; k < NB; k++) acc[c * NB + k] -= fw * psi[k];
        }
    }
#pragma unroll
    for (int r = 0; r < BL; r++) {
        double v = acc[r];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        acc[r] = v;
    }
#pragma unroll
    for (int r = 0; r < BL; r++)
        if ((r & 31) == lane) b[(size_t)cell * BL + r] = acc[r];
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicCAS(nonphys, 0, cell + 1);
}

// ---------------------------------------------------------------------------
// Jacobian: one CTA per cell.  Thread t < nb*nb owns the test/trial pair
// (k, j) of every nc x nc component coupling of the diagonal block and of
// the neighbour blocks.  Quadrature-point data (basis values, flux
// Jacobians) is staged in shared memory in chunks.
//   diagonal  +=  sum_q w phi_j (Ax dpsi_k/dx + Ay dpsi_k/dy)
//             -=  sum_faces sum_q w psi_k phi_j dFhat(u, u2, n, +1)
//   neighbour  =  - sum_q w psi_k phi_j^nbr dFhat(u, u2, n, -1)
// (Equation.cpp:193-279, computeVolumeJacobian :59-73,
//  computeBoundaryJacobian :75-112).  Output: scale * J (+ M on the diagonal).
// ---------------------------------------------------------------------------
constexpr int JT = 128;  // threads per CTA
// volume qp per chunk: one thread stages each point (basis values and flux
// Jacobians), so larger chunks keep more warps busy in that phase; 48 keeps
// the static shared memory below 48 KB and three CTAs on an SM
constexpr int VQC = 48;
constexpr int FQC = 36;  // face qp per chunk (whole faces)

template <class Phys, int P, class TOut>
// at most 168 registers a thread, so three CTAs share an SM (246 unbounded,
// two CTAs); the few spilled bytes cost less than the lost occupancy
__global__ void __launch_bounds__(JT, 3) k_jacobian(Geo g, Phys ph, BCParams bc, const double *__restrict__ u,
                                                 double t, double scale, int add_mass,
                                                 const double *__restrict__ mass, const int *__restrict__ rowptr,
                                                 TOut *__restrict__ J) {
    constexpr int NB = nbasis<P>(), NC = Phys::NC, BL = NB * NC, NQF = nqf_of(P), NC2 = NC * NC;
    constexpr int FPC = FQC / NQF;  // faces per chunk
    // the nc x nc flux-Jacobian rows are staged and read as double2 (16-byte
    // aligned) and padded by two doubles: with rows of 16 doubles (128 bytes)
    // every staging thread's store fell in the same bank; at 144 bytes a
    // quarter-warp's 16-byte stores cover distinct banks
    constexpr bool V2 = NC2 % 2 == 0;
    constexpr int NC2P = V2 ? NC2 + 2 : NC2;
    // basis rows at an odd stride: a half-warp's staging stores (one row per
    // thread) then fall in distinct banks
    constexpr int NBP = NB % 2 == 0 ? NB + 1 : NB;
    const int cell = blockIdx.x;
    const int tid = threadIdx.x;
    __shared__ double sU[BL];
    // volume chunk
    __shared__ double sPW[VQC][NBP], sDX[VQC][NBP], sDY[VQC][NBP];
    __shared__ __align__(16) double sAx[VQC][NC2P], sAy[VQC][NC2P];
    // face chunk (aliases are avoided for clarity; sizes are small)
    __shared__ double fPsiW[FQC][NBP], fPhiO[FQC][NBP], fPhiN[FQC][NBP];
    __shared__ __align__(16) double fMp[FQC][NC2P], fMm[FQC][NC2P];

    for (int r = tid; r < BL; r += JT) sU[r] = u[(size_t)cell * BL + r];
    const double4 box = g.bb[cell];
    const double sx = 2.0 / box.z, sy = 2.0 / box.w;
    const bool owner = tid < NB * NB;
    const int kk = tid % NB, jj = tid / NB;
    double acc[NC2];
#pragma unroll
    for (int e = 0; e < NC2; e++) acc[e] = 0.0;
    __syncthreads();

    // ---- volume
    const int v0 = g.vq_ptr[cell], v1 = g.vq_ptr[cell + 1];
    for (int c0 = v0; c0 < v1; c0 += VQC) {
        const int cnt = min(VQC, v1 - c0);
        for (int q = tid; q < cnt; q += JT) {
            const int qq = c0 + q;
            double psi[NB], dx[NB], dy[NB];
            basis_grad<P>(g.vxi[qq], g.veta[qq], sx, sy, psi, dx, dy);
            double uu[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) s += sU[c * NB + k] * psi[k];
                uu[c] = s;
            }
            double Ax[NC2], Ay[NC2];
            ph.fluxjac(uu, g.vx[qq], g.vy[qq], Ax, Ay);
            const double w = g.vw[qq];
#pragma unroll
            for (int k = 0; k < NB; k++) {
                sPW[q][k] = w * psi[k];
                sDX[q][k] = dx[k];
                sDY[q][k] = dy[k];
            }
            if constexpr (V2) {
#pragma unroll
                for (int e = 0; e < NC2 / 2; e++) {
                    reinterpret_cast<double2 *>(sAx[q])[e] = make_double2(Ax[2 * e], Ax[2 * e + 1]);
                    reinterpret_cast<double2 *>(sAy[q])[e] = make_double2(Ay[2 * e], Ay[2 * e + 1]);
                }
            } else {
#pragma unroll
                for (int e = 0; e < NC2; e++) {
                    sAx[q][e] = Ax[e];
                    sAy[q][e] = Ay[e];
                }
            }
        }
        __syncthreads();
        if (owner) {
            for (int q = 0; q < cnt; q++) {
                const double pw = sPW[q][jj];
                const double ax = sDX[q][kk] * pw, ay = sDY[q][kk] * pw;
                if constexpr (V2) {
                    const double2 *Ax2 = reinterpret_cast<const double2 *>(sAx[q]);
                    const double2 *Ay2 = reinterpret_cast<const double2 *>(sAy[q]);
#pragma unroll
                    for (int e = 0; e < NC2 / 2; e++) {
                        const double2 a = Ax2[e], b = Ay2[e];
                        acc[2 * e] += a.x * ax + b.x * ay;
                        acc[2 * e + 1] += a.y * ax + b.y * ay;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < NC2; e++) acc[e] += sAx[q][e] * ax + sAy[q][e] * ay;
                }
            }
        }
        __syncthreads();
    }

    // ---- faces, in chunks of whole faces
    const int fa = g.f_ptr[cell], fb = g.f_ptr[cell + 1];
    const int diag = rowptr[cell];
    const size_t bl2 = (size_t)BL * BL;
    for (int fc = fa; fc < fb; fc += FPC) {
        const int nfc = min(FPC, fb - fc);
        for (int q = tid; q < nfc * NQF; q += JT) {
            const int f = fc + q / NQF;
            const int fq = fc * NQF + q;
            double psi[NB], phin[NB];
            basis<P>(g.qxi[fq], g.qeta[fq], psi);
            double um[NC], u2[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double s = 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) s += sU[c * NB + k] * psi[k];
                um[c] = s;
            }
            const int nbr = g.f_nbr[f];
            const double nx = g.f_nx[f], ny = g.f_ny[f], x = g.qx[fq], y = g.qy[fq];
            if (nbr >= 0) {
                basis<P>(g.qxin[fq], g.qetan[fq], phin);
                const double *Un = u + (size_t)nbr * BL;
#pragma unroll
                for (int c = 0; c < NC; c++) {
                    double s = 0.0;
#pragma unroll
                    for (int k = 0; k < NB; k++) s += __ldg(Un + c * NB + k) * phin[k];
                    u2[c] = s;
                }
            } else {
                boundary_state(ph, bc, nbr, um, x, y, t, nx, ny, u2);
#pragma unroll
                for (int k = 0; k < NB; k++) phin[k] = 0.0;
            }
            double Mp[NC2], Mm[NC2];
            ph.numfluxjac(um, u2, x, y, nx, ny, 1, Mp);
            ph.numfluxjac(um, u2, x, y, nx, ny, -1, Mm);
            if (nbr == CPG_BC_WALL || nbr == CPG_BC_OUTFLOW) {
                // chain rule through the state-dependent exterior value
                double R[NC2];
                if (nbr == CPG_BC_WALL) {
                    ph.wall_deriv(nx, ny, R);
                } else {
#pragma unroll
                    for (int e = 0; e < NC2; e++) R[e] = (e % (NC + 1) == 0) ? 1.0 : 0.0;
                }
#pragma unroll
                for (int r = 0; r < NC; r++)
#pragma unroll
                    for (int c = 0; c < NC; c++) {
                        double s = 0.0;
#pragma unroll
                        for (int m = 0; m < NC; m++) s += Mm[r * NC + m] * R[m * NC + c];
                        Mp[r * NC + c] += s;
                    }
            }
            const double w = g.qw[fq];
#pragma unroll
            for (int k = 0; k < NB; k++) {
                fPsiW[q][k] = w * psi[k];
                fPhiO[q][k] = psi[k];
                fPhiN[q][k] = phin[k];
            }
            if constexpr (V2) {
#pragma unroll
                for (int e = 0; e < NC2 / 2; e++) {
                    reinterpret_cast<double2 *>(fMp[q])[e] = make_double2(Mp[2 * e], Mp[2 * e + 1]);
                    reinterpret_cast<double2 *>(fMm[q])[e] = make_double2(Mm[2 * e], Mm[2 * e + 1]);
                }
            } else {
#pragma unroll
                for (int e = 0; e < NC2; e++) {
                    fMp[q][e] = Mp[e];
                    fMm[q][e] = Mm[e];
                }
            }
        }
        __syncthreads();
        if (owner) {
            for (int fl = 0; fl < nfc; fl++) {
                const int f = fc + fl;
                double nacc[NC2];
#pragma unroll
                for (int e = 0; e < NC2; e++) nacc[e] = 0.0;
                for (int q = fl * NQF; q < (fl + 1) * NQF; q++) {
                    const double pwk = fPsiW[q][kk];
                    const double dg = pwk * fPhiO[q][jj], nb = pwk * fPhiN[q][jj];
                    if constexpr (V2) {
                        const double2 *Mp2 = reinterpret_cast<const double2 *>(fMp[q]);
                        const double2 *Mm2 = reinterpret_cast<const double2 *>(fMm[q]);
#pragma unroll
                        for (int e = 0; e < NC2 / 2; e++) {
                            const double2 a = Mp2[e], b = Mm2[e];
                            acc[2 * e] -= dg * a.x;
                            acc[2 * e + 1] -= dg * a.y;
                            nacc[2 * e] -= nb * b.x;
                            nacc[2 * e + 1] -= nb * b.y;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < NC2; e++) {
                            acc[e] -= dg * fMp[q][e];
                            nacc[e] -= nb * fMm[q][e];
                        }
                    }
                }
                const int blk = g.f_blk[f];
                if (blk >= 0) {
                    TOut *B = J + (size_t)blk * bl2;
#pragma unroll
                    for (int c = 0; c < NC; c++)
#pragma unroll
                        for (int c2 = 0; c2 < NC; c2++)
                            B[(size_t)(c2 * NB + jj) * BL + (c * NB + kk)] = (TOut)(scale * nacc[c * NC + c2]);
                }
            }
        }
        __syncthreads();
    }
    if (owner) {
        TOut *B = J + (size_t)diag * bl2;
        const double mkj = add_mass ? mass[(size_t)cell * NB * NB + jj * NB + kk] : 0.0;
#pragma unroll
        for (int c = 0; c < NC; c++)
#pragma unroll
            for (int c2 = 0; c2 < NC; c2++) {
                double v = scale * acc[c * NC + c2];
                if (c == c2) v += mkj;
                B[(size_t)(c2 * NB + jj) * BL + (c * NB + kk)] = (TOut)v;
            }
    }
}

// ---------------------------------------------------------------------------
// mass matrix: y = alpha * Mi x + beta * z  (Mi = M or M^{-1} per cell,
// replicated over components)
// ---------------------------------------------------------------------------
template <int NB>
__global__ void k_mass(int n, int nc, const double *__restrict__ Mi, const double *__restrict__ x, double alpha,
                       const double *__restrict__ z, double beta, double *__restrict__ y, const int *skip) {
    if (skip && *skip) return;  // a Krylov solve that has converged
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int BL = NB * nc;
    if (idx >= (int64_t)n * BL) return;
    const int cell = (int)(idx / BL), r = (int)(idx % BL), c = r / NB, k = r % NB;
    const double *M = Mi + (size_t)cell * NB * NB;
    const double *xc = x + (size_t)cell * BL + c * NB;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < NB; j++) s += M[j * NB + k] * xc[j];
    double v = alpha * s;
    if (z) v = v + beta * z[idx];
    y[idx] = v;
}

// per-CTA partial sums of u_c^T M u_c; fixed grid for deterministic results
constexpr int RED_CTAS = 256;
template <int NB>
__global__ void k_l2_partial(int n, int nc, const double *__restrict__ M, const double *__restrict__ u,
                             double *__restrict__ part) {
    __shared__ double sh[4][256];
    double acc[4] = {0, 0, 0, 0};
    const int BL = NB * nc;
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < n; cell += gridDim.x * blockDim.x) {
        const double *Mc = M + (size_t)cell * NB * NB;
        for (int c = 0; c < nc; c++) {
            const double *uc = u + (size_t)cell * BL + c * NB;
            double s = 0.0;
            for (int j = 0; j < NB; j++) {
                double mj = 0.0;
                for (int k = 0; k < NB; k++) mj += Mc[j * NB + k] * uc[k];
                s += uc[j] * mj;
            }
            acc[c] += s;
        }
    }
    for (int c = 0; c < 4; c++) sh[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off)
            for (int c = 0; c < 4; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = sh[threadIdx.x][0];
}
// per-CTA partial sums of sum_q w_q (u_h(x_q) - exact(x_q))^2 over the cells'
// volume quadrature points (MeshFn::L2Error); fixed grid, deterministic
template <int P, int NC>
__global__ void k_l2_error_partial(Geo g, int kind, BCParams prm, double t, const double *__restrict__ u,
                                   double *__restrict__ part) {
    constexpr int NB = nbasis<P>(), BL = NB * NC;
    __shared__ double sh[4][256];
    double acc[4] = {0, 0, 0, 0};
    for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < g.n; cell += gridDim.x * blockDim.x) {
        const double *uc = u + (size_t)cell * BL;
        double cs[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) cs[c] = 0.0;
        for (int q = g.vq_ptr[cell]; q < g.vq_ptr[cell + 1]; q++) {
            double psi[NB], ex[NC];
            basis<P>(g.vxi[q], g.veta[q], psi);
            field_eval<NC>(kind, prm.dparams, g.vx[q], g.vy[q], t, ex);
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double v = 0.0;
#pragma unroll
                for (int k = 0; k < NB; k++) v += uc[c * NB + k] * psi[k];
                const double d = v - ex[c];
                cs[c] += g.vw[q] * (d * d);
            }
        }
#pragma unroll
        for (int c = 0; c < NC; c++) acc[c] += cs[c];
    }
    for (int c = 0; c < 4; c++) sh[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off)
            for (int c = 0; c < 4; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x < 4) part[blockIdx.x * 4 + threadIdx.x] = sh[threadIdx.x][0];
}
__global__ void k_l2_final(int nparts, const double *__restrict__ part, double *__restrict__ out) {
    const int c = threadIdx.x;
    if (c >= 4) return;
    double s = 0.0;
    for (int p = 0; p < nparts; p++) s += part[p * 4 + c];
    out[c] = s;
}

// MeshFn::interp: coefficients = pinv * f(tensor Gauss points of the box)
template <int NC>
__global__ void k_interp(int n, int nb, int m, const double4 *__restrict__ bb, const double *__restrict__ gl,
                         const double *__restrict__ pinv, int kind, BCParams prm, double t,
                         double *__restrict__ u) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= n) return;
    const double4 box = bb[cell];
    const int nq = m * m, BL = nb * NC;
    double cf[NC][15];
    for (int c = 0; c < NC; c++)
        for (int k = 0; k < nb; k++) cf[c][k] = 0.0;
    for (int i = 0; i < m; i++)
        for (int j = 0; j < m; j++) {
            double o[4];
            field_eval<NC>(kind, prm.dparams, (gl[i] + 1) * box.z / 2.0 + box.x, (gl[j] + 1) * box.w / 2.0 + box.y,
                           t, o);
            const int e = i * m + j;
            for (int k = 0; k < nb; k++) {
                const double p = pinv[k * nq + e];
                for (int c = 0; c < NC; c++) cf[c][k] += p * o[c];
            }
        }
    for (int c = 0; c < NC; c++)
        for (int k = 0; k < nb; k++) u[(size_t)cell * BL + c * nb + k] = cf[c][k];
}

// dispatch on physics and degree
template <class F>
cpg_status with_physics(const cpg_equation *eq, F &&f) {
    auto by_deg = [&](auto ph) -> cpg_status {
        switch (eq->degree) {
            case 1: return f(ph, std::integral_constant<int, 1>{});
            case 2: return f(ph, std::integral_constant<int, 2>{});
            case 3: return f(ph, std::integral_constant<int, 3>{});
        }
        return fail(eq->ctx, CPG_ERR_UNSUPPORTED, "degree must be 1..3");
    };
    switch (eq->physics) {
        case CPG_ADVECTION_CONST: {
            Advection<false> ph;
            ph.bx = eq->beta[0];
            ph.by = eq->beta[1];
            return by_deg(ph);
        }
        case CPG_ADVECTION_ROTATING: {
            Advection<true> ph;
            ph.bx = ph.by = 0;
            return by_deg(ph);
        }
        case CPG_EULER: {
            Euler ph;
            ph.gamma = eq->gamma;
            ph.exact = eq->exact_jacobian;
            return by_deg(ph);
        }
    }
    return fail(eq->ctx, CPG_ERR_INVALID_ARG, "unknown physics");
}

// dense inverse by Gauss-Jordan with partial pivoting (host, small blocks)
bool host_inverse(int n, const double *A, double *Ainv) {
    std::vector<double> a(A, A + (size_t)n * n);
    std::vector<double> b((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) b[(size_t)i * n + i] = 1.0;
    for (int p = 0; p < n; p++) {
        int piv = p;
        for (int r = p + 1; r < n; r++)
            if (std::fabs(a[(size_t)p * n + r]) > std::fabs(a[(size_t)p * n + piv])) piv = r;
        if (a[(size_t)p * n + piv] == 0.0) return false;
        if (piv != p)
            for (int c = 0; c < n; c++) {
                std::swap(a[(size_t)c * n + p], a[(size_t)c * n + piv]);
                std::swap(b[(size_t)c * n + p], b[(size_t)c * n + piv]);
            }
        const double d = a[(size_t)p * n + p];
        for (int c = 0; c < n; c++) {
            a[(size_t)c * n + p] /= d;
            b[(size_t)c * n + p] /= d;
        }
        for (int r = 0; r < n; r++) {
            if (r == p) continue;
            const double f = a[(size_t)p * n + r];
            if (f == 0.0) continue;
            for (int c = 0; c < n; c++) {
                a[(size_t)c * n + r] -= f * a[(size_t)c * n + p];
                b[(size_t)c * n + r] -= f * b[(size_t)c * n + p];
            }
        }
    }
    std::memcpy(Ainv, b.data(), sizeof(double) * n * n);
    return true;
}

// Gauss-Legendre nodes of order m, ascending (Newton on P_m)
std::vector<double> gauss_nodes(int m) {
    std::vector<double> x(m);
    for (int i = 0; i < m; i++) {
        long double z = std::cos(M_PI * (i + 0.75) / (m + 0.5));
        for (int it = 0; it < 60; it++) {
            long double p0 = 1, p1 = z;
            for (int k = 2; k <= m; k++) {
                long double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const long double dp = m * (z * p1 - p0) / (z * z - 1);
            const long double dz = p1 / dp;
            z -= dz;
            if (std::fabs((double)dz) < 1e-18) break;
        }
        x[m - 1 - i] = (double)z;
    }
    for (int i = 0; i < m / 2; i++) {
        const double a = 0.5 * (x[m - 1 - i] - x[i]);
        x[m - 1 - i] = a;
        x[i] = -a;
    }
    if (m % 2) x[m / 2] = 0.0;
    return x;
}

template <int P>
void host_basis(double xi, double eta, double *psi) {
    basis<P>(xi, eta, psi);
}
void host_basis_dyn(int p, double xi, double eta, double *psi) {
    if (p == 1) host_basis<1>(xi, eta, psi);
    else if (p == 2) host_basis<2>(xi, eta, psi);
    else host_basis<3>(xi, eta, psi);
}

void free_equation(cpg_equation *eq) {
    void *ptrs[] = {eq->bb, eq->vq_ptr, eq->f_ptr, eq->f_nbr, eq->f_blk, eq->vx, eq->vy, eq->vxi, eq->veta,
                    eq->vw, eq->f_nx, eq->f_ny, eq->qx, eq->qy, eq->qxi, eq->qeta, eq->qxin, eq->qetan,
                    eq->qw, eq->mass, eq->mass_inv, eq->interp_pinv, eq->rowptr_d, eq->colidx_d};
    for (void *p : ptrs) dfree(p);
}

}  // namespace

extern "C" {

cpg_status cpg_equation_create(cpg_ctx *ctx, const cpg_mesh *mm, const cpg_equation_desc *d, cpg_equation **out) {
    if (!ctx || !mm || !d || !out) return CPG_ERR_INVALID_ARG;
    *out = nullptr;
    if (d->degree < 1 || d->degree > 3) return fail(ctx, CPG_ERR_UNSUPPORTED, "degree must be 1..3");
    if (d->physics < 0 || d->physics > 2) return fail(ctx, CPG_ERR_INVALID_ARG, "unknown physics");
    const Mesh &m = cpg_mesh_ref(mm);
    cpg_equation *eq = new (std::nothrow) cpg_equation();
    if (!eq) return fail(ctx, CPG_ERR_OOM, "host allocation");
    eq->ctx = ctx;
    eq->physics = d->physics;
    eq->degree = d->degree;
    eq->nb = (d->degree + 1) * (d->degree + 2) / 2;
    eq->nc = d->physics == CPG_EULER ? 4 : 1;
    eq->bl = eq->nb * eq->nc;
    eq->n = m.n;
    eq->nqf = nqf_of(d->degree);
    eq->gamma = d->gamma;
    eq->beta[0] = d->beta[0];
    eq->beta[1] = d->beta[1];
    eq->exact_jacobian = d->exact_jacobian ? 1 : 0;
    eq->bc.dkind = d->dirichlet_kind;
    for (int q = 0; q < 8; q++) eq->bc.dparams[q] = d->dirichlet_params[q];
    for (int q = 0; q < 4; q++) eq->bc.inflow[q] = d->inflow_state[q];

    const int n = m.n, p = d->degree, nb = eq->nb, nqf = eq->nqf;
    const quad::TriRule tr = quad::tri_rule(2 * p);
    const quad::LineRule lr = quad::line_rule(2 * p);
    std::vector<double4> bb(n);
    std::vector<int> vq_ptr(n + 1, 0), f_ptr(n + 1, 0), f_nbr, f_blk;
    std::vector<double> vx, vy, vxi, veta, vw, fnx, fny, qx, qy, qxi, qeta, qxin, qetan, qw;
    std::vector<double> mass((size_t)n * nb * nb, 0.0), minv((size_t)n * nb * nb, 0.0);
    eq->rowptr.assign(1, 0);
    eq->colidx.clear();
    for (int i = 0; i < n; i++) bb[i] = make_double4(m.bb[4 * i], m.bb[4 * i + 1], m.bb[4 * i + 2], m.bb[4 * i + 3]);
    for (int i = 0; i < n; i++) {
        const double x0 = m.bb[4 * i], y0 = m.bb[4 * i + 1], w = m.bb[4 * i + 2], h = m.bb[4 * i + 3];
        // volume qp: Quadrature::polygonIntegral (Quadrature.cpp:13-57)
        for (int t = m.tri_ptr[i]; t < m.tri_ptr[i + 1]; t++) {
            const double *T = &m.tri[6 * (size_t)t];
            const double x1 = T[0], y1 = T[1], x2 = T[2], y2 = T[3], x3 = T[4], y3 = T[5];
            const double area = 0.5 * std::fabs(x1 * y2 + x2 * y3 + x3 * y1 - x1 * y3 - x3 * y2 - x2 * y1);
            for (int k = 0; k < tr.n; k++) {
                const double a = tr.p[k][0], b = tr.p[k][1];
                const double x = x1 * (1 - a - b) + x2 * a + x3 * b;
                const double y = y1 * (1 - a - b) + y2 * a + y3 * b;
                vx.push_back(x);
                vy.push_back(y);
                vxi.push_back(2.0 * (x - x0) / w - 1);
                veta.push_back(2.0 * (y - y0) / h - 1);
                vw.push_back(tr.p[k][2] * area);
            }
        }
        vq_ptr[i + 1] = (int)vx.size();
        // mass block M(k, j) = sum_q w psi_k psi_j (MassMatrix.cpp:30-94)
        double *Mi = mass.data() + (size_t)i * nb * nb;
        for (int q = vq_ptr[i]; q < vq_ptr[i + 1]; q++) {
            double psi[15];
            host_basis_dyn(p, vxi[q], veta[q], psi);
            for (int j = 0; j < nb; j++)
                for (int k = 0; k < nb; k++) Mi[j * nb + k] += vw[q] * psi[k] * psi[j];
        }
        if (!host_inverse(nb, Mi, minv.data() + (size_t)i * nb * nb)) {
            free_equation(eq);
            delete eq;
            return fail(ctx, CPG_ERR_SINGULAR_BLOCK, "singular mass block at cell " + std::to_string(i));
        }
        // Jacobian pattern row (Jacobian.cpp:7-47)
        eq->colidx.push_back(i);
        // faces: getOutwardNormal (PolyMesh.cpp:248-273) and lineIntegral
        // points (Quadrature.cpp:67-101)
        const int s = m.cell_ptr[i], nv = m.cell_ptr[i + 1] - s;
        double cx = 0, cy = 0;
        for (int k = 0; k < nv; k++) {
            cx += m.vxy[2 * (s + k)];
            cy += m.vxy[2 * (s + k) + 1];
        }
        cx /= nv;
        cy /= nv;
        for (int e = 0; e < nv; e++) {
            const int a = s + e, b = s + (e + 1) % nv;
            const double ax = m.vxy[2 * a], ay = m.vxy[2 * a + 1], bx = m.vxy[2 * b], by = m.vxy[2 * b + 1];
            const double dx = ax - bx, dy = ay - by;
            const double length = std::sqrt(dx * dx + dy * dy);
            const double sv = -dy * (ax - cx) + dx * (ay - cy);
            const int sg = (0.0 < sv) - (sv < 0.0);
            fnx.push_back(-sg * dy / length);
            fny.push_back(sg * dx / length);
            const int nbr = m.nbr[a];
            f_nbr.push_back(nbr);
            if (nbr >= 0) {
                f_blk.push_back((int)eq->colidx.size());
                eq->colidx.push_back(nbr);
            } else {
                f_blk.push_back(-1);
            }
            const double sx = m.shift[2 * a], sy = m.shift[2 * a + 1];
            const double len = std::sqrt((bx - ax) * (bx - ax) + (by - ay) * (by - ay));
            for (int k = 0; k < lr.n; k++) {
                const double xi = lr.p[k][0];
                const double x = ax + 0.5 * (xi + 1) * (bx - ax);
                const double y = ay + 0.5 * (xi + 1) * (by - ay);
                qx.push_back(x);
                qy.push_back(y);
                qxi.push_back(2.0 * (x - x0) / w - 1);
                qeta.push_back(2.0 * (y - y0) / h - 1);
                if (nbr >= 0) {
                    const double nx0 = m.bb[4 * nbr], ny0 = m.bb[4 * nbr + 1];
                    const double nw = m.bb[4 * nbr + 2], nh = m.bb[4 * nbr + 3];
                    qxin.push_back(2.0 * ((x + sx) - nx0) / nw - 1);
                    qetan.push_back(2.0 * ((y + sy) - ny0) / nh - 1);
                } else {
                    qxin.push_back(0.0);
                    qetan.push_back(0.0);
                }
                qw.push_back(lr.p[k][1] * 0.5 * len);
            }
        }
        f_ptr[i + 1] = (int)f_nbr.size();
        eq->rowptr.push_back((int)eq->colidx.size());
    }
    (void)nqf;
    eq->n_vqp = (int)vx.size();
    eq->n_faces = (int)f_nbr.size();
    // Dirichlet faces read the boundary field at time t; nothing else does
    eq->time_dependent_bc = std::count(f_nbr.begin(), f_nbr.end(), (int)CPG_BC_DIRICHLET) > 0 ? 1 : 0;
    // interpolation pseudo-inverse (MeshFn::interp, MeshFn.cpp:56-145)
    const int mq = p + 1, nq = mq * mq;
    eq->gl_nodes = gauss_nodes(mq);
    std::vector<double> G((size_t)nq * nb), pinv((size_t)nb * nq);
    for (int i = 0; i < mq; i++)
        for (int j = 0; j < mq; j++) {
            double psi[15];
            host_basis_dyn(p, eq->gl_nodes[i], eq->gl_nodes[j], psi);
            for (int k = 0; k < nb; k++) G[(size_t)(i * mq + j) * nb + k] = psi[k];
        }
    {
        // normal equations in long double: pinv = (G^T G)^{-1} G^T
        std::vector<long double> N((size_t)nb * nb, 0.0L), Ni((size_t)nb * nb, 0.0L);
        for (int a = 0; a < nb; a++)
            for (int b = 0; b < nb; b++) {
                long double s = 0;
                for (int e = 0; e < nq; e++) s += (long double)G[(size_t)e * nb + a] * G[(size_t)e * nb + b];
                N[a * nb + b] = s;
            }
        for (int a = 0; a < nb; a++) Ni[a * nb + a] = 1.0L;
        for (int c = 0; c < nb; c++) {  // SPD: Gauss-Jordan without pivoting
            const long double d = N[c * nb + c];
            for (int k = 0; k < nb; k++) {
                N[c * nb + k] /= d;
                Ni[c * nb + k] /= d;
            }
            for (int r = 0; r < nb; r++) {
                if (r == c) continue;
                const long double f = N[r * nb + c];
                for (int k = 0; k < nb; k++) {
                    N[r * nb + k] -= f * N[c * nb + k];
                    Ni[r * nb + k] -= f * Ni[c * nb + k];
                }
            }
        }
        for (int k = 0; k < nb; k++)
            for (int e = 0; e < nq; e++) {
                long double s = 0;
                for (int a = 0; a < nb; a++) s += Ni[k * nb + a] * G[(size_t)e * nb + a];
                pinv[(size_t)k * nq + e] = (double)s;
            }
    }
    cpg_status st = CPG_OK;
    auto up = [&](auto **dst, const auto &src) {
        if (st == CPG_OK) st = upload(ctx, dst, src);
    };
    up(&eq->bb, bb);
    up(&eq->vq_ptr, vq_ptr);
    up(&eq->f_ptr, f_ptr);
    up(&eq->f_nbr, f_nbr);
    up(&eq->f_blk, f_blk);
    up(&eq->vx, vx);
    up(&eq->vy, vy);
    up(&eq->vxi, vxi);
    up(&eq->veta, veta);
    up(&eq->vw, vw);
    up(&eq->f_nx, fnx);
    up(&eq->f_ny, fny);
    up(&eq->qx, qx);
    up(&eq->qy, qy);
    up(&eq->qxi, qxi);
    up(&eq->qeta, qeta);
    up(&eq->qxin, qxin);
    up(&eq->qetan, qetan);
    up(&eq->qw, qw);
    up(&eq->mass, mass);
    up(&eq->mass_inv, minv);
    up(&eq->interp_pinv, pinv);
    up(&eq->rowptr_d, eq->rowptr);
    up(&eq->colidx_d, eq->colidx);
    if (st != CPG_OK) {
        free_equation(eq);
        delete eq;
        return st;
    }
    // ILU(0) level counts of the pattern (for information)
    {
        std::vector<int> lv(n, 0), uv(n, 0);
        int nl = 0, nu = 0;
        for (int j = 0; j < n; j++) {
            int l = 0;
            for (int k = eq->rowptr[j]; k < eq->rowptr[j + 1]; k++)
                if (eq->colidx[k] < j) l = std::max(l, lv[eq->colidx[k]] + 1);
            lv[j] = l;
            nl = std::max(nl, l + 1);
        }
        for (int i = n - 1; i >= 0; i--) {
            int l = 0;
            for (int k = eq->rowptr[i]; k < eq->rowptr[i + 1]; k++)
                if (eq->colidx[k] > i) l = std::max(l, uv[eq->colidx[k]] + 1);
            uv[i] = l;
            nu = std::max(nu, l + 1);
        }
        eq->levels_lower = nl;
        eq->levels_upper = nu;
    }
    *out = eq;
    return CPG_OK;
}

void cpg_equation_destroy(cpg_equation *eq) {
    if (!eq) return;
    // cudaFree synchronizes the device; the context may already be gone
    free_equation(eq);
    delete eq;
}

cpg_status cpg_equation_get_info(const cpg_equation *eq, cpg_equation_info *info) {
    if (!eq || !info) return CPG_ERR_INVALID_ARG;
    info->n_cells = eq->n;
    info->nb = eq->nb;
    info->nc = eq->nc;
    info->bl = eq->bl;
    info->n_dof = (int64_t)eq->n * eq->bl;
    info->nnzb = (int64_t)eq->colidx.size();
    info->n_vqp = eq->n_vqp;
    info->n_faces = eq->n_faces;
    info->nqf = eq->nqf;
    info->levels_lower = eq->levels_lower;
    info->levels_upper = eq->levels_upper;
    return CPG_OK;
}

// Equation::assemble (Equation.cpp:152-191) as seen from the C ABI: the
// residual, then -- outside stream capture -- a read of the state word, so
// that a non-physical state is reported by the call that met it.  The
// steppers launch the kernel alone (assemble_raw) and read the word at the
// synchronisation their Newton norms make anyway.
cpg_status cpg_assemble(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double t, double *b) {
    if (!ctx || !eq || !u || !b) return CPG_ERR_INVALID_ARG;
    CPG_TRY(assemble_raw(ctx, eq, u, t, b));
    if (ctx->deferred_checks) return CPG_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CPG_CUDA(ctx, cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return CPG_OK;
    return check_state(ctx, "residual");
}

cpg_status cpg_jacobian(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double t, double scale, int add_mass,
                        cpg_bsr *J) {
    if (!ctx || !eq || !u || !J) return CPG_ERR_INVALID_ARG;
    if (J->n_rows != eq->n || J->bl != eq->bl || J->nnzb != (int64_t)eq->colidx.size())
        return fail(ctx, CPG_ERR_INVALID_ARG, "Jacobian matrix does not have the equation's pattern");
    return with_physics(eq, [&](auto ph, auto pc) -> cpg_status {
        constexpr int P = decltype(pc)::value;
        if (J->precision == CPG_F32) {
            k_jacobian<decltype(ph), P, float><<<eq->n, JT, 0, ctx->stream>>>(
                eq->geo(), ph, eq->bc, u, t, scale, add_mass, eq->mass, eq->rowptr_d, (float *)J->vals);
        } else {
            k_jacobian<decltype(ph), P, double><<<eq->n, JT, 0, ctx->stream>>>(
                eq->geo(), ph, eq->bc, u, t, scale, add_mass, eq->mass, eq->rowptr_d, (double *)J->vals);
        }
        bsr_touch(J);
        return launched(ctx, "jacobian kernel");
    });
}

static cpg_status mass_op(cpg_ctx *ctx, const cpg_equation *eq, const double *Mi, const double *x, double alpha,
                          const double *z, double beta, double *y) {
    const int64_t N = (int64_t)eq->n * eq->bl;
    const int T = 256;
    const int grid = (int)((N + T - 1) / T);
    switch (eq->nb) {
        case 3: k_mass<3><<<grid, T, 0, ctx->stream>>>(eq->n, eq->nc, Mi, x, alpha, z, beta, y, ctx->skip_dev); break;
        case 6: k_mass<6><<<grid, T, 0, ctx->stream>>>(eq->n, eq->nc, Mi, x, alpha, z, beta, y, ctx->skip_dev); break;
        case 10: k_mass<10><<<grid, T, 0, ctx->stream>>>(eq->n, eq->nc, Mi, x, alpha, z, beta, y, ctx->skip_dev); break;
        default: return fail(ctx, CPG_ERR_UNSUPPORTED, "basis size");
    }
    return launched(ctx, "mass kernel");
}

cpg_status cpg_mass_apply(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double *y) {
    if (!ctx || !eq || !x || !y) return CPG_ERR_INVALID_ARG;
    return mass_op(ctx, eq, eq->mass, x, 1.0, nullptr, 0.0, y);
}

cpg_status cpg_mass_solve(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double *y) {
    if (!ctx || !eq || !x || !y) return CPG_ERR_INVALID_ARG;
    return mass_op(ctx, eq, eq->mass_inv, x, 1.0, nullptr, 0.0, y);
}

cpg_status cpg_mass_export(cpg_ctx *ctx, const cpg_equation *eq, double *mass_host) {
    if (!ctx || !eq || !mass_host) return CPG_ERR_INVALID_ARG;
    CPG_CUDA(ctx, cudaMemcpyAsync(mass_host, eq->mass, sizeof(double) * eq->n * eq->nb * eq->nb,
                                  cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CPG_OK;
}

cpg_status cpg_l2norm(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double *out_host) {
    if (!ctx || !eq || !u || !out_host) return CPG_ERR_INVALID_ARG;
    double *part, *hp;
    CPG_TRY(scratch(ctx, RED_CTAS * 4 + 4, &part));
    CPG_TRY(pinned(ctx, 4, &hp));
    switch (eq->nb) {
        case 3: k_l2_partial<3><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
        case 6: k_l2_partial<6><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
        case 10: k_l2_partial<10><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
        default: return fail(ctx, CPG_ERR_UNSUPPORTED, "basis size");
    }
    CPG_TRY(launched(ctx, "l2 partial kernel"));
    k_l2_final<<<1, 32, 0, ctx->stream>>>(RED_CTAS, part, part + RED_CTAS * 4);
    CPG_TRY(launched(ctx, "l2 final kernel"));
    CPG_CUDA(ctx, cudaMemcpyAsync(hp, part + RED_CTAS * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < eq->nc; c++) {
        if (!std::isfinite(hp[c])) return fail(ctx, CPG_ERR_NONFINITE, "non-finite L2 norm");
        out_host[c] = std::sqrt(std::max(0.0, hp[c]));
    }
    return CPG_OK;
}

cpg_status cpg_l2error(cpg_ctx *ctx, const cpg_equation *eq, const double *u, int kind, const double *params,
                       double t, double *out_host) {
    if (!ctx || !eq || !u || !out_host || kind < 0 || kind > 3) return CPG_ERR_INVALID_ARG;
    BCParams prm{};
    for (int q = 0; q < 8; q++) prm.dparams[q] = params ? params[q] : 0.0;
    double *part, *hp;
    CPG_TRY(scratch(ctx, RED_CTAS * 4 + 4, &part));
    CPG_TRY(pinned(ctx, 4, &hp));
    const Geo g = eq->geo();
    auto launch = [&](auto pc) {
        constexpr int P = decltype(pc)::value;
        if (eq->nc == 4) k_l2_error_partial<P, 4><<<RED_CTAS, 256, 0, ctx->stream>>>(g, kind, prm, t, u, part);
        else k_l2_error_partial<P, 1><<<RED_CTAS, 256, 0, ctx->stream>>>(g, kind, prm, t, u, part);
    };
    switch (eq->degree) {
        case 1: launch(std::integral_constant<int, 1>{}); break;
        case 2: launch(std::integral_constant<int, 2>{}); break;
        case 3: launch(std::integral_constant<int, 3>{}); break;
        default: return fail(ctx, CPG_ERR_UNSUPPORTED, "degree must be 1..3");
    }
    CPG_TRY(launched(ctx, "l2 error kernel"));
    k_l2_final<<<1, 32, 0, ctx->stream>>>(RED_CTAS, part, part + RED_CTAS * 4);
    CPG_TRY(launched(ctx, "l2 final kernel"));
    CPG_CUDA(ctx, cudaMemcpyAsync(hp, part + RED_CTAS * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < eq->nc; c++) {
        if (!std::isfinite(hp[c])) return fail(ctx, CPG_ERR_NONFINITE, "non-finite L2 error");
        out_host[c] = std::sqrt(std::max(0.0, hp[c]));
    }
    return CPG_OK;
}

cpg_status cpg_interp(cpg_ctx *ctx, const cpg_equation *eq, int kind, const double *params, double t, double *u) {
    if (!ctx || !eq || !u || kind < 0 || kind > 3) return CPG_ERR_INVALID_ARG;
    BCParams prm{};
    for (int q = 0; q < 8; q++) prm.dparams[q] = params ? params[q] : 0.0;
    // node table lives in the scratch buffer
    double *gl;
    CPG_TRY(scratch(ctx, 16, &gl));
    CPG_CUDA(ctx, cudaMemcpyAsync(gl, eq->gl_nodes.data(), sizeof(double) * eq->gl_nodes.size(),
                                  cudaMemcpyHostToDevice, ctx->stream));
    const int T = 128, grid = (eq->n + T - 1) / T;
    if (eq->nc == 4)
        k_interp<4><<<grid, T, 0, ctx->stream>>>(eq->n, eq->nb, eq->degree + 1, eq->bb, gl, eq->interp_pinv, kind,
                                                 prm, t, u);
    else
        k_interp<1><<<grid, T, 0, ctx->stream>>>(eq->n, eq->nb, eq->degree + 1, eq->bb, gl, eq->interp_pinv, kind,
                                                 prm, t, u);
    CPG_TRY(launched(ctx, "interp kernel"));
    // the node table copy above is asynchronous from pageable memory of a
    // long-lived vector; synchronize so the scratch buffer may be reused
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return CPG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// L2 norm without any allocation.
//
// cpg_l2norm keeps its partial sums in the context's scratch buffer and reads
// the result back through a pinned host buffer; both are allocated (or grown)
// on demand.  A caller that hands all of the device memory to its own pool --
// the serving loop, for instance, admits each solve against a fixed memory
// budget -- or that may not allocate inside its Newton loop can use
// cpg_l2norm_noalloc instead: its partial sums live in the file-scope device
// array below, which every GPU that loads this library holds until the
// process exits, and the result is copied straight into the caller's host
// array.
// ---------------------------------------------------------------------------
namespace {
constexpr int L2_NOALLOC_MAX_NC = 4;  // components a call may reduce
// 4 partial-sum slots per reduction CTA (k_l2_partial) plus the 4 totals
constexpr int L2_NOALLOC_DOUBLES = RED_CTAS * 4 + 4;  // 1028 doubles, 8224 bytes
static __device__ __align__(256) double g_l2_noalloc[L2_NOALLOC_DOUBLES];
std::mutex g_l2_noalloc_mu;
double *g_l2_noalloc_addr[128] = {};  // device address of the array, per device
}  // namespace

extern "C" cpg_status cpg_l2norm_noalloc(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double *out_host) {
    if (!ctx || !eq || !u || !out_host) return CPG_ERR_INVALID_ARG;
    const size_t need = (size_t)RED_CTAS * 4 + (size_t)eq->nc;
    if (eq->nc > L2_NOALLOC_MAX_NC || need > (size_t)L2_NOALLOC_DOUBLES)
        return fail(ctx, CPG_ERR_INVALID_ARG,
                    "cpg_l2norm_noalloc: " + std::to_string(eq->nc) + " components need " + std::to_string(need) +
                        " doubles of static scratch; the maximum is " + std::to_string(L2_NOALLOC_DOUBLES) +
                        " doubles (" + std::to_string(L2_NOALLOC_MAX_NC) + " components)");
    if (eq->nb != 3 && eq->nb != 6 && eq->nb != 10) return fail(ctx, CPG_ERR_UNSUPPORTED, "basis size");
    int dev = -1;
    CPG_CUDA(ctx, cudaGetDevice(&dev));
    if (dev != ctx->device || dev < 0 || dev >= 128)
        return fail(ctx, CPG_ERR_INVALID_ARG, "cpg_l2norm_noalloc: make the context's device current");
    double *part = nullptr;
    {
        // set-up, once per device, with that device current: the host-side
        // name of the array is not a device address
        std::lock_guard<std::mutex> lock(g_l2_noalloc_mu);
        if (!g_l2_noalloc_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_l2_noalloc);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress of the static norm scratch");
            g_l2_noalloc_addr[dev] = (double *)p;
        }
        part = g_l2_noalloc_addr[dev];
    }
    // every slot read below is written earlier in the same call, so nothing
    // needs clearing; calls that overlap on the GPU share the array and race
    switch (eq->nb) {
        case 3: k_l2_partial<3><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
        case 6: k_l2_partial<6><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
        default: k_l2_partial<10><<<RED_CTAS, 256, 0, ctx->stream>>>(eq->n, eq->nc, eq->mass, u, part); break;
    }
    CPG_TRY(launched(ctx, "l2 partial kernel (static scratch)"));
    k_l2_final<<<1, 32, 0, ctx->stream>>>(RED_CTAS, part, part + RED_CTAS * 4);
    CPG_TRY(launched(ctx, "l2 final kernel (static scratch)"));
    double sums[L2_NOALLOC_MAX_NC];
    CPG_CUDA(ctx, cudaMemcpyAsync(sums, part + RED_CTAS * 4, sizeof(double) * eq->nc, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    CPG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (int c = 0; c < eq->nc; c++) {
        if (!std::isfinite(sums[c])) return fail(ctx, CPG_ERR_NONFINITE, "non-finite L2 norm");
        out_host[c] = std::sqrt(std::max(0.0, sums[c]));
    }
    return CPG_OK;
}

namespace cpg {
cpg_status assemble_raw(cpg_ctx *ctx, const cpg_equation *eq, const double *u, double t, double *b) {
    return with_physics(eq, [&](auto ph, auto pc) -> cpg_status {
        constexpr int P = decltype(pc)::value;
        const int cells_per_cta = 4;
        const int grid = (eq->n + cells_per_cta - 1) / cells_per_cta;
        k_residual<decltype(ph), P><<<grid, 32 * cells_per_cta, 0, ctx->stream>>>(eq->geo(), ph, eq->bc, u, t, b,
                                                                                  ctx->flag_dev + FLAG_NONPHYS);
        return launched(ctx, "residual kernel");
    });
}
// y = alpha * M x + beta * z (Newton residual r = M k - dt b)
cpg_status mass_apply_axpy(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double alpha, const double *z,
                           double beta, double *y) {
    return mass_op(ctx, eq, eq->mass, x, alpha, z, beta, y);
}
// y = alpha * M^{-1} x
cpg_status mass_solve_scaled(cpg_ctx *ctx, const cpg_equation *eq, const double *x, double alpha, double *y) {
    return mass_op(ctx, eq, eq->mass_inv, x, alpha, nullptr, 0.0, y);
}
}  // namespace cpg
