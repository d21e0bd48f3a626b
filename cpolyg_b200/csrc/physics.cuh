// Device physics functors: the four pure virtuals of Equation
// (src/Equation.h:46-51) as compile-time functors, plus boundary states.
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace cpg {

// analytic fields for initial data and Dirichlet states (cpg_init_kind)
template <int NC>
__host__ __device__ inline void field_eval(int kind, const double *P, double x, double y, double t,
                                           double *out) {
    if (kind == CPG_INIT_CONSTANT) {
        for (int c = 0; c < NC; c++) out[c] = P[c];
    } else if (kind == CPG_INIT_GAUSSIAN) {
        // centre (x0, y0) + (bx, by) t, nearest periodic image when Lx, Ly > 0
        double dx = x - (P[1] + P[3] * t), dy = y - (P[2] + P[4] * t);
        if (P[5] > 0) dx -= P[5] * round(dx / P[5]);
        if (P[6] > 0) dy -= P[6] * round(dy / P[6]);
        out[0] = exp(-P[0] * (dx * dx + dy * dy));
        for (int c = 1; c < NC; c++) out[c] = 0.0;
    } else if (kind == CPG_INIT_VORTEX) {
        // isentropic vortex of strength beta (Shu), nearest periodic image
        const double beta = P[0], x0 = P[1], y0 = P[2], ui = P[3], vi = P[4], g = P[5];
        const double Lx = P[6], Ly = P[7];
        double dx = x - (x0 + ui * t), dy = y - (y0 + vi * t);
        if (Lx > 0) dx -= Lx * round(dx / Lx);
        if (Ly > 0) dy -= Ly * round(dy / Ly);
        const double r2 = dx * dx + dy * dy;
        const double e = exp(0.5 * (1.0 - r2));
        const double du = -beta / (2.0 * M_PI) * dy * e;
        const double dv = beta / (2.0 * M_PI) * dx * e;
        const double T = 1.0 - (g - 1.0) * beta * beta / (8.0 * g * M_PI * M_PI) * e * e;
        const double rho = pow(T, 1.0 / (g - 1.0));
        const double p = pow(rho, g);
        const double u = ui + du, v = vi + dv;
        if (NC >= 4) {
            out[0] = rho;
            out[1] = rho * u;
            out[2] = rho * v;
            out[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
        } else {
            out[0] = rho;
        }
    } else {  // CPG_INIT_DENSITY_BUMP
        const double A = P[0], w = P[1], x0 = P[2], y0 = P[3], mach = P[4], g = P[5];
        const double dx = x - x0, dy = y - y0;
        const double rho = 1.0 + A * exp(-(dx * dx + dy * dy) / (w * w));
        const double p = 1.0 / g, u = mach;
        if (NC >= 4) {
            out[0] = rho;
            out[1] = rho * u;
            out[2] = 0.0;
            out[3] = p / (g - 1.0) + 0.5 * rho * u * u;
        } else {
            out[0] = rho;
        }
    }
}

struct BCParams {
    int dkind;
    double dparams[8];
    double inflow[4];
};

// Linear advection with constant (CONST) or rotating velocity
// (eqns/Advection.cpp:8-66)
template <bool ROT>
struct Advection {
    static constexpr int NC = 1;
    double bx, by;
    __device__ __forceinline__ double betaX(double x, double y) const { return ROT ? 2 * y - 1 : bx; }
    __device__ __forceinline__ double betaY(double x, double y) const { return ROT ? -2 * x + 1 : by; }
    __device__ __forceinline__ void flux(const double *U, double x, double y, double *Fx, double *Fy) const {
        Fx[0] = betaX(x, y) * U[0];
        Fy[0] = betaY(x, y) * U[0];
    }
    __device__ __forceinline__ void numflux(const double *Um, const double *Up, double x, double y, double nx,
                                            double ny, double *F) const {
        const double bn = betaX(x, y) * nx + betaY(x, y) * ny;
        F[0] = bn > 0 ? Um[0] * bn : Up[0] * bn;
    }
    __device__ __forceinline__ void fluxjac(const double *U, double x, double y, double *Ax, double *Ay) const {
        Ax[0] = betaX(x, y);
        Ay[0] = betaY(x, y);
    }
    // J[r*NC + c]
    __device__ __forceinline__ void numfluxjac(const double *U, const double *U2, double x, double y, double nx,
                                               double ny, int sgn, double *J) const {
        const double bn = nx * betaX(x, y) + ny * betaY(x, y);
        J[0] = (sgn * bn > 0) ? bn : 0.0;
    }
    // every finite scalar is an admissible state
    __device__ __forceinline__ bool admissible(const double *U) const { return true; }
    __device__ __forceinline__ void wall(const double *Um, double nx, double ny, double *Up) const { Up[0] = Um[0]; }
    __device__ __forceinline__ void wall_deriv(double nx, double ny, double *R) const { R[0] = 1.0; }
};

// 2D Euler, Rusanov flux (eqns/Euler.cpp:7-179)
struct Euler {
    static constexpr int NC = 4;
    double gamma;
    // 0: the reference's flux Jacobians (entry (3,1) of A_x reads
    //    H - (g-1)(u^2+v^2), Euler.cpp:154-163; neighbour blocks use the own
    //    state, Euler.cpp:168-179); 1: exact derivatives (H - (g-1) u^2, and
    //    A(u2), d alpha/d u2 for the neighbour blocks)
    int exact;
    __device__ __forceinline__ void eflux(const double *U, double *fx, double *fy, double &c, double &u,
                                          double &v) const {
        const double rho = U[0], rhoU = U[1], rhoV = U[2], rhoE = U[3];
        u = rhoU / rho;
        v = rhoV / rho;
        const double P = (gamma - 1) * (rhoE - 0.5 * (rhoU * rhoU + rhoV * rhoV) / rho);
        fx[0] = rhoU;
        fx[1] = rhoU * u + P;
        fx[2] = rhoU * v;
        fx[3] = (rhoE + P) * u;
        fy[0] = rhoV;
        fy[1] = rhoU * v;
        fy[2] = rhoV * v + P;
        fy[3] = (rhoE + P) * v;
        c = sqrt(gamma * P / rho);
    }
    __device__ __forceinline__ void flux(const double *U, double x, double y, double *Fx, double *Fy) const {
        double c, u, v;
        eflux(U, Fx, Fy, c, u, v);
    }
    __device__ __forceinline__ void numflux(const double *Um, const double *Up, double x, double y, double nx,
                                            double ny, double *F) const {
        double fxm[4], fym[4], fxp[4], fyp[4], cm, um, vm, cp, up, vp;
        eflux(Um, fxm, fym, cm, um, vm);
        eflux(Up, fxp, fyp, cp, up, vp);
        const double vnm = um * nx + vm * ny, vnp = up * nx + vp * ny;
        // fmax returns its other operand for a NaN one, so a NaN sound speed
        // (negative pressure) would vanish from alpha; adding 0*(cm+cp)
        // carries it into the flux and leaves every finite alpha unchanged
        const double alpha = fmax(fmax(fmax(fabs(vnm - cm), fabs(vnm)), fmax(fabs(vnm + cm), fabs(vnp - cp))),
                                  fmax(fabs(vnp), fabs(vnp + cp))) +
                             0.0 * (cm + cp);
#pragma unroll
        for (int k = 0; k < 4; k++)
            F[k] = 0.5 * ((fxp[k] + fxm[k]) * nx + (fyp[k] + fym[k]) * ny + alpha * (Um[k] - Up[k]));
    }
    // Ax, Ay row-major 4x4 (Euler.cpp:134-166)
    __device__ __forceinline__ void fluxjac(const double *U, double x, double y, double *A0, double *A1) const {
        const double g = gamma, rho = U[0];
        const double u = U[1] / rho, v = U[2] / rho, E = U[3] / rho;
        const double usq = u * u + v * v, e = E - 0.5 * usq, P = (g - 1) * rho * e, H = E + P / rho;
        A0[0] = 0; A0[1] = 1; A0[2] = 0; A0[3] = 0;
        A0[4] = -u * u + 0.5 * (g - 1) * usq; A0[5] = (3 - g) * u; A0[6] = -(g - 1) * v; A0[7] = g - 1;
        A0[8] = -u * v; A0[9] = v; A0[10] = u; A0[11] = 0;
        A0[12] = u * (0.5 * (g - 1) * usq - H); A0[13] = H - (g - 1) * usq; A0[14] = -(g - 1) * u * v; A0[15] = g * u;
        A1[0] = 0; A1[1] = 0; A1[2] = 1; A1[3] = 0;
        A1[4] = -u * v; A1[5] = v; A1[6] = u; A1[7] = 0;
        A1[8] = -v * v + 0.5 * (g - 1) * usq; A1[9] = -(g - 1) * u; A1[10] = (3 - g) * v; A1[11] = g - 1;
        A1[12] = v * (0.5 * (g - 1) * usq - H); A1[13] = -(g - 1) * u * v; A1[14] = H - (g - 1) * v * v; A1[15] = g * v;
        if (exact) A0[13] = H - (g - 1) * u * u;
    }
    // alphaDerivative (Euler.cpp:35-98)
    __device__ __forceinline__ void alpha_der(const double *v1s, const double *v2s, double nx, double ny,
                                              double *der, double &alpha) const {
        const double g = gamma;
        der[0] = der[1] = der[2] = der[3] = 0.0;
        const double u1 = v1s[1] / v1s[0], v1 = v1s[2] / v1s[0];
        const double u2 = v2s[1] / v2s[0], v2 = v2s[2] / v2s[0];
        const double P1 = (g - 1) * (v1s[3] - 0.5 * (v1s[1] * v1s[1] + v1s[2] * v1s[2]) / v1s[0]);
        const double c1 = sqrt(g * P1 / v1s[0]);
        const double P2 = (g - 1) * (v2s[3] - 0.5 * (v2s[1] * v2s[1] + v2s[2] * v2s[2]) / v2s[0]);
        const double c2 = sqrt(g * P2 / v2s[0]);
        const double vn1 = u1 * nx + v1 * ny, vn2 = u2 * nx + v2 * ny;
        const double eigs[6] = {vn1 - c1, vn1, vn1 + c1, vn2 - c2, vn2, vn2 + c2};
        int idx = 0;
        alpha = fabs(eigs[0]);
#pragma unroll
        for (int k = 1; k < 6; k++)
            if (fabs(eigs[k]) > alpha) {
                alpha = fabs(eigs[k]);
                idx = k;
            }
        if (idx <= 2) {
            const double rho = v1s[0], E = v1s[3] / rho;
            der[0] = -u1 / rho * nx - v1 / rho * ny;
            der[1] = 1 / rho * nx;
            der[2] = 1 / rho * ny;
            const double usq = u1 * u1 + v1 * v1;
            const double a = sqrt(g * g - g), b = rho * sqrt(4 * E - 2 * usq);
            if (idx == 0) {
                der[0] -= a * (usq - E) / b;
                der[1] -= -a * u1 / b;
                der[2] -= -a * v1 / b;
                der[3] -= a / b;
            } else if (idx == 2) {
                der[0] += a * (usq - E) / b;
                der[1] += -a * u1 / b;
                der[2] += -a * v1 / b;
                der[3] += a / b;
            }
            if (eigs[idx] < 0) {
                der[0] = -der[0];
                der[1] = -der[1];
                der[2] = -der[2];
                der[3] = -der[3];
            }
        }
    }
    // numericalFluxJacobian (Euler.cpp:168-179), J[r*4+c]
    __device__ __forceinline__ void numfluxjac(const double *U, const double *U2, double x, double y, double nx,
                                               double ny, int sgn, double *J) const {
        double A0[16], A1[16], ap[4], alpha;
        if (sgn < 0 && exact) {  // derivative with respect to the neighbour state
            fluxjac(U2, x, y, A0, A1);
            alpha_der(U2, U, nx, ny, ap, alpha);
        } else {
            fluxjac(U, x, y, A0, A1);
            alpha_der(U, U2, nx, ny, ap, alpha);
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
            for (int c = 0; c < 4; c++)
                J[r * 4 + c] = 0.5 * (A0[r * 4 + c] * nx + A1[r * 4 + c] * ny + (r == c ? sgn * alpha : 0.0) +
                                      (U[r] - U2[r]) * ap[c]);
    }
    // positive density and pressure (false for NaN as well)
    __device__ __forceinline__ bool admissible(const double *U) const {
        const double rho = U[0];
        const double P = (gamma - 1) * (U[3] - 0.5 * (U[1] * U[1] + U[2] * U[2]) / rho);
        return rho > 0.0 && P > 0.0 && P < INFINITY;
    }
    __device__ __forceinline__ void wall(const double *Um, double nx, double ny, double *Up) const {
        const double mn = Um[1] * nx + Um[2] * ny;
        Up[0] = Um[0];
        Up[1] = Um[1] - 2 * mn * nx;
        Up[2] = Um[2] - 2 * mn * ny;
        Up[3] = Um[3];
    }
    __device__ __forceinline__ void wall_deriv(double nx, double ny, double *R) const {
#pragma unroll
        for (int q = 0; q < 16; q++) R[q] = (q % 5 == 0) ? 1.0 : 0.0;
        R[5] = 1 - 2 * nx * nx;
        R[6] = -2 * nx * ny;
        R[9] = -2 * nx * ny;
        R[10] = 1 - 2 * ny * ny;
    }
};

// exterior state u+ for a boundary code (BoundaryConditions::boundaryValue,
// src/BoundaryConditions.cpp:7-37, extended with wall / outflow / inflow)
template <class Phys>
__device__ __forceinline__ void boundary_state(const Phys &ph, const BCParams &bc, int code, const double *Um,
                                               double x, double y, double t, double nx, double ny, double *Up) {
    constexpr int NC = Phys::NC;
    if (code == CPG_BC_WALL) {
        ph.wall(Um, nx, ny, Up);
    } else if (code == CPG_BC_OUTFLOW) {
#pragma unroll
        for (int c = 0; c < NC; c++) Up[c] = Um[c];
    } else if (code == CPG_BC_INFLOW) {
#pragma unroll
        for (int c = 0; c < NC; c++) Up[c] = bc.inflow[c];
    } else {
        field_eval<NC>(bc.dkind, bc.dparams, x, y, t, Up);
    }
}

}  // namespace cpg
