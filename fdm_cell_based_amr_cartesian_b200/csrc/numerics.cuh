// numerics.cuh — FP64 device numerics of the WCNS residual and the
// hanging-node WLS-WENO interpolation.
//
// The exact variant of libfdm compiles this with -fmad=false so that every
// product and sum is rounded as written: the evaluation order below is the
// reference's (left to right, parentheses as in the Fortran), and default
// REAL(4) literals carry their promoted values.  Products with a structural
// 0 of the eigenvector matrices are left out; for finite operands that only
// changes the sign of an exact zero.
#pragma once
#include "fdm_common.cuh"

namespace fdm {

// REAL(4) literals promoted to REAL(8) (src/nnd_center_RK.F90:319, 331)
#define FDM_EPS_WCNS 9.99994610111476e-41          /* 1.e-40  */
#define FDM_D1_WCNS 0.09090909361839294            /* 1./11.  */
#define FDM_D2_WCNS 0.9090909361839294             /* 10./11. */

struct Prim { double r, u, v, p; };

// ---------------------------------------------------- division policies
// Every division of the face flux goes through a policy object.  DivIEEE
// divides as written (the compiler's correctly rounded division); DivNR
// (numerics_nr.cuh) forms the same correctly rounded quotients without
// branches.  A Den is a denominator with its reciprocal where the policy
// uses one; gm1 = gama - 1 and d2 of WCNS_Z3 are the constant denominators.
struct Den {
    double b, y;
};
struct DivIEEE {
    Den gm1, d2;
    __device__ __forceinline__ explicit DivIEEE(double g) : gm1{g - 1.0, 0.0}, d2{FDM_D2_WCNS, 0.0} {}
    __device__ __forceinline__ Den den(double b) const { return Den{b, 0.0}; }
    __device__ __forceinline__ double q(double a, const Den &d) const { return a / d.b; }
    __device__ __forceinline__ double q(double a, double b) const { return a / b; }
};

__device__ __forceinline__ Prim load_prim(const double4 *__restrict__ s, int64_t i) {
    const double4 q = s[i];
    return Prim{q.x, q.y, q.z, q.w};
}

// conserved variables and the physical flux of one point
// (compute_E / compute_F, src/nnd_center_RK.F90:171-185, 293-307)
template <int DIR, class D>
__device__ __forceinline__ void cons_flux_d(const Prim &q, D &dv, double U[4], double F[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    U[0] = q.r;
    U[1] = q.r * q.u;
    U[2] = q.r * q.v;
    U[3] = dv.q(q.p, dv.gm1) + 0.5 * q.r * ke;
    if (DIR == 0) {
        F[0] = q.r * q.u;
        F[1] = q.r * q.u * q.u + q.p;
        F[2] = q.r * q.u * q.v;
        F[3] = q.u * (dv.q(q.p, dv.gm1) + 0.5 * q.r * ke + q.p);
    } else {
        F[0] = q.r * q.v;
        F[1] = q.r * q.u * q.v;
        F[2] = q.r * q.v * q.v + q.p;
        F[3] = q.v * (dv.q(q.p, dv.gm1) + 0.5 * q.r * ke + q.p);
    }
}
template <int DIR>
__device__ __forceinline__ void cons_flux(const Prim &q, double g, double U[4], double F[4]) {
    DivIEEE dv(g);
    cons_flux_d<DIR>(q, dv, U, F);
}
template <int DIR>
__device__ __forceinline__ void phys_flux(const Prim &q, double g, double F[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    if (DIR == 0) {
        F[0] = q.r * q.u;
        F[1] = q.r * q.u * q.u + q.p;
        F[2] = q.r * q.u * q.v;
        F[3] = q.u * (q.p / (g - 1.0) + 0.5 * q.r * ke + q.p);
    } else {
        F[0] = q.r * q.v;
        F[1] = q.r * q.u * q.v;
        F[2] = q.r * q.v * q.v + q.p;
        F[3] = q.v * (q.p / (g - 1.0) + 0.5 * q.r * ke + q.p);
    }
}

// Characteristic basis at a face (REcalc / RFcalc,
// src/nnd_center_RK.F90:114-169, 236-291), kept in the few scalars the
// structured matrices need.
struct Eig {
    double u, v, a, q2, H1, H2;   // H1 = a*a/(g-1)+q2-(u|v)*a, H2 = ...+(u|v)*a
    double Ri[4][4];
};

template <int DIR, class D>
__device__ __forceinline__ void eigen_d(const double Um[4], double g, D &dv, Eig &E) {
    const double r0 = Um[0];
    const Den dr = dv.den(Um[0]);
    const double u = dv.q(Um[1], dr);
    const double v = dv.q(Um[2], dr);
    const double p = (g - 1.0) * r0 * (dv.q(Um[3], dr) - 0.5 * (u * u + v * v));
    const double a = sqrt(dv.q(g * p, dr));
    const double q2 = 0.5 * (u * u + v * v);
    const double aa = a * a, a2 = 2.0 * a * a;
    const Den daa = dv.den(aa), da2 = dv.den(a2);
    E.u = u; E.v = v; E.a = a; E.q2 = q2;
    const double c = DIR == 0 ? u : v;
    E.H1 = dv.q(a * a, dv.gm1) + q2 - c * a;
    E.H2 = dv.q(a * a, dv.gm1) + q2 + c * a;
    if (DIR == 0) {
        E.Ri[0][0] = dv.q((g - 1.0) * q2 + a * u, da2);
        E.Ri[1][0] = dv.q(aa - (g - 1.0) * q2, daa);
        E.Ri[2][0] = dv.q((g - 1.0) * q2 - a * u, da2);
        E.Ri[3][0] = v;
        E.Ri[0][1] = dv.q((1.0 - g) * u - a, da2);
        E.Ri[1][1] = dv.q((g - 1.0) * u, daa);
        E.Ri[2][1] = dv.q((1.0 - g) * u + a, da2);
        E.Ri[3][1] = 0.0;
        E.Ri[0][2] = dv.q((1.0 - g) * v, da2);
        E.Ri[1][2] = dv.q((g - 1.0) * v, daa);
        E.Ri[2][2] = dv.q((1.0 - g) * v, da2);
        E.Ri[3][2] = -1.0;
    } else {
        E.Ri[0][0] = dv.q((g - 1.0) * q2 + a * v, da2);
        E.Ri[1][0] = dv.q(aa - (g - 1.0) * q2, daa);
        E.Ri[2][0] = dv.q((g - 1.0) * q2 - a * v, da2);
        E.Ri[3][0] = -u;
        E.Ri[0][1] = dv.q((1.0 - g) * u, da2);
        E.Ri[1][1] = dv.q((g - 1.0) * u, daa);
        E.Ri[2][1] = dv.q((1.0 - g) * u, da2);
        E.Ri[3][1] = 1.0;
        E.Ri[0][2] = dv.q((1.0 - g) * v - a, da2);
        E.Ri[1][2] = dv.q((g - 1.0) * v, daa);
        E.Ri[2][2] = dv.q((1.0 - g) * v + a, da2);
        E.Ri[3][2] = 0.0;
    }
    E.Ri[0][3] = dv.q(g - 1.0, da2);
    E.Ri[1][3] = dv.q(1.0 - g, daa);
    E.Ri[2][3] = dv.q(g - 1.0, da2);
    E.Ri[3][3] = 0.0;
}
template <int DIR>
__device__ __forceinline__ void eigen(const double Um[4], double g, Eig &E) {
    DivIEEE dv(g);
    eigen_d<DIR>(Um, g, dv, E);
}

// w = Ri * X (one column), MATMUL order; the 4th row of Ri is sparse
template <int DIR>
__device__ __forceinline__ void project(const Eig &E, const double X[4], double w[4]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
        w[r] = E.Ri[r][0] * X[0] + E.Ri[r][1] * X[1] + E.Ri[r][2] * X[2] + E.Ri[r][3] * X[3];
    if (DIR == 0) w[3] = E.Ri[3][0] * X[0] + -X[2];
    else w[3] = E.Ri[3][0] * X[0] + X[1];
}

// hp = R * uL (WCNS_Z3 lines :349-352) with the structured R of REcalc/RFcalc
template <int DIR>
__device__ __forceinline__ void back_project(const Eig &E, const double uL[4], double hp[4]) {
    hp[0] = uL[0] + uL[1] + uL[2];
    if (DIR == 0) {
        hp[1] = (E.u - E.a) * uL[0] + E.u * uL[1] + (E.u + E.a) * uL[2];
        hp[2] = E.v * uL[0] + E.v * uL[1] + E.v * uL[2] + -uL[3];
        hp[3] = E.H1 * uL[0] + E.q2 * uL[1] + E.H2 * uL[2] + -E.v * uL[3];
    } else {
        hp[1] = E.u * uL[0] + E.u * uL[1] + E.u * uL[2] + uL[3];
        hp[2] = (E.v - E.a) * uL[0] + E.v * uL[1] + (E.v + E.a) * uL[2];
        hp[3] = E.H1 * uL[0] + E.q2 * uL[1] + E.H2 * uL[2] + E.u * uL[3];
    }
}

// Scalar body of the WCNS_Z3 loop (src/nnd_center_RK.F90:330-347) for one
// characteristic component: third-order Z-type interpolation.
template <class D>
__device__ __forceinline__ double wcns_z3_d(double u1, double u2, double u3, D &dv) {
    const double d1 = FDM_D1_WCNS, d2 = FDM_D2_WCNS;
    double t = -u1 + u2;
    double IS1 = t * t;
    t = -u2 + u3;
    const double IS2a = t * t;
    t = u1 - 2. * u2 + u3;
    const double IS3 = t * t;
    const double p1 = u2;
    const double p2 = dv.q((-u1 + 6.0 * u2 + 3.0 * u3) / 8.0 - d1 * p1, dv.d2);
    IS1 = fmin(IS1, IS2a);
    const double IS2 = IS3 + u1 * u1 + u2 * u2 + u3 * u3 - u1 * u2 - u2 * u3 - u1 * u3;
    t = 10. * fabs(IS2 - 3. * IS1);
    const double tau3 = t * t;
    const double a1 = d1 * (1.0 + dv.q(tau3, FDM_EPS_WCNS + IS1));
    const double a2 = d2 * (1.0 + dv.q(tau3, FDM_EPS_WCNS + IS2));
    const Den ds = dv.den(a1 + a2);
    const double w1 = dv.q(a1, ds);
    const double w2 = dv.q(a2, ds);
    return w1 * p1 + w2 * p2;
}
__device__ __forceinline__ double wcns_z3(double u1, double u2, double u3) {
    DivIEEE dv(1.4);   // gm1 is not used here
    return wcns_z3_d(u1, u2, u3, dv);
}

// the record of slot i read again through the non-coherent path, as an
// opaque load (the optimiser may not replace it by an earlier read, so the
// earlier values need not stay in registers)
__device__ __forceinline__ Prim load_prim_again(const double4 *s, int64_t i) {
    const double *p = reinterpret_cast<const double *>(s + i);
    double a, b, c, d;
    asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%4];\n\tld.global.nc.v2.f64 {%2, %3}, [%4+16];"
                 : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
                 : "l"(p));
    return Prim{a, b, c, d};
}
// the conserved state of cons_flux alone (the same operations)
template <int DIR, class D>
__device__ __forceinline__ void cons_state_d(const Prim &q, D &dv, double U[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    U[0] = q.r;
    U[1] = q.r * q.u;
    U[2] = q.r * q.v;
    U[3] = dv.q(q.p, dv.gm1) + 0.5 * q.r * ke;
}
template <int DIR>
__device__ __forceinline__ void cons_state(const Prim &q, double g, double U[4]) {
    DivIEEE dv(g);
    cons_state_d<DIR>(q, dv, U);
}
// the physical flux of cons_flux alone (the same operations)
template <int DIR, class D>
__device__ __forceinline__ void phys_flux_d(const Prim &q, D &dv, double F[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    if (DIR == 0) {
        F[0] = q.r * q.u;
        F[1] = q.r * q.u * q.u + q.p;
        F[2] = q.r * q.u * q.v;
        F[3] = q.u * (dv.q(q.p, dv.gm1) + 0.5 * q.r * ke + q.p);
    } else {
        F[0] = q.r * q.v;
        F[1] = q.r * q.u * q.v;
        F[2] = q.r * q.v * q.v + q.p;
        F[3] = q.v * (dv.q(q.p, dv.gm1) + 0.5 * q.r * ke + q.p);
    }
}
// The face flux in the reference's order: the four conserved states and the
// four fluxes formed first, then the projections and reconstructions;
// every division through the policy dv.
template <int DIR, class D>
__device__ __forceinline__ void face_flux_ref_d(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3,
                                                double g, D &dv, double lam, double out[4]) {
    double U0[4], U1[4], U2[4], U3[4], F0[4], F1[4], F2[4], F3[4];
    cons_flux_d<DIR>(s0, dv, U0, F0);
    cons_flux_d<DIR>(s1, dv, U1, F1);
    cons_flux_d<DIR>(s2, dv, U2, F2);
    cons_flux_d<DIR>(s3, dv, U3, F3);
    double Um[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) Um[r] = (U1[r] + U2[r]) / 2.0;
    Eig E;
    eigen_d<DIR>(Um, g, dv, E);
    double w0[4], w1[4], w2[4], w3[4];
    double uwL[4], uwR[4], ugL[4], ugR[4];
    project<DIR>(E, U0, w0); project<DIR>(E, U1, w1);
    project<DIR>(E, U2, w2); project<DIR>(E, U3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        uwL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
        uwR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
    }
    project<DIR>(E, F0, w0); project<DIR>(E, F1, w1);
    project<DIR>(E, F2, w2); project<DIR>(E, F3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ugL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
        ugR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
    }
    double wL[4], wR[4], gL[4], gR[4];
    back_project<DIR>(E, uwL, wL);
    back_project<DIR>(E, uwR, wR);
    back_project<DIR>(E, ugL, gL);
    back_project<DIR>(E, ugR, gR);
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
}

// Numerical flux at the face between s1 and s2 from the 4-point stencil
// s0..s3 (one half of LXL_X_wcns3 / LXL_Y_wcns3, src/nnd_center_RK.F90:84-106,
// 205-227): characteristic projection at the face mean, four WCNS_Z3
// reconstructions and the global Lax-Friedrichs split.
template <int DIR, bool SPLIT = true>
__device__ __forceinline__ void face_flux(const Prim &s0, const Prim &s1, const Prim &s2,
                                          const Prim &s3, double g, double lam, double out[4]) {
    if constexpr (SPLIT) {
        // The state half (U, its projections and reconstructions, back-projected)
        // is finished before the flux half starts, so the four conserved states
        // and the four fluxes are never held at once (fewer registers); every
        // value is formed by the same operations as in the reference's order.
        double wL[4], wR[4];
        Eig E;
        {
            double U0[4], U1[4], U2[4], U3[4];
            cons_state<DIR>(s1, g, U1);
            cons_state<DIR>(s2, g, U2);
            double Um[4];
    #pragma unroll
            for (int r = 0; r < 4; ++r) Um[r] = (U1[r] + U2[r]) / 2.0;
            eigen<DIR>(Um, g, E);
            cons_state<DIR>(s0, g, U0);
            cons_state<DIR>(s3, g, U3);
            double w0[4], w1[4], w2[4], w3[4], uwL[4], uwR[4];
            project<DIR>(E, U0, w0); project<DIR>(E, U1, w1);
            project<DIR>(E, U2, w2); project<DIR>(E, U3, w3);
    #pragma unroll
            for (int r = 0; r < 4; ++r) {
                uwL[r] = wcns_z3(w0[r], w1[r], w2[r]);
                uwR[r] = wcns_z3(w3[r], w2[r], w1[r]);
            }
            back_project<DIR>(E, uwL, wL);
            back_project<DIR>(E, uwR, wR);
        }
        double F0[4], F1[4], F2[4], F3[4];
        phys_flux<DIR>(s0, g, F0); phys_flux<DIR>(s1, g, F1);
        phys_flux<DIR>(s2, g, F2); phys_flux<DIR>(s3, g, F3);
        double w0[4], w1[4], w2[4], w3[4], ugL[4], ugR[4];
        project<DIR>(E, F0, w0); project<DIR>(E, F1, w1);
        project<DIR>(E, F2, w2); project<DIR>(E, F3, w3);
    #pragma unroll
        for (int r = 0; r < 4; ++r) {
            ugL[r] = wcns_z3(w0[r], w1[r], w2[r]);
            ugR[r] = wcns_z3(w3[r], w2[r], w1[r]);
        }
        double gL[4], gR[4];
        back_project<DIR>(E, ugL, gL);
        back_project<DIR>(E, ugR, gR);
    #pragma unroll
        for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
    } else {
        // the same values with the four states and fluxes formed first (for
        // the batched kernel, whose register budget this order suits better)
        DivIEEE dv(g);
        face_flux_ref_d<DIR>(s0, s1, s2, s3, g, dv, lam, out);
    }
}

// face_flux in the split order, reading the stencil records (slots a..d of
// cur) once for the state half and again for the flux half; every division
// through the policy dv
template <int DIR, class D>
__device__ __forceinline__ void face_flux_slots_d(const double4 *__restrict__ cur, int32_t ia, int32_t ib,
                                                  int32_t ic, int32_t id, double g, D &dv, double lam,
                                                  double out[4]) {
    double wL[4], wR[4];
    Eig E;
    {
        const Prim s0 = load_prim(cur, ia), s1 = load_prim(cur, ib), s2 = load_prim(cur, ic), s3 = load_prim(cur, id);
        double U0[4], U1[4], U2[4], U3[4];
        cons_state_d<DIR>(s1, dv, U1);
        cons_state_d<DIR>(s2, dv, U2);
        double Um[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) Um[r] = (U1[r] + U2[r]) / 2.0;
        eigen_d<DIR>(Um, g, dv, E);
        cons_state_d<DIR>(s0, dv, U0);
        cons_state_d<DIR>(s3, dv, U3);
        double w0[4], w1[4], w2[4], w3[4], uwL[4], uwR[4];
        project<DIR>(E, U0, w0); project<DIR>(E, U1, w1);
        project<DIR>(E, U2, w2); project<DIR>(E, U3, w3);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            uwL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
            uwR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
        }
        back_project<DIR>(E, uwL, wL);
        back_project<DIR>(E, uwR, wR);
    }
    double F0[4], F1[4], F2[4], F3[4];
    phys_flux_d<DIR>(load_prim_again(cur, ia), dv, F0);
    phys_flux_d<DIR>(load_prim_again(cur, ib), dv, F1);
    phys_flux_d<DIR>(load_prim_again(cur, ic), dv, F2);
    phys_flux_d<DIR>(load_prim_again(cur, id), dv, F3);
    double w0[4], w1[4], w2[4], w3[4], ugL[4], ugR[4];
    project<DIR>(E, F0, w0); project<DIR>(E, F1, w1);
    project<DIR>(E, F2, w2); project<DIR>(E, F3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ugL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
        ugR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
    }
    double gL[4], gR[4];
    back_project<DIR>(E, ugL, gL);
    back_project<DIR>(E, ugR, gR);
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
}
template <int DIR>
__device__ __forceinline__ void face_flux_slots(const double4 *__restrict__ cur, int32_t ia, int32_t ib,
                                                int32_t ic, int32_t id, double g, double lam, double out[4]) {
    DivIEEE dv(g);
    face_flux_slots_d<DIR>(cur, ia, ib, ic, id, g, dv, lam, out);
}

// ------------------------------------------------ face flux, 4 lanes/face
// Lane r of a group of four computes characteristic component r: its row of
// Ri, the four WCNS_Z3 reconstructions of that component, and, after the
// reconstructed components are exchanged within the group, row r of R*uL
// and flux component r.  Every value is formed by the same operations in
// the same order as in face_flux, so both give identical bits.
struct EigRow {
    double u, v, a, q2, H1, H2;
    double ri[4];   // row r of Ri
};

template <int DIR>
__device__ __forceinline__ void eigen_row(const double Um[4], double g, int r, EigRow &E) {
    const double r0 = Um[0];
    const double u = Um[1] / Um[0];
    const double v = Um[2] / Um[0];
    const double p = (g - 1.0) * r0 * (Um[3] / r0 - 0.5 * (u * u + v * v));
    const double a = sqrt(g * p / r0);
    const double q2 = 0.5 * (u * u + v * v);
    const double aa = a * a, a2 = 2.0 * a * a;
    E.u = u; E.v = v; E.a = a; E.q2 = q2;
    const double c = DIR == 0 ? u : v;
    E.H1 = a * a / (g - 1) + q2 - c * a;
    E.H2 = a * a / (g - 1) + q2 + c * a;
    if (r == 0) {
        E.ri[0] = ((g - 1.0) * q2 + a * c) / a2;
        E.ri[1] = DIR == 0 ? ((1.0 - g) * u - a) / a2 : ((1.0 - g) * u) / a2;
        E.ri[2] = DIR == 0 ? ((1.0 - g) * v) / a2 : ((1.0 - g) * v - a) / a2;
        E.ri[3] = (g - 1.0) / a2;
    } else if (r == 1) {
        E.ri[0] = (aa - (g - 1.0) * q2) / aa;
        E.ri[1] = ((g - 1.0) * u) / aa;
        E.ri[2] = ((g - 1.0) * v) / aa;
        E.ri[3] = (1.0 - g) / aa;
    } else if (r == 2) {
        E.ri[0] = ((g - 1.0) * q2 - a * c) / a2;
        E.ri[1] = DIR == 0 ? ((1.0 - g) * u + a) / a2 : ((1.0 - g) * u) / a2;
        E.ri[2] = DIR == 0 ? ((1.0 - g) * v) / a2 : ((1.0 - g) * v + a) / a2;
        E.ri[3] = (g - 1.0) / a2;
    } else {
        E.ri[0] = DIR == 0 ? v : -u;
        E.ri[1] = 0.0;
        E.ri[2] = 0.0;
        E.ri[3] = 0.0;
    }
}

// component r of Ri * X
template <int DIR>
__device__ __forceinline__ double project_row(const EigRow &E, int r, const double X[4]) {
    if (r < 3) return E.ri[0] * X[0] + E.ri[1] * X[1] + E.ri[2] * X[2] + E.ri[3] * X[3];
    return DIR == 0 ? E.ri[0] * X[0] + -X[2] : E.ri[0] * X[0] + X[1];
}

// row r of R * uL
template <int DIR>
__device__ __forceinline__ double back_row(const EigRow &E, int r, const double uL[4]) {
    if (r == 0) return uL[0] + uL[1] + uL[2];
    if (DIR == 0) {
        if (r == 1) return (E.u - E.a) * uL[0] + E.u * uL[1] + (E.u + E.a) * uL[2];
        if (r == 2) return E.v * uL[0] + E.v * uL[1] + E.v * uL[2] + -uL[3];
        return E.H1 * uL[0] + E.q2 * uL[1] + E.H2 * uL[2] + -E.v * uL[3];
    }
    if (r == 1) return E.u * uL[0] + E.u * uL[1] + E.u * uL[2] + uL[3];
    if (r == 2) return (E.v - E.a) * uL[0] + E.v * uL[1] + (E.v + E.a) * uL[2];
    return E.H1 * uL[0] + E.q2 * uL[1] + E.H2 * uL[2] + E.u * uL[3];
}

// ------------------------------------------------------------ WLS-WENO
// integrate_square_poly (src/XuanGua.F90:342-355)
__device__ __forceinline__ double isq_poly(double k0, double k1, double k2, const double *box) {
    const double x_min = box[0], x_max = box[1], y_min = box[2], y_max = box[3];
    const double term1 = k0 * k0 * (x_max - x_min) * (y_max - y_min);
    const double term2 = 2 * k0 * k1 * (x_max * x_max - x_min * x_min) / 2 * (y_max - y_min) +
                         2 * k0 * k2 * (x_max - x_min) * (y_max * y_max - y_min * y_min) / 2;
    const double term3 = k1 * k1 * (x_max * x_max * x_max - x_min * x_min * x_min) / 3 * (y_max - y_min) +
                         2 * k1 * k2 * (x_max * x_max - x_min * x_min) / 2 * (y_max * y_max - y_min * y_min) / 2 +
                         k2 * k2 * (x_max - x_min) * (y_max * y_max * y_max - y_min * y_min * y_min) / 3;
    return term1 + term2 + term3;
}
// compute_smoothness (src/XuanGua.F90:309-340)
__device__ __forceinline__ double smooth2(const double a[6], const double *box) {
    const double a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5];
    const double dxb = box[1] - box[0], dyb = box[3] - box[2];
    double beta = 0.0;
    beta = beta + isq_poly(a1, 2 * a3, a4, box);
    beta = beta + isq_poly(a2, a4, 2 * a5, box);
    beta = beta + (2 * a3) * (2 * a3) * dxb * dyb;
    beta = beta + a4 * a4 * dxb * dyb;
    beta = beta + (2 * a5) * (2 * a5) * dxb * dyb;
    return beta;
}
__device__ __forceinline__ double smooth1(const double b[3], const double *box) {
    return (b[1] * b[1] + b[2] * b[2]) * (box[1] - box[0]) * (box[3] - box[2]);
}

// Per-stage part of WLSI_US_WENO (src/XuanGua.F90:257-307) for one variable:
// the geometry (x, y, w, the three brinv inverses) was prepared at regrid.
__device__ __forceinline__ double wls_eval_var(const double *__restrict__ geo, int m1, int m2,
                                               const double *phi) {
    const int m = m1 + m2;
    const double *x = geo + G_X, *y = geo + G_Y, *w = geo + G_W;
    const double xx = geo[G_XX], yy = geo[G_YY];
    const double *box = geo + G_BOX;
    // the loops run over the fixed WLS_MAXM slots with the members' count as a
    // predicate, so the arrays stay in registers (the sums keep their order)
    double wphi[WLS_MAXM];
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) wphi[i] = i < m ? w[i] * phi[i] : 0.0;
    double pt[6];
    {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, s5 = 0.0;
#pragma unroll
        for (int i = 0; i < WLS_MAXM; ++i) {
            if (i >= m) continue;
            const double xi = x[i], yi = y[i], wp = wphi[i];
            s0 = s0 + 1.0 * wp;
            s1 = s1 + xi * wp;
            s2 = s2 + yi * wp;
            s3 = s3 + (xi * yi) * wp;
            s4 = s4 + (xi * xi) * wp;
            s5 = s5 + (yi * yi) * wp;
        }
        pt[0] = s0; pt[1] = s1; pt[2] = s2; pt[3] = s3; pt[4] = s4; pt[5] = s5;
    }
    double arr[6];
    const double *L = geo + G_L;
#pragma unroll
    for (int a = 0; a < 6; ++a) {
        double s = 0.0;
#pragma unroll
        for (int b = 0; b < 6; ++b) s = s + L[a * 6 + b] * pt[b];
        arr[a] = s;
    }
    const double var_large = arr[0] + xx * arr[1] + yy * arr[2] + xx * yy * arr[3] +
                             xx * xx * arr[4] + yy * yy * arr[5];
    const double sm_large = smooth2(arr, box);
    double p1[3] = {0.0, 0.0, 0.0}, p2[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) {
        if (i >= m1) continue;
        p1[0] = p1[0] + 1.0 * wphi[i];
        p1[1] = p1[1] + x[i] * wphi[i];
        p1[2] = p1[2] + y[i] * wphi[i];
    }
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) {
        if (i < m1 || i >= m) continue;
        p2[0] = p2[0] + 1.0 * wphi[i];
        p2[1] = p2[1] + x[i] * wphi[i];
        p2[2] = p2[2] + y[i] * wphi[i];
    }
    double c1[3], c2[3];
    const double *A = geo + G_A, *B = geo + G_B;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double s = 0.0, t = 0.0;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            s = s + A[a * 3 + b] * p1[b];
            t = t + B[a * 3 + b] * p2[b];
        }
        c1[a] = s;
        c2[a] = t;
    }
    const double vs1 = c1[0] + xx * c1[1] + yy * c1[2];
    const double vs2 = c2[0] + xx * c2[1] + yy * c2[2];
    const double sm1 = smooth1(c1, box), sm2 = smooth1(c2, box);
    const double eps = 1.e-6;
    double sa = 0.0;
    sa = sa + fabs(sm_large - sm1);
    sa = sa + fabs(sm_large - sm2);
    double tau = sa / 2.0;
    tau = tau * tau;
    const double al0 = 0.98 * (1.0 + tau / (eps + sm_large));
    const double al1 = 0.01 * (1.0 + tau / (eps + sm1));
    const double al2 = 0.01 * (1.0 + tau / (eps + sm2));
    double sal = 0.0;
    sal = sal + al0;
    sal = sal + al1;
    sal = sal + al2;
    const double om0 = al0 / sal, om1 = al1 / sal, om2 = al2 / sal;
    return om0 * (1.0 / 0.98 * var_large - (0.01 / 0.98 * vs1 + 0.01 / 0.98 * vs2)) +
           (om1 * vs1 + om2 * vs2);
}

}  // namespace fdm
