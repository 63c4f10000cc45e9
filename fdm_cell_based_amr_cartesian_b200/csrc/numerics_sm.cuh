// numerics_sm.cuh — the face flux with the characteristic basis of the face
// held in shared memory instead of registers.
//
// A face's flux keeps the basis (12 entries of Ri plus u, v, a, q2, H1, H2:
// 18 doubles) live through all eight projections and four back-projections,
// which is a quarter of the registers that cap the face kernel's occupancy.
// Here each thread writes its face's basis into its own column of a
// structure-of-arrays block in shared memory (consecutive threads,
// consecutive doubles: no bank conflicts) and reads each entry where it is
// used.  The operations and their order are those of eigen_d, project and
// back_project (numerics.cuh), so the bits are the same.
#pragma once
#include "numerics.cuh"

namespace fdm {

template <int TB>
struct EigShared {
    double u[TB], v[TB], a[TB], q2[TB], H1[TB], H2[TB];
    double Ri[3][4][TB];   // rows 0..2; row 3 is (v | -u, 0 | 1, -1 | 0, 0)
};

template <int DIR, int TB, class D>
__device__ __forceinline__ void eigen_sm(const double Um[4], double g, D &dv, EigShared<TB> &S, int t) {
    const double r0 = Um[0];
    const Den dr = dv.den(Um[0]);
    const double u = dv.q(Um[1], dr);
    const double v = dv.q(Um[2], dr);
    const double p = (g - 1.0) * r0 * (dv.q(Um[3], dr) - 0.5 * (u * u + v * v));
    const double a = sqrt(dv.q(g * p, dr));
    const double q2 = 0.5 * (u * u + v * v);
    const double aa = a * a, a2 = 2.0 * a * a;
    const Den daa = dv.den(aa), da2 = dv.den(a2);
    S.u[t] = u; S.v[t] = v; S.a[t] = a; S.q2[t] = q2;
    const double c = DIR == 0 ? u : v;
    S.H1[t] = dv.q(a * a, dv.gm1) + q2 - c * a;
    S.H2[t] = dv.q(a * a, dv.gm1) + q2 + c * a;
    if (DIR == 0) {
        S.Ri[0][0][t] = dv.q((g - 1.0) * q2 + a * u, da2);
        S.Ri[1][0][t] = dv.q(aa - (g - 1.0) * q2, daa);
        S.Ri[2][0][t] = dv.q((g - 1.0) * q2 - a * u, da2);
        S.Ri[0][1][t] = dv.q((1.0 - g) * u - a, da2);
        S.Ri[1][1][t] = dv.q((g - 1.0) * u, daa);
        S.Ri[2][1][t] = dv.q((1.0 - g) * u + a, da2);
        S.Ri[0][2][t] = dv.q((1.0 - g) * v, da2);
        S.Ri[1][2][t] = dv.q((g - 1.0) * v, daa);
        S.Ri[2][2][t] = dv.q((1.0 - g) * v, da2);
    } else {
        S.Ri[0][0][t] = dv.q((g - 1.0) * q2 + a * v, da2);
        S.Ri[1][0][t] = dv.q(aa - (g - 1.0) * q2, daa);
        S.Ri[2][0][t] = dv.q((g - 1.0) * q2 - a * v, da2);
        S.Ri[0][1][t] = dv.q((1.0 - g) * u, da2);
        S.Ri[1][1][t] = dv.q((g - 1.0) * u, daa);
        S.Ri[2][1][t] = dv.q((1.0 - g) * u, da2);
        S.Ri[0][2][t] = dv.q((1.0 - g) * v - a, da2);
        S.Ri[1][2][t] = dv.q((g - 1.0) * v, daa);
        S.Ri[2][2][t] = dv.q((1.0 - g) * v + a, da2);
    }
    S.Ri[0][3][t] = dv.q(g - 1.0, da2);
    S.Ri[1][3][t] = dv.q(1.0 - g, daa);
    S.Ri[2][3][t] = dv.q(g - 1.0, da2);
}

// w = Ri * X, as project()
template <int DIR, int TB>
__device__ __forceinline__ void project_sm(const EigShared<TB> &S, int t, const double X[4], double w[4]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
        w[r] = S.Ri[r][0][t] * X[0] + S.Ri[r][1][t] * X[1] + S.Ri[r][2][t] * X[2] + S.Ri[r][3][t] * X[3];
    if (DIR == 0) w[3] = S.v[t] * X[0] + -X[2];
    else w[3] = -S.u[t] * X[0] + X[1];
}

// hp = R * uL, as back_project()
template <int DIR, int TB>
__device__ __forceinline__ void back_project_sm(const EigShared<TB> &S, int t, const double uL[4], double hp[4]) {
    const double u = S.u[t], v = S.v[t], a = S.a[t];
    hp[0] = uL[0] + uL[1] + uL[2];
    if (DIR == 0) {
        hp[1] = (u - a) * uL[0] + u * uL[1] + (u + a) * uL[2];
        hp[2] = v * uL[0] + v * uL[1] + v * uL[2] + -uL[3];
        hp[3] = S.H1[t] * uL[0] + S.q2[t] * uL[1] + S.H2[t] * uL[2] + -v * uL[3];
    } else {
        hp[1] = u * uL[0] + u * uL[1] + u * uL[2] + uL[3];
        hp[2] = (v - a) * uL[0] + v * uL[1] + (v + a) * uL[2];
        hp[3] = S.H1[t] * uL[0] + S.q2[t] * uL[1] + S.H2[t] * uL[2] + u * uL[3];
    }
}

// face_flux_slots_d with the basis in shared memory (thread t's column)
template <int DIR, int TB, class D>
__device__ __forceinline__ void face_flux_slots_sm(const double4 *__restrict__ cur, int32_t ia, int32_t ib, int32_t ic,
                                                   int32_t id, double g, D &dv, double lam, EigShared<TB> &S,
                                                   int t, double out[4]) {
    double wL[4], wR[4];
    {
        const Prim s0 = load_prim(cur, ia), s1 = load_prim(cur, ib), s2 = load_prim(cur, ic), s3 = load_prim(cur, id);
        double U0[4], U1[4], U2[4], U3[4];
        cons_state_d<DIR>(s1, dv, U1);
        cons_state_d<DIR>(s2, dv, U2);
        double Um[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) Um[r] = (U1[r] + U2[r]) / 2.0;
        eigen_sm<DIR, TB>(Um, g, dv, S, t);
        cons_state_d<DIR>(s0, dv, U0);
        cons_state_d<DIR>(s3, dv, U3);
        double w0[4], w1[4], w2[4], w3[4], uwL[4], uwR[4];
        project_sm<DIR, TB>(S, t, U0, w0); project_sm<DIR, TB>(S, t, U1, w1);
        project_sm<DIR, TB>(S, t, U2, w2); project_sm<DIR, TB>(S, t, U3, w3);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            uwL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
            uwR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
        }
        back_project_sm<DIR, TB>(S, t, uwL, wL);
        back_project_sm<DIR, TB>(S, t, uwR, wR);
    }
    double F0[4], F1[4], F2[4], F3[4];
    phys_flux_d<DIR>(load_prim_again(cur, ia), dv, F0);
    phys_flux_d<DIR>(load_prim_again(cur, ib), dv, F1);
    phys_flux_d<DIR>(load_prim_again(cur, ic), dv, F2);
    phys_flux_d<DIR>(load_prim_again(cur, id), dv, F3);
    double w0[4], w1[4], w2[4], w3[4], ugL[4], ugR[4];
    project_sm<DIR, TB>(S, t, F0, w0); project_sm<DIR, TB>(S, t, F1, w1);
    project_sm<DIR, TB>(S, t, F2, w2); project_sm<DIR, TB>(S, t, F3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ugL[r] = wcns_z3_d(w0[r], w1[r], w2[r], dv);
        ugR[r] = wcns_z3_d(w3[r], w2[r], w1[r], dv);
    }
    double gL[4], gR[4];
    back_project_sm<DIR, TB>(S, t, ugL, gL);
    back_project_sm<DIR, TB>(S, t, ugR, gR);
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
}

}  // namespace fdm
