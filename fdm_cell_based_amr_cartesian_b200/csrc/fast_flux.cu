// fast_flux.cu — the WCNS face flux of flux_variant 1 ("fast").
//
// The same scheme as numerics.cuh's face_flux (conserved variables and
// fluxes, characteristic projection at the face mean, four WCNS_Z3
// reconstructions per component, global Lax-Friedrichs split), rearranged
// for the FP64 pipe: this file is compiled with FMA contraction, divisions
// by the same value share one reciprocal, and the Z weights
//   w1 = d1 (1 + tau/(eps+IS1)) / [d1 (1 + tau/(eps+IS1)) + d2 (1 + tau/(eps+IS2))]
// are formed with one division, after multiplying through by
// (eps+IS1)(eps+IS2).  About 20 correctly rounded divisions per face remain
// of the exact path's 106.  Results differ from the exact path by rounding
// only; the per-step bar (1e-12 relative) is tested against the oracle.
#include <algorithm>

#include "items.cuh"

namespace fdm {
namespace fast {

template <int DIR>
__device__ __forceinline__ void cons_flux_f(const Prim &q, double ig1, double U[4], double F[4]) {
    const double ke = q.u * q.u + q.v * q.v;
    const double E = q.p * ig1 + 0.5 * q.r * ke;
    const double un = DIR == 0 ? q.u : q.v;
    U[0] = q.r;
    U[1] = q.r * q.u;
    U[2] = q.r * q.v;
    U[3] = E;
    F[0] = q.r * un;
    F[1] = U[1] * un + (DIR == 0 ? q.p : 0.0);
    F[2] = U[2] * un + (DIR == 0 ? 0.0 : q.p);
    F[3] = un * (E + q.p);
}

template <int DIR>
__device__ __forceinline__ void eigen_f(const double Um[4], double g, double ig1, Eig &E) {
    const double r0 = Um[0];
    const double ir = 1.0 / r0;
    const double u = Um[1] * ir;
    const double v = Um[2] * ir;
    const double q2 = 0.5 * (u * u + v * v);
    const double p = (g - 1.0) * (Um[3] - r0 * q2);
    const double a = sqrt(g * p * ir);
    const double aa = a * a;
    const double iaa = 1.0 / aa, ia2 = 0.5 * iaa;
    const double gm = g - 1.0;
    E.u = u; E.v = v; E.a = a; E.q2 = q2;
    const double c = DIR == 0 ? u : v;
    E.H1 = aa * ig1 + q2 - c * a;
    E.H2 = aa * ig1 + q2 + c * a;
    if (DIR == 0) {
        E.Ri[0][0] = (gm * q2 + a * u) * ia2;
        E.Ri[1][0] = (aa - gm * q2) * iaa;
        E.Ri[2][0] = (gm * q2 - a * u) * ia2;
        E.Ri[3][0] = v;
        E.Ri[0][1] = (-gm * u - a) * ia2;
        E.Ri[1][1] = (gm * u) * iaa;
        E.Ri[2][1] = (-gm * u + a) * ia2;
        E.Ri[3][1] = 0.0;
        E.Ri[0][2] = (-gm * v) * ia2;
        E.Ri[1][2] = (gm * v) * iaa;
        E.Ri[2][2] = (-gm * v) * ia2;
        E.Ri[3][2] = -1.0;
    } else {
        E.Ri[0][0] = (gm * q2 + a * v) * ia2;
        E.Ri[1][0] = (aa - gm * q2) * iaa;
        E.Ri[2][0] = (gm * q2 - a * v) * ia2;
        E.Ri[3][0] = -u;
        E.Ri[0][1] = (-gm * u) * ia2;
        E.Ri[1][1] = (gm * u) * iaa;
        E.Ri[2][1] = (-gm * u) * ia2;
        E.Ri[3][1] = 1.0;
        E.Ri[0][2] = (-gm * v - a) * ia2;
        E.Ri[1][2] = (gm * v) * iaa;
        E.Ri[2][2] = (-gm * v + a) * ia2;
        E.Ri[3][2] = 0.0;
    }
    E.Ri[0][3] = gm * ia2;
    E.Ri[1][3] = -gm * iaa;
    E.Ri[2][3] = gm * ia2;
    E.Ri[3][3] = 0.0;
}

// WCNS_Z3 with one division: a1, a2 scaled by (eps+IS1)(eps+IS2)
__device__ __forceinline__ double wcns_z3_f(double u1, double u2, double u3) {
    const double d1 = FDM_D1_WCNS, d2 = FDM_D2_WCNS, id2 = 1.0 / FDM_D2_WCNS;
    double t = u2 - u1;
    const double IS1a = t * t;
    t = u3 - u2;
    const double IS2a = t * t;
    t = u1 - 2.0 * u2 + u3;
    const double IS3 = t * t;
    const double p1 = u2;
    const double p2 = ((-u1 + 6.0 * u2 + 3.0 * u3) * 0.125 - d1 * p1) * id2;
    const double IS1 = fmin(IS1a, IS2a);
    const double IS2 = IS3 + u1 * u1 + u2 * u2 + u3 * u3 - u1 * u2 - u2 * u3 - u1 * u3;
    t = 10.0 * fabs(IS2 - 3.0 * IS1);
    const double tau3 = t * t;
    const double e1 = FDM_EPS_WCNS + IS1, e2 = FDM_EPS_WCNS + IS2;
    const double a1 = d1 * (e1 + tau3) * e2;
    const double a2 = d2 * (e2 + tau3) * e1;
    return (a1 * p1 + a2 * p2) / (a1 + a2);
}

template <int DIR>
__device__ __forceinline__ void face_flux_f(const Prim &s0, const Prim &s1, const Prim &s2, const Prim &s3, double g,
                                          double ig1, double lam, double out[4]) {
    double U0[4], U1[4], U2[4], U3[4], F0[4], F1[4], F2[4], F3[4];
    cons_flux_f<DIR>(s0, ig1, U0, F0);
    cons_flux_f<DIR>(s1, ig1, U1, F1);
    cons_flux_f<DIR>(s2, ig1, U2, F2);
    cons_flux_f<DIR>(s3, ig1, U3, F3);
    double Um[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) Um[r] = 0.5 * (U1[r] + U2[r]);
    Eig E;
    eigen_f<DIR>(Um, g, ig1, E);
    double w0[4], w1[4], w2[4], w3[4];
    double uwL[4], uwR[4], ugL[4], ugR[4];
    project<DIR>(E, U0, w0); project<DIR>(E, U1, w1);
    project<DIR>(E, U2, w2); project<DIR>(E, U3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        uwL[r] = wcns_z3_f(w0[r], w1[r], w2[r]);
        uwR[r] = wcns_z3_f(w3[r], w2[r], w1[r]);
    }
    project<DIR>(E, F0, w0); project<DIR>(E, F1, w1);
    project<DIR>(E, F2, w2); project<DIR>(E, F3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ugL[r] = wcns_z3_f(w0[r], w1[r], w2[r]);
        ugR[r] = wcns_z3_f(w3[r], w2[r], w1[r]);
    }
    double wL[4], wR[4], gL[4], gR[4];
    back_project<DIR>(E, uwL, wL);
    back_project<DIR>(E, uwR, wR);
    back_project<DIR>(E, ugL, gL);
    back_project<DIR>(E, ugR, gR);
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
}

// the same flux with the state half finished before the flux half, and the
// stencil records read again for the flux half (fewer live registers)
template <int DIR>
__device__ __forceinline__ void face_flux_f_slots(const double4 *__restrict__ cur, int32_t ia, int32_t ib,
                                                  int32_t ic, int32_t id, double g, double ig1, double lam,
                                                  double out[4]) {
    double wL[4], wR[4];
    Eig E;
    {
        double U0[4], U1[4], U2[4], U3[4], Fd[4];
        cons_flux_f<DIR>(load_prim(cur, ib), ig1, U1, Fd);
        cons_flux_f<DIR>(load_prim(cur, ic), ig1, U2, Fd);
        double Um[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) Um[r] = 0.5 * (U1[r] + U2[r]);
        eigen_f<DIR>(Um, g, ig1, E);
        cons_flux_f<DIR>(load_prim(cur, ia), ig1, U0, Fd);
        cons_flux_f<DIR>(load_prim(cur, id), ig1, U3, Fd);
        double w0[4], w1[4], w2[4], w3[4], uwL[4], uwR[4];
        project<DIR>(E, U0, w0); project<DIR>(E, U1, w1);
        project<DIR>(E, U2, w2); project<DIR>(E, U3, w3);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            uwL[r] = wcns_z3_f(w0[r], w1[r], w2[r]);
            uwR[r] = wcns_z3_f(w3[r], w2[r], w1[r]);
        }
        back_project<DIR>(E, uwL, wL);
        back_project<DIR>(E, uwR, wR);
    }
    double F0[4], F1[4], F2[4], F3[4], Ud[4];
    cons_flux_f<DIR>(load_prim_again(cur, ia), ig1, Ud, F0);
    cons_flux_f<DIR>(load_prim_again(cur, ib), ig1, Ud, F1);
    cons_flux_f<DIR>(load_prim_again(cur, ic), ig1, Ud, F2);
    cons_flux_f<DIR>(load_prim_again(cur, id), ig1, Ud, F3);
    double w0[4], w1[4], w2[4], w3[4], ugL[4], ugR[4];
    project<DIR>(E, F0, w0); project<DIR>(E, F1, w1);
    project<DIR>(E, F2, w2); project<DIR>(E, F3, w3);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        ugL[r] = wcns_z3_f(w0[r], w1[r], w2[r]);
        ugR[r] = wcns_z3_f(w3[r], w2[r], w1[r]);
    }
    double gL[4], gR[4];
    back_project<DIR>(E, ugL, gL);
    back_project<DIR>(E, ugR, gR);
#pragma unroll
    for (int r = 0; r < 4; ++r) out[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
}

template <int DIR>
__device__ __forceinline__ void face_item(const Tables &T, const double4 *__restrict__ cur, double4 *F, double lam,
                                          double g, double ig1, int64_t f) {
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    double out[4];
    face_flux_f_slots<DIR>(cur, a, b, c, d, g, ig1, lam, out);
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

}  // namespace fast

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

template <int DIR, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) k_faces_fast(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                         const DevScalars *__restrict__ sc, double g) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (f >= T.NI + (DIR == 0 ? T.nux : T.nuy)) return;
    fast::face_item<DIR>(T, cur, F, DIR == 0 ? sc->lambda_x : sc->lambda_y, g, 1.0 / (g - 1.0), f);
}

// hard-face list of the learned gate
template <int DIR>
__global__ void __launch_bounds__(256, 2) k_faces_list_fast(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                            const int32_t *__restrict__ hard,
                                                            const uint32_t *__restrict__ count,
                                                            const DevScalars *__restrict__ sc, double g) {
    const int64_t n = *count;
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y, ig1 = 1.0 / (g - 1.0);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        fast::face_item<DIR>(T, cur, F, lam, g, ig1, hard[i]);
}

template <int TB, int MINB>
static void faces_fast(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    k_faces_fast<0, TB, MINB><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, h->G.gama);
    k_faces_fast<1, TB, MINB><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, h->G.gama);
}

// the launch shapes of the autotuner, one thread per face
void launch_faces_fast(fdm_handle *h, const double4 *cur) {
    switch (h->face_variant) {
        case 1: faces_fast<128, 4>(h, cur); break;
        case 2: faces_fast<64, 7>(h, cur); break;
        case 3: faces_fast<256, 2>(h, cur); break;
        case 5: faces_fast<128, 5>(h, cur); break;
        case 6: faces_fast<64, 10>(h, cur); break;
        default: faces_fast<128, 3>(h, cur); break;
    }
}

void launch_faces_list_fast(fdm_handle *h, const double4 *cur, const int32_t *hx, const int32_t *hy,
                            const uint32_t *cnt, int lx, int ly) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    if (lx > 0) k_faces_list_fast<0><<<lx, 256, 0, h->s>>>(T, cur, h->Fx.as<double4>(), hx, cnt, sc, h->G.gama);
    if (ly > 0) k_faces_list_fast<1><<<ly, 256, 0, h->s>>>(T, cur, h->Fy.as<double4>(), hy, cnt + 1, sc, h->G.gama);
}

}  // namespace fdm
