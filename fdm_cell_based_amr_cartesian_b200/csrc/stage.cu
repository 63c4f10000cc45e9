// stage.cu — one SSP-RK3 stage on the device.
//
//   k_requests  hanging-node values (WLS-WENO / interpA / copy) into the
//               virtual slots                 (src/XuanGua.F90:45-398)
//   k_faces     WCNS flux of every distinct face, x and y
//                                             (src/nnd_center_RK.F90:66-353)
//   k_cells     residual, forward-Euler candidate, RK3 blend, residual
//               norms and the next lambda     (src/nnd_center_RK.F90:15-64,
//                                              src/solution.F90:279-286,386-404)
//   k_ghost     boundary images               (src/solution.F90:288-293,109-168)
//
// State lives in three slot arrays of 32-byte (rho,u,v,p) records: interior
// leaves (key order), ghost leaves, corner leaves, then the virtual slots.
#include "handle.cuh"
#include "numerics.cuh"

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

// interpA over a subtree whose leaves are [lo, hi) of the sorted array
// (src/XuanGua.F90:359-398): children combined as
// 0.25*(son1 + son2 + son3 + son4) = 0.25*(((q0 + q1) + q3) + q2).
// One warp: the lanes stage the subtree's leaves in shared memory, lane 0
// folds them in key order with a stack of pending sibling groups.
constexpr int RW_CAP = 256;     // leaves staged per pass
constexpr int RW_STACK = 48;    // >= 3 pending siblings x 15 levels + 1
struct RestrictSmem {
    double4 v[RW_CAP];
    int8_t l[RW_CAP];
    double4 st[RW_STACK];
    int8_t sl[RW_STACK];
};

__device__ double4 restrict_warp(const Tables &T, const double4 *__restrict__ buf, int64_t lo, int64_t hi,
                                 RestrictSmem &sm) {
    const int lane = threadIdx.x & 31;
    int top = 0;
    for (int64_t base = lo; base < hi; base += RW_CAP) {
        const int n = (int)min((int64_t)RW_CAP, hi - base);
        for (int k = lane; k < n; k += 32) {
            sm.v[k] = buf[__ldg(T.lslot + base + k)];
            sm.l[k] = (int8_t)(__ldg(T.lkey + base + k) & 15u);
        }
        __syncwarp();
        if (lane == 0) {
            for (int k = 0; k < n; ++k) {
                if (top >= RW_STACK) break;  // cannot happen for a valid subtree
                sm.st[top] = sm.v[k];
                sm.sl[top] = sm.l[k];
                ++top;
                while (top >= 4 && sm.sl[top - 1] == sm.sl[top - 2] && sm.sl[top - 1] == sm.sl[top - 3] &&
                       sm.sl[top - 1] == sm.sl[top - 4]) {
                    const double4 e0 = sm.st[top - 4], e1 = sm.st[top - 3], e2 = sm.st[top - 2], e3 = sm.st[top - 1];
                    double4 v;
                    v.x = 0.25 * (e0.x + e1.x + e3.x + e2.x);
                    v.y = 0.25 * (e0.y + e1.y + e3.y + e2.y);
                    v.z = 0.25 * (e0.z + e1.z + e3.z + e2.z);
                    v.w = 0.25 * (e0.w + e1.w + e3.w + e2.w);
                    const int8_t l = (int8_t)(sm.sl[top - 1] - 1);
                    top -= 4;
                    sm.st[top] = v;
                    sm.sl[top] = l;
                    ++top;
                }
            }
        }
        __syncwarp();
    }
    double4 r = sm.st[0];
    __syncwarp();
    return r;
}

__global__ void __launch_bounds__(64) k_requests(Tables T, double4 *cur) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= T.NR) return;
    const int64_t out = T.NI + T.NG + T.NC + r;
    const int kind = T.rq_kind[r];
    const int32_t *mem = T.rq_mem + r * WLS_MAXM;
    if (kind == RQ_COPY) {
        cur[out] = cur[mem[0]];
        return;
    }
    if (kind == RQ_RESTRICT) return;   // k_requests_restrict
    const int m1 = T.rq_m[2 * r], m2 = T.rq_m[2 * r + 1];
    const int m = m1 + m2;
    const double *geo = T.rq_geo + r * RQ_GEO;
    double ph[4][WLS_MAXM];
    for (int i = 0; i < m; ++i) {
        const double4 q = cur[mem[i]];
        ph[0][i] = q.x; ph[1][i] = q.y; ph[2][i] = q.z; ph[3][i] = q.w;
    }
    double4 v;
    v.x = wls_eval_var(geo, m1, m2, ph[0]);
    v.y = wls_eval_var(geo, m1, m2, ph[1]);
    v.z = wls_eval_var(geo, m1, m2, ph[2]);
    v.w = wls_eval_var(geo, m1, m2, ph[3]);
    cur[out] = v;
}

// interpA fallbacks of parent_value_weno: one warp per request
__global__ void __launch_bounds__(128) k_requests_restrict(Tables T, double4 *cur) {
    __shared__ RestrictSmem sm[4];
    const int64_t r = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (r >= T.NR) return;
    if (T.rq_kind[r] != RQ_RESTRICT) return;
    const double4 v = restrict_warp(T, cur, T.rq_m[2 * r], T.rq_m[2 * r + 1], sm[threadIdx.x >> 5]);
    if ((threadIdx.x & 31) == 0) cur[T.NI + T.NG + T.NC + r] = v;
}

// One thread per face.  Faces [0, NI) are the right (top) faces of the
// interior leaves; faces [NI, NI+nu) are left (bottom) faces that are not
// shared with a same-level neighbour.  TB threads per block, at least MINB
// blocks per SM (the register budget follows from both).
template <int DIR, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) k_faces(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                    const DevScalars *__restrict__ sc, double g) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    int32_t a, b, c, d;
    if (f < T.NI) {
        const int32_t *s = T.ist + f * 8;
        if (DIR == 0) { a = s[1]; b = (int32_t)f; c = s[0]; d = s[4]; }
        else { a = s[3]; b = (int32_t)f; c = s[2]; d = s[6]; }
    } else {
        const int32_t i = DIR == 0 ? T.uxl[f - T.NI] : T.uyl[f - T.NI];
        const int32_t *s = T.ist + (int64_t)i * 8;
        if (DIR == 0) { a = s[5]; b = s[1]; c = i; d = s[0]; }
        else { a = s[7]; b = s[3]; c = i; d = s[2]; }
    }
    const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    double out[4];
    face_flux<DIR>(p0, p1, p2, p3, g, lam, out);
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// Four lanes per face (see face_flux in numerics.cuh for the per-face
// algebra).  All 32 lanes of a warp run the shuffles; lanes past the last
// face work on a clamped face and do not store.
template <int DIR>
__global__ void __launch_bounds__(256) k_faces4(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                const DevScalars *__restrict__ sc, double g) {
    const int64_t gt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nf = T.NI + (DIR == 0 ? T.nux : T.nuy);
    const int r = (int)(gt & 3);
    int64_t f = gt >> 2;
    const bool store = f < nf;
    if (!store) f = nf - 1;
    int32_t a, b, c, d;
    if (f < T.NI) {
        const int32_t *s = T.ist + f * 8;
        if (DIR == 0) { a = s[1]; b = (int32_t)f; c = s[0]; d = s[4]; }
        else { a = s[3]; b = (int32_t)f; c = s[2]; d = s[6]; }
    } else {
        const int32_t i = DIR == 0 ? T.uxl[f - T.NI] : T.uyl[f - T.NI];
        const int32_t *s = T.ist + (int64_t)i * 8;
        if (DIR == 0) { a = s[5]; b = s[1]; c = i; d = s[0]; }
        else { a = s[7]; b = s[3]; c = i; d = s[2]; }
    }
    const Prim P[4] = {load_prim(cur, a), load_prim(cur, b), load_prim(cur, c), load_prim(cur, d)};
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    double Um[4];
    {
        double U1[4], U2[4], Fd[4];
        cons_flux<DIR>(P[1], g, U1, Fd);
        cons_flux<DIR>(P[2], g, U2, Fd);
#pragma unroll
        for (int k = 0; k < 4; ++k) Um[k] = (U1[k] + U2[k]) / 2.0;
    }
    EigRow E;
    eigen_row<DIR>(Um, g, r, E);
    double w[4], q[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double Uk[4], Fk[4];
        cons_flux<DIR>(P[k], g, Uk, Fk);
        w[k] = project_row<DIR>(E, r, Uk);
        q[k] = project_row<DIR>(E, r, Fk);
    }
    const double uwL = wcns_z3(w[0], w[1], w[2]);
    const double uwR = wcns_z3(w[3], w[2], w[1]);
    const double ugL = wcns_z3(q[0], q[1], q[2]);
    const double ugR = wcns_z3(q[3], q[2], q[1]);
    double awL[4], awR[4], agL[4], agR[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        awL[k] = __shfl_sync(0xffffffffu, uwL, k, 4);
        awR[k] = __shfl_sync(0xffffffffu, uwR, k, 4);
        agL[k] = __shfl_sync(0xffffffffu, ugL, k, 4);
        agR[k] = __shfl_sync(0xffffffffu, ugR, k, 4);
    }
    const double wL = back_row<DIR>(E, r, awL), wR = back_row<DIR>(E, r, awR);
    const double gL = back_row<DIR>(E, r, agL), gR = back_row<DIR>(E, r, agR);
    const double out = 0.5 * (gL + gR - lam * (wR - wL));
    if (store) reinterpret_cast<double *>(F + f)[r] = out;
}

// Residual + forward-Euler candidate (LXL) fused with updateRK.
// mode 0: write the blended stage value into next; mode 1: write the
// primitive candidate Ut into next (no blend) for the split API.
__global__ void __launch_bounds__(256) k_cells(Tables T, LevelTab LT, const double4 *__restrict__ cur,
                                                const double4 *__restrict__ un, double4 *next,
                                                const double4 *__restrict__ Fx, const double4 *__restrict__ Fy,
                                                DevScalars *sc, double *res_part, int krk, int mode, double g) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double rm[4] = {0.0, 0.0, 0.0, 0.0}, rs[4] = {0.0, 0.0, 0.0, 0.0};
    double lx = 0.0, ly = 0.0;
    if (i < T.NI) {
        const int lvl = T.ilvl[i];
        const int32_t *s = T.ist + i * 8;
        const Prim q = load_prim(cur, i);
        const Prim qp = load_prim(cur, s[0]), qm = load_prim(cur, s[1]);
        const Prim rp = load_prim(cur, s[2]), rmn = load_prim(cur, s[3]);
        const double4 fxr = Fx[i], fxl = Fx[T.ifxl[i]];
        const double4 fyr = Fy[i], fyl = Fy[T.ifyl[i]];
        double Ep[4], Em[4], Gp[4], Gm[4];
        phys_flux<0>(qp, g, Ep);
        phys_flux<0>(qm, g, Em);
        phys_flux<1>(rp, g, Gp);
        phys_flux<1>(rmn, g, Gm);
        const double FR[4] = {fxr.x, fxr.y, fxr.z, fxr.w}, FL[4] = {fxl.x, fxl.y, fxl.z, fxl.w};
        const double HR[4] = {fyr.x, fyr.y, fyr.z, fyr.w}, HL[4] = {fyl.x, fyl.y, fyl.z, fyl.w};
        const double cxa = LT.cxa[lvl], cxb = LT.cxb[lvl], cya = LT.cya[lvl], cyb = LT.cyb[lvl];
        const double dx = LT.dx[lvl], dy = LT.dy[lvl];
        const double tstep = sc->tstep;
        double U[4];
        U[0] = q.r;
        U[1] = q.r * q.u;
        U[2] = q.r * q.v;
        U[3] = q.p / (g - 1.0) + 0.5 * q.r * (q.u * q.u + q.v * q.v);
        double Ut[4];
#pragma unroll
        for (int n = 0; n < 4; ++n) {
            const double dE = cxa * (FR[n] - FL[n]) - cxb * (Ep[n] - Em[n]);
            const double dF = cya * (HR[n] - HL[n]) - cyb * (Gp[n] - Gm[n]);
            const double fu = -dE - dF;
            Ut[n] = U[n] + fu * tstep;
            const double fr = fu * dx * dy;
            rm[n] = fabs(fr);
            rs[n] = fr * fr;
        }
        const double r0 = Ut[0];
        const double u0 = Ut[1] / Ut[0];
        const double v0 = Ut[2] / Ut[0];
        const double p0 = (g - 1.0) * r0 * (Ut[3] / r0 - 0.5 * (u0 * u0 + v0 * v0));
        double4 o;
        if (mode == 1) {
            o = make_double4(r0, u0, v0, p0);
        } else {
            const double4 n0 = un[i];
            const double ra = krk == 1 ? 0.0 : krk == 2 ? 3.0 / 4.0 : 1.0 / 3.0;
            const double rb = krk == 1 ? 1.0 : krk == 2 ? 1.0 / 4.0 : 2.0 / 3.0;
            o.x = ra * n0.x + rb * r0;
            o.y = ra * n0.y + rb * u0;
            o.z = ra * n0.z + rb * v0;
            o.w = ra * n0.w + rb * p0;
            if (krk == 3) {
                const double c = sqrt(g * o.w / o.x);
                lx = fabs(o.y) + c;
                ly = fabs(o.z) + c;
            }
        }
        next[i] = o;
    }
    // block reductions: residual max / sum of squares, lambda max
    __shared__ double sh[8][8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        for (int o = 16; o; o >>= 1) {
            rm[n] = fmax(rm[n], __shfl_xor_sync(0xffffffffu, rm[n], o));
            rs[n] += __shfl_xor_sync(0xffffffffu, rs[n], o);
        }
    }
    for (int o = 16; o; o >>= 1) {
        lx = fmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        ly = fmax(ly, __shfl_xor_sync(0xffffffffu, ly, o));
    }
    if (lane == 0) {
        for (int n = 0; n < 4; ++n) { sh[wid][n] = rm[n]; sh[wid][4 + n] = rs[n]; }
    }
    __shared__ double shl[8][2];
    if (lane == 0) { shl[wid][0] = lx; shl[wid][1] = ly; }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int n = threadIdx.x;
        double v = sh[0][n];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = n < 4 ? fmax(v, sh[w][n]) : v + sh[w][n];
        res_part[blockIdx.x * 8 + n] = v;
    }
    if (krk == 3 && mode == 0 && threadIdx.x == 0) {
        double a = shl[0][0], b = shl[0][1];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { a = fmax(a, shl[w][0]); b = fmax(b, shl[w][1]); }
        atomicMax((unsigned long long *)&sc->lam_next_x, (unsigned long long)__double_as_longlong(a));
        atomicMax((unsigned long long *)&sc->lam_next_y, (unsigned long long)__double_as_longlong(b));
    }
}

__global__ void k_blend(int64_t NI, const double4 *__restrict__ un, const double4 *__restrict__ ut, double4 *cur,
                        int krk) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= NI) return;
    const double ra = krk == 1 ? 0.0 : krk == 2 ? 3.0 / 4.0 : 1.0 / 3.0;
    const double rb = krk == 1 ? 1.0 : krk == 2 ? 1.0 / 4.0 : 2.0 / 3.0;
    const double4 a = un[i], b = ut[i];
    cur[i] = make_double4(ra * a.x + rb * b.x, ra * a.y + rb * b.y, ra * a.z + rb * b.z, ra * a.w + rb * b.w);
}

struct GhostStates {
    double s[6][4];   // bc_state[0..3], dmr_post, dmr_pre
    double x0, cot, speed;
};

// one warp per ghost leaf (interpA images can span hundreds of leaves)
__global__ void __launch_bounds__(128) k_ghost(Tables T, double4 *buf, GhostStates GS,
                                               const DevScalars *__restrict__ sc, int j) {
    __shared__ RestrictSmem sm[4];
    const int64_t gi = blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (gi >= T.NG) return;
    const int kind = T.gh_kind[gi];
    if (kind == GH_NONE) return;
    double4 v;
    if (kind == GH_RESTRICT) {
        v = restrict_warp(T, buf, T.gh_a[gi], T.gh_b[gi], sm[threadIdx.x >> 5]);
    } else if (kind == GH_COPY) {
        v = buf[T.gh_a[gi]];
    } else {
        // boundary time of body_boundary_RK (src/solution.F90:320-326)
        double t = sc->tt;
        if (j == 2) t = sc->tt + sc->tstep;
        else if (j == 3) t = sc->tt + 0.5 * sc->tstep;
        int st = T.gh_a[gi];
        if (kind == GH_DMR_TOP) {
            const double xs = GS.x0 + T.gh_y[gi] * GS.cot + GS.speed * t;
            st = T.gh_x[gi] < xs ? 4 : 5;
        }
        v = make_double4(GS.s[st][0], GS.s[st][1], GS.s[st][2], GS.s[st][3]);
    }
    if (lane != 0) return;
    const int fl = T.gh_flip[gi];
    if (fl == 1) v.y = -v.y;
    else if (fl == 2) v.z = -v.z;
    buf[T.NI + gi] = v;
}

__global__ void k_lambda(int64_t NI, const double4 *__restrict__ cur, DevScalars *sc, double g) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double lx = 0.0, ly = 0.0;
    if (i < NI) {
        const double4 o = cur[i];
        const double c = sqrt(g * o.w / o.x);
        lx = fabs(o.y) + c;
        ly = fabs(o.z) + c;
    }
    for (int o = 16; o; o >>= 1) {
        lx = fmax(lx, __shfl_xor_sync(0xffffffffu, lx, o));
        ly = fmax(ly, __shfl_xor_sync(0xffffffffu, ly, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax((unsigned long long *)&sc->lam_next_x, (unsigned long long)__double_as_longlong(lx));
        atomicMax((unsigned long long *)&sc->lam_next_y, (unsigned long long)__double_as_longlong(ly));
    }
}

// lambda/time-step control (src/solution.F90:185-201)
__global__ void k_step_control(DevScalars *sc, fdm_params P, int use_dt) {
    if (threadIdx.x || blockIdx.x) return;
    if (sc->done) return;
    sc->lambda_x = fmax(sc->lambda_x, sc->lam_next_x);
    sc->lambda_y = fmax(sc->lambda_y, sc->lam_next_y);
    sc->lam_next_x = 0.0;
    sc->lam_next_y = 0.0;
    if (use_dt && P.iflag_localdt) {
        const double div = (double)(1ll << sc->l_max);
        sc->tstep = P.cfl / (sc->lambda_x / (P.x_factor * P.h / div) + sc->lambda_y / (P.h / div));
    }
    if (sc->tt + sc->tstep > P.t_end) sc->tstep = P.t_end - sc->tt;
}

// residual partials -> Res_max / Res_rms sums; fixed reduction tree, so the
// result is identical run to run
__global__ void __launch_bounds__(256) k_res_finalize(const double *__restrict__ res_part, int nb, DevScalars *sc) {
    __shared__ double sh[256][8];
    double v[8];
    for (int n = 0; n < 8; ++n) v[n] = 0.0;
    for (int b = threadIdx.x; b < nb; b += 256)
        for (int n = 0; n < 8; ++n) v[n] = n < 4 ? fmax(v[n], res_part[b * 8 + n]) : v[n] + res_part[b * 8 + n];
    for (int n = 0; n < 8; ++n) sh[threadIdx.x][n] = v[n];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int n = 0; n < 8; ++n)
                sh[threadIdx.x][n] = n < 4 ? fmax(sh[threadIdx.x][n], sh[threadIdx.x + w][n])
                                           : sh[threadIdx.x][n] + sh[threadIdx.x + w][n];
        __syncthreads();
    }
    if (threadIdx.x < 8) {
        const int n = threadIdx.x;
        if (n < 4) sc->res_max[n] = sh[0][n];
        else sc->res_rms[n - 4] = sh[0][n];
    }
}

// end of one solute iteration: tt, rms, NaN stop, t_end (src/solution.F90:205-215)
__global__ void k_step_end(DevScalars *sc, int64_t NI) {
    if (threadIdx.x || blockIdx.x) return;
    if (sc->done) return;
    sc->tt = sc->tt + sc->tstep;
    sc->it = sc->it + 1;
    for (int n = 0; n < 4; ++n) {
        sc->res_rms[n] = sqrt(sc->res_rms[n] / (1.0 * (double)NI));
        if (isnan(sc->res_rms[n])) sc->status = FDM_ERR_NAN;
    }
    if (!(sc->tt < sc->t_end)) sc->done = 1;
}

__global__ void k_set_tstep(DevScalars *sc, double tstep) {
    if (threadIdx.x || blockIdx.x) return;
    sc->tstep = tstep;
}

// ------------------------------------------------------------ launchers
void launch_requests(fdm_handle *h, const double4 *cur) {
    if (h->NR == 0) return;
    k_requests<<<nblk(h->NR, 64), 64, 0, h->s>>>(h->tables(), (double4 *)cur);
    if (h->n_restrict > 0) k_requests_restrict<<<nblk(h->NR, 4), 128, 0, h->s>>>(h->tables(), (double4 *)cur);
}
// Launch shapes of the face kernel that the autotuner chooses from.
template <int TB, int MINB>
static void faces_1lane(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    k_faces<0, TB, MINB><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, h->G.gama);
    k_faces<1, TB, MINB><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, h->G.gama);
}
static void faces_4lane(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    k_faces4<0><<<nblk(4 * (h->NI + h->nux), 256), 256, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, h->G.gama);
    k_faces4<1><<<nblk(4 * (h->NI + h->nuy), 256), 256, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, h->G.gama);
}

const char *face_variant_name(int v) {
    switch (v) {
        case 0: return "1 thread/face, 128 threads, >=3 blocks/SM";
        case 1: return "1 thread/face, 128 threads, >=4 blocks/SM";
        case 2: return "1 thread/face, 64 threads, >=7 blocks/SM";
        case 3: return "1 thread/face, 256 threads, >=2 blocks/SM";
        case 4: return "4 threads/face, 256 threads";
        default: return "?";
    }
}

void launch_faces(fdm_handle *h, const double4 *cur, int krk) {
    if (h->gate_on) {
        launch_gated_faces(h, cur, krk);
        return;
    }
    switch (h->face_variant) {
        case 1: faces_1lane<128, 4>(h, cur); break;
        case 2: faces_1lane<64, 7>(h, cur); break;
        case 3: faces_1lane<256, 2>(h, cur); break;
        case 4: faces_4lane(h, cur); break;
        default: faces_1lane<128, 3>(h, cur); break;
    }
}

void launch_cells(fdm_handle *h, const double4 *cur, const double4 *un, double4 *next, int krk, int mode) {
    const int nb = nblk(h->NI, 256);
    k_cells<<<nb, 256, 0, h->s>>>(h->tables(), h->lt, cur, un, next, h->Fx.as<double4>(), h->Fy.as<double4>(),
                                  h->scal.as<DevScalars>(), h->res_part.as<double>(), krk, mode, h->G.gama);
    // Res_max / Res_rms are reset every stage and read after the last one
    // (src/solution.F90:276-277, 209-210): reduce them once, after stage 3
    if (krk == 3 || mode == 1) k_res_finalize<<<1, 256, 0, h->s>>>(h->res_part.as<double>(), nb, h->scal.as<DevScalars>());
}
void launch_ghosts(fdm_handle *h, double4 *next, int j) {
    if (h->NG == 0) return;
    GhostStates GS;
    for (int s = 0; s < 4; ++s)
        for (int k = 0; k < 4; ++k) GS.s[s][k] = h->p.bc_state[s][k];
    for (int k = 0; k < 4; ++k) { GS.s[4][k] = h->p.dmr_post[k]; GS.s[5][k] = h->p.dmr_pre[k]; }
    GS.x0 = h->p.dmr_x0;
    GS.cot = h->p.dmr_angle_cot;
    GS.speed = h->p.dmr_shock_speed;
    k_ghost<<<nblk(h->NG, 4), 128, 0, h->s>>>(h->tables(), next, GS, h->scal.as<DevScalars>(), j);
}
void launch_blend(fdm_handle *h, const double4 *un, double4 *cur, int krk) {
    k_blend<<<nblk(h->NI, 256), 256, 0, h->s>>>(h->NI, un, h->Ut.as<double4>(), cur, krk);
}
void launch_lambda(fdm_handle *h, const double4 *cur) {
    k_lambda<<<nblk(h->NI, 256), 256, 0, h->s>>>(h->NI, cur, h->scal.as<DevScalars>(), h->G.gama);
}
void launch_step_control(fdm_handle *h) {
    k_step_control<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>(), h->p, 1);
}
void launch_step_end(fdm_handle *h) {
    k_step_end<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>(), h->NI);
}
void launch_set_tstep(fdm_handle *h, double tstep) {
    k_set_tstep<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>(), tstep);
}

// One RK stage on the three state buffers: B0 holds the step-start state
// (Un); stage 1: B0 -> B1, stage 2: B1 -> B2, stage 3: B2 -> B0.
int launch_stage(fdm_handle *h, int krk) {
    double4 *b0 = h->B[0].as<double4>(), *b1 = h->B[1].as<double4>(), *b2 = h->B[2].as<double4>();
    const double4 *cur = krk == 1 ? b0 : krk == 2 ? b1 : b2;
    double4 *next = krk == 1 ? b1 : krk == 2 ? b2 : b0;
    launch_requests(h, cur);
    launch_faces(h, cur, krk);
    launch_cells(h, cur, b0, next, krk, 0);
    launch_ghosts(h, next, 3);
    return FDM_OK;
}

}  // namespace fdm
