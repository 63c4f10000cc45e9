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
#include "items.cuh"
#include "numerics.cuh"
#include "numerics_nr.cuh"
#include "numerics_sm.cuh"

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

// four threads per request, one per component
__global__ void __launch_bounds__(256) k_requests4(Tables T, double4 *cur) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t r = g >> 2;
    if (r >= T.NR) return;
    request_item_var(T, cur, r, (int)(g & 3));
}

// interpA fallbacks of parent_value_weno: one warp per listed request
__global__ void __launch_bounds__(128) k_requests_restrict(Tables T, double4 *cur) {
    __shared__ RestrictSmem sm[4];
    const int64_t w = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (w >= T.NRR) return;
    request_restrict_warp(T, cur, T.rq_rlist[w], sm[threadIdx.x >> 5]);
}

// One thread per face; TB threads per block, at least MINB blocks per SM
// (the register budget follows from both).
template <int DIR, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) k_faces(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                    const DevScalars *__restrict__ sc, double g) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    face_item<DIR>(T, cur, F, DIR == 0 ? sc->lambda_x : sc->lambda_y, g, f);
}

// The same faces with every division formed by DivNR (numerics_nr.cuh):
// identical quotients without the branches of the compiler's division, so
// the reconstructions of a face can be interleaved.  A face with an operand
// outside DivNR's range is computed again with the compiler's division.
template <int DIR, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) k_faces_nr(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                       const DevScalars *__restrict__ sc, double g, Den gm1,
                                                       Den d2) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    double out[4];
    DivNR dv(gm1, d2);
    face_flux_slots_d<DIR>(cur, a, b, c, d, g, dv, lam, out);
    if (!dv.ok) face_flux_slots<DIR>(cur, a, b, c, d, g, lam, out);
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// One thread per face in the reference's operation order (the four states
// and fluxes formed first), with the compiler's division (NR false) or the
// branch-free one (NR true; a face with an operand outside its range is
// computed again with the compiler's division).
template <int DIR, int TB, int MINB, bool NR>
__global__ void __launch_bounds__(TB, MINB) k_faces_ref(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                        const DevScalars *__restrict__ sc, double g, Den gm1,
                                                        Den d2) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
    double out[4];
    if constexpr (NR) {
        DivNR dv(gm1, d2);
        face_flux_ref_d<DIR>(p0, p1, p2, p3, g, dv, lam, out);
        if (!dv.ok) face_flux<DIR, false>(p0, p1, p2, p3, g, lam, out);
    } else {
        face_flux<DIR, false>(p0, p1, p2, p3, g, lam, out);
    }
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// The faces with the constant denominators divided by one correction
// (DivConst, numerics_nr.cuh), every other division as the compiler forms
// it; SPLIT: the split order (state half, then flux half), else the
// reference's order.  A face with an operand outside the range is computed
// again with the compiler's division.
template <int DIR, int TB, int MINB, bool SPLIT>
__global__ void __launch_bounds__(TB, MINB) k_faces_c(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                      const DevScalars *__restrict__ sc, double g, DenC gm1,
                                                      DenC d2) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    double out[4];
    DivConst dv(gm1, d2);
    if constexpr (SPLIT) {
        face_flux_slots_d<DIR>(cur, a, b, c, d, g, dv, lam, out);
        if (!dv.ok) face_flux_slots<DIR>(cur, a, b, c, d, g, lam, out);
    } else {
        const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
        face_flux_ref_d<DIR>(p0, p1, p2, p3, g, dv, lam, out);
        if (!dv.ok) face_flux<DIR, false>(p0, p1, p2, p3, g, lam, out);
    }
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// Variant 15's arithmetic with the face's characteristic basis in shared
// memory (numerics_sm.cuh): fewer live registers, so more warps per SM.
template <int DIR, int TB, int MINB>
__global__ void __launch_bounds__(TB, MINB) k_faces_sm(Tables T, const double4 *__restrict__ cur, double4 *F,
                                                       const DevScalars *__restrict__ sc, double g, DenC gm1,
                                                       DenC d2) {
    __shared__ EigShared<TB> S;
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    if (f >= T.NI + nu) return;
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    const double lam = DIR == 0 ? sc->lambda_x : sc->lambda_y;
    double out[4];
    DivConst dv(gm1, d2);
    face_flux_slots_sm<DIR, TB>(cur, a, b, c, d, g, dv, lam, S, threadIdx.x, out);
    if (!dv.ok) {   // the compiler's division, the basis again in shared memory
        DivIEEE di(g);
        face_flux_slots_sm<DIR, TB>(cur, a, b, c, d, g, di, lam, S, threadIdx.x, out);
    }
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// Diagnostics: the faces whose branch-free division meets an operand
// outside its range (and so are computed again with the compiler's
// division), counted over the current state; nothing is written to F.
template <int DIR>
__global__ void __launch_bounds__(128) k_faces_nr_count(Tables T, const double4 *__restrict__ cur,
                                                        const DevScalars *__restrict__ sc, double g, Den gm1,
                                                        Den d2, unsigned long long *count) {
    const int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t nu = DIR == 0 ? T.nux : T.nuy;
    bool fell = false;
    if (f < T.NI + nu) {
        int32_t a, b, c, d;
        face_slots<DIR>(T, f, a, b, c, d);
        double out[4];
        DivNR dv(gm1, d2);
        face_flux_slots_d<DIR>(cur, a, b, c, d, g, dv, DIR == 0 ? sc->lambda_x : sc->lambda_y, out);
        fell = !dv.ok;
    }
    const unsigned m = __ballot_sync(0xffffffffu, fell);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}
int count_nr_fallbacks(fdm_handle *h, int64_t out[2]) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const double g = h->G.gama;
    const Den gm1{g - 1.0, 1.0 / (g - 1.0)}, d2{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};
    FDM_CK(h, h->tmp[7].ensure(2 * sizeof(unsigned long long)));
    unsigned long long *cnt = h->tmp[7].as<unsigned long long>();
    FDM_CK(h, cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), h->s));
    launch_requests(h, h->B[0].as<double4>());
    k_faces_nr_count<0><<<nblk(h->NI + h->nux, 128), 128, 0, h->s>>>(T, h->B[0].as<double4>(), sc, g, gm1, d2, cnt);
    k_faces_nr_count<1><<<nblk(h->NI + h->nuy, 128), 128, 0, h->s>>>(T, h->B[0].as<double4>(), sc, g, gm1, d2,
                                                                       cnt + 1);
    unsigned long long hc[2];
    FDM_CK(h, cudaMemcpyAsync(hc, cnt, sizeof hc, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    out[0] = (int64_t)hc[0];
    out[1] = (int64_t)hc[1];
    return FDM_OK;
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

// Residual + forward-Euler candidate fused with updateRK, 256 leaves per
// block (the residual partials are per block of 256).
__global__ void __launch_bounds__(256) k_cells(Tables T, LevelTab LT, const double4 *__restrict__ cur,
                                                const double4 *__restrict__ un, double4 *next,
                                                const double4 *__restrict__ Fx, const double4 *__restrict__ Fy,
                                                DevScalars *sc, double *res_part, int krk, int mode, double g) {
    __shared__ CellsSmem S;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double rm[4] = {0.0, 0.0, 0.0, 0.0}, rs[4] = {0.0, 0.0, 0.0, 0.0};
    double lx = 0.0, ly = 0.0;
    // an iteration after t_end (or after a NaN residual) leaves the state as it is
    if (i < T.NI && !(mode == 0 && sc->done))
        cell_item(T, LT, cur, un, next, Fx, Fy, sc->tstep, krk, mode, g, i, rm, rs, lx, ly);
    cells_block_reduce(rm, rs, lx, ly, res_part + blockIdx.x * 8, sc, krk == 3 && mode == 0, S);
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

// ghost leaves imaged by a copy or a boundary state: one thread each
__global__ void __launch_bounds__(256) k_ghost_simple(Tables T, double4 *buf, GhostStates GS,
                                                      const DevScalars *__restrict__ sc, int j) {
    const int64_t gi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (gi >= T.NG) return;
    const int kind = T.gh_kind[gi];
    if (kind == GH_NONE || kind == GH_RESTRICT) return;
    ghost_store(T, buf, gi, ghost_simple_value(T, buf, GS, sc, j, gi, kind));
}

// ghost leaves imaged by a subtree restriction (interpA images can span
// hundreds of leaves): one warp each
__global__ void __launch_bounds__(128) k_ghost(Tables T, double4 *buf, GhostStates GS,
                                               const DevScalars *__restrict__ sc, int j) {
    __shared__ RestrictSmem sm[4];
    const int64_t gi = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (gi >= T.NG) return;
    if (T.gh_kind[gi] != GH_RESTRICT) return;
    ghost_warp(T, buf, GS, sc, j, gi, sm[threadIdx.x >> 5]);
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
    step_control_item(sc, P, use_dt);
}

// residual partials -> Res_max / Res_rms sums
__global__ void __launch_bounds__(256) k_res_finalize(const double *__restrict__ res_part, int nb, DevScalars *sc,
                                                      int keep_when_done) {
    __shared__ double sh[256][8];
    if (keep_when_done && sc->done) return;   // a no-op iteration keeps the last residual
    res_finalize_block(res_part, nb, sc, sh);
}

// end of one solute iteration: tt, rms, NaN stop, t_end (src/solution.F90:205-215)
__global__ void k_step_end(DevScalars *sc, int64_t NI) {
    if (threadIdx.x || blockIdx.x) return;
    step_end_item(sc, NI);
}

__global__ void k_set_tstep(DevScalars *sc, double tstep) {
    if (threadIdx.x || blockIdx.x) return;
    sc->tstep = tstep;
}

// ------------------------------------------------------------ launchers
void launch_requests(fdm_handle *h, const double4 *cur) {
    if (h->NR == 0) return;
    k_requests4<<<nblk(4 * h->NR, 256), 256, 0, h->s>>>(h->tables(), (double4 *)cur);
    if (h->n_restrict > 0)
        k_requests_restrict<<<nblk(h->n_restrict, 4), 128, 0, h->s>>>(h->tables(), (double4 *)cur);
}
// Launch shapes of the face kernel that the autotuner chooses from.
template <int TB, int MINB>
static void faces_1lane(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    k_faces<0, TB, MINB><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, h->G.gama);
    k_faces<1, TB, MINB><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, h->G.gama);
}
template <int TB, int MINB>
static void faces_nr(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const double g = h->G.gama;
    // constant denominators with their correctly rounded reciprocals (IEEE
    // division on the host)
    const Den gm1{g - 1.0, 1.0 / (g - 1.0)}, d2{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};
    k_faces_nr<0, TB, MINB><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, g, gm1, d2);
    k_faces_nr<1, TB, MINB><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, g, gm1, d2);
}
template <int TB, int MINB, bool NR>
static void faces_ref(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const double g = h->G.gama;
    const Den gm1{g - 1.0, 1.0 / (g - 1.0)}, d2{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};
    k_faces_ref<0, TB, MINB, NR><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, g, gm1, d2);
    k_faces_ref<1, TB, MINB, NR><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, g, gm1, d2);
}
template <int TB, int MINB, bool SPLIT>
static void faces_c(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const double g = h->G.gama;
    const DenC gm1{g - 1.0, 1.0 / (g - 1.0)}, d2{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};
    k_faces_c<0, TB, MINB, SPLIT><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, g, gm1, d2);
    k_faces_c<1, TB, MINB, SPLIT><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, g, gm1, d2);
}
template <int TB, int MINB>
static void faces_sm(fdm_handle *h, const double4 *cur) {
    const Tables T = h->tables();
    const DevScalars *sc = h->scal.as<DevScalars>();
    const double g = h->G.gama;
    const DenC gm1{g - 1.0, 1.0 / (g - 1.0)}, d2{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};
    k_faces_sm<0, TB, MINB><<<nblk(h->NI + h->nux, TB), TB, 0, h->s>>>(T, cur, h->Fx.as<double4>(), sc, g, gm1, d2);
    k_faces_sm<1, TB, MINB><<<nblk(h->NI + h->nuy, TB), TB, 0, h->s>>>(T, cur, h->Fy.as<double4>(), sc, g, gm1, d2);
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
        case 5: return "1 thread/face, 128 threads, >=5 blocks/SM";
        case 6: return "1 thread/face, 64 threads, >=10 blocks/SM";
        case 7: return "1 thread/face, branch-free division, 128 threads, >=3 blocks/SM";
        case 8: return "1 thread/face, branch-free division, 128 threads, >=4 blocks/SM";
        case 9: return "1 thread/face, branch-free division, 256 threads, >=2 blocks/SM";
        case 10: return "1 thread/face, branch-free division, 64 threads, >=10 blocks/SM";
        case 11: return "1 thread/face, reference order, 256 threads, >=2 blocks/SM";
        case 12: return "1 thread/face, reference order, 128 threads, >=4 blocks/SM";
        case 13: return "1 thread/face, reference order, branch-free division, 256 threads, >=2 blocks/SM";
        case 14: return "1 thread/face, reference order, branch-free division, 128 threads, >=4 blocks/SM";
        case 15: return "1 thread/face, constant divisors by one correction, 256 threads, >=2 blocks/SM";
        case 16: return "1 thread/face, constant divisors by one correction, 64 threads, >=10 blocks/SM";
        case 17: return "1 thread/face, reference order, constant divisors by one correction, 256 threads, >=2 blocks/SM";
        case 18: return "1 thread/face, variant 15 with the basis in shared memory, 128 threads, >=4 blocks/SM";
        case 19: return "1 thread/face, variant 15 with the basis in shared memory, 128 threads, >=5 blocks/SM";
        case 20: return "1 thread/face, variant 15 with the basis in shared memory, 128 threads, >=6 blocks/SM";
        default: return "?";
    }
}

void launch_faces(fdm_handle *h, const double4 *cur, int krk) {
    if (h->gate_on) {
        launch_gated_faces(h, cur, krk);
        return;
    }
    if (h->p.flux_variant == 1) {
        launch_faces_fast(h, cur);
        return;
    }
    switch (h->face_variant) {
        case 1: faces_1lane<128, 4>(h, cur); break;
        case 2: faces_1lane<64, 7>(h, cur); break;
        case 3: faces_1lane<256, 2>(h, cur); break;
        case 4: faces_4lane(h, cur); break;
        case 5: faces_1lane<128, 5>(h, cur); break;
        case 6: faces_1lane<64, 10>(h, cur); break;
        case 7: faces_nr<128, 3>(h, cur); break;
        case 8: faces_nr<128, 4>(h, cur); break;
        case 9: faces_nr<256, 2>(h, cur); break;
        case 10: faces_nr<64, 10>(h, cur); break;
        case 11: faces_ref<256, 2, false>(h, cur); break;
        case 12: faces_ref<128, 4, false>(h, cur); break;
        case 13: faces_ref<256, 2, true>(h, cur); break;
        case 14: faces_ref<128, 4, true>(h, cur); break;
        case 15: faces_c<256, 2, true>(h, cur); break;
        case 16: faces_c<64, 10, true>(h, cur); break;
        case 17: faces_c<256, 2, false>(h, cur); break;
        case 18: faces_sm<128, 4>(h, cur); break;
        case 19: faces_sm<128, 5>(h, cur); break;
        case 20: faces_sm<128, 6>(h, cur); break;
        default: faces_1lane<128, 3>(h, cur); break;
    }
}

void launch_cells(fdm_handle *h, const double4 *cur, const double4 *un, double4 *next, int krk, int mode) {
    const int nb = nblk(h->NI, 256);
    k_cells<<<nb, 256, 0, h->s>>>(h->tables(), h->lt, cur, un, next, h->Fx.as<double4>(), h->Fy.as<double4>(),
                                  h->scal.as<DevScalars>(), h->res_part.as<double>(), krk, mode, h->G.gama);
    // Res_max / Res_rms are reset every stage and read after the last one
    // (src/solution.F90:276-277, 209-210): reduce them once, after stage 3
    if (krk == 3 || mode == 1)
        k_res_finalize<<<1, 256, 0, h->s>>>(h->res_part.as<double>(), nb, h->scal.as<DevScalars>(), mode == 0);
}
void launch_ghosts(fdm_handle *h, double4 *next, int j) {
    if (h->NG == 0) return;
    const GhostStates GS = ghost_states(h->p);
    k_ghost_simple<<<nblk(h->NG, 256), 256, 0, h->s>>>(h->tables(), next, GS, h->scal.as<DevScalars>(), j);
    if (h->n_ghost_restrict > 0)
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
