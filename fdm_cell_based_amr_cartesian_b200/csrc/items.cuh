// items.cuh — the per-item work of one SSP-RK3 stage, shared by the
// single-mesh kernels (stage.cu, gate.cu) and the batched persistent kernel
// (batch.cu), so both paths run the same arithmetic:
//
//   request_item / request_restrict_warp   hanging-node values
//                                          (src/XuanGua.F90:45-398)
//   face_item                              WCNS flux of one face
//                                          (src/nnd_center_RK.F90:66-353)
//   cell_item + cells_block_reduce         residual, forward-Euler candidate,
//                                          RK3 blend, residual norms, lambda
//                                          (src/nnd_center_RK.F90:15-64,
//                                           src/solution.F90:279-286,386-404)
//   ghost_warp                             boundary images
//                                          (src/solution.F90:288-293,109-168)
//   step_control_item / step_end_item /    solute bookkeeping
//   res_finalize_block                     (src/solution.F90:185-215)
#pragma once

#include "handle.cuh"
#include "numerics.cuh"

namespace fdm {

// interpA over a subtree whose leaves are [lo, hi) of the sorted array
// (src/XuanGua.F90:359-398): children combined as
// 0.25*(son1 + son2 + son3 + son4) = 0.25*(((q0 + q1) + q3) + q2).
// One warp: the lanes stage the subtree's leaves in shared memory.  A
// subtree of up to RW_CAP leaves is folded level by level by all lanes; a
// larger one is folded by lane 0 in key order with a stack of pending
// sibling groups.  Every father is formed from the same four values in the
// same order either way.
constexpr int RW_CAP = 256;     // leaves staged per pass
constexpr int RW_STACK = 48;    // >= 3 pending siblings x 15 levels + 1
struct RestrictSmem {
    double4 v[RW_CAP];
    int8_t l[RW_CAP];
    union {
        struct {
            double4 st[RW_STACK];
            int8_t sl[RW_STACK];
        } s;                   // the stack of the lane-0 fold
        uint32_t p[RW_CAP];    // path bits of the staged entries (level fold)
    } u;
};

// the fold of n <= RW_CAP leaves from lo: at the deepest level present,
// every group of four siblings (consecutive in key order, the first with
// digit 0) becomes its father; the list is compacted and the next level up
// follows
__device__ __forceinline__ double4 restrict_warp_levels(const Tables &T, const double4 *__restrict__ buf,
                                                        int64_t lo, int n, RestrictSmem &sm) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int lmax = 0;
    for (int k = lane; k < n; k += 32) {
        const uint64_t key = __ldg(T.lkey + lo + k);
        sm.v[k] = buf[__ldg(T.lslot + lo + k)];
        sm.l[k] = (int8_t)(key & 15u);
        sm.u.p[k] = (uint32_t)((key >> 4) & ((1ull << 30) - 1ull));
        lmax = max(lmax, (int)(key & 15u));
    }
    lmax = __reduce_max_sync(FULL, lmax);
    __syncwarp();
    while (n > 1 && lmax > 0) {
        const int sh = 2 * (LMAX - lmax);
        int off = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            double4 vi = make_double4(0.0, 0.0, 0.0, 0.0);
            int8_t li = 0;
            uint32_t pi = 0;
            bool keep = false;
            if (i < n) {
                vi = sm.v[i];
                li = sm.l[i];
                pi = sm.u.p[i];
                const bool deep = li == lmax;
                const bool first = deep && ((pi >> sh) & 3u) == 0u && i + 3 < n;
                keep = !deep || first;
                if (first) {   // the father (its path: the first son's, digit 0)
                    const double4 e0 = vi, e1 = sm.v[i + 1], e2 = sm.v[i + 2], e3 = sm.v[i + 3];
                    vi.x = 0.25 * (e0.x + e1.x + e3.x + e2.x);
                    vi.y = 0.25 * (e0.y + e1.y + e3.y + e2.y);
                    vi.z = 0.25 * (e0.z + e1.z + e3.z + e2.z);
                    vi.w = 0.25 * (e0.w + e1.w + e3.w + e2.w);
                    li = (int8_t)(lmax - 1);
                }
            }
            const unsigned km = __ballot_sync(FULL, keep);
            const int pos = off + __popc(km & ((1u << lane) - 1u));
            off += __popc(km);
            __syncwarp();
            if (keep) {   // positions only move down, below what later chunks read
                sm.v[pos] = vi;
                sm.l[pos] = li;
                sm.u.p[pos] = pi;
            }
            __syncwarp();
        }
        n = off;
        --lmax;
    }
    const double4 r = sm.v[0];
    __syncwarp();
    return r;
}

__device__ __forceinline__ double4 restrict_warp(const Tables &T, const double4 *__restrict__ buf, int64_t lo,
                                                 int64_t hi, RestrictSmem &sm) {
    if (hi - lo <= RW_CAP) return restrict_warp_levels(T, buf, lo, (int)(hi - lo), sm);
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
                sm.u.s.st[top] = sm.v[k];
                sm.u.s.sl[top] = sm.l[k];
                ++top;
                while (top >= 4 && sm.u.s.sl[top - 1] == sm.u.s.sl[top - 2] && sm.u.s.sl[top - 1] == sm.u.s.sl[top - 3] &&
                       sm.u.s.sl[top - 1] == sm.u.s.sl[top - 4]) {
                    const double4 e0 = sm.u.s.st[top - 4], e1 = sm.u.s.st[top - 3], e2 = sm.u.s.st[top - 2], e3 = sm.u.s.st[top - 1];
                    double4 v;
                    v.x = 0.25 * (e0.x + e1.x + e3.x + e2.x);
                    v.y = 0.25 * (e0.y + e1.y + e3.y + e2.y);
                    v.z = 0.25 * (e0.z + e1.z + e3.z + e2.z);
                    v.w = 0.25 * (e0.w + e1.w + e3.w + e2.w);
                    const int8_t l = (int8_t)(sm.u.s.sl[top - 1] - 1);
                    top -= 4;
                    sm.u.s.st[top] = v;
                    sm.u.s.sl[top] = l;
                    ++top;
                }
            }
        }
        __syncwarp();
    }
    double4 r = sm.u.s.st[0];
    __syncwarp();
    return r;
}

// hanging-node request r of kind WLS or COPY (RESTRICT: request_restrict_warp)
__device__ __forceinline__ void request_item(const Tables &T, double4 *cur, int64_t r) {
    const int64_t out = T.NI + T.NG + T.NC + r;
    const int kind = T.rq_kind[r];
    const int32_t *mem = T.rq_mem + r * WLS_MAXM;
    if (kind == RQ_COPY) {
        cur[out] = cur[mem[0]];
        return;
    }
    if (kind == RQ_RESTRICT) return;
    const int m1 = T.rq_m[2 * r], m2 = T.rq_m[2 * r + 1];
    const int m = m1 + m2;
    const double *geo = T.rq_geo + r * RQ_GEO;
    double ph[4][WLS_MAXM];
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) {
        const double4 q = i < m ? cur[mem[i]] : make_double4(0.0, 0.0, 0.0, 0.0);
        ph[0][i] = q.x; ph[1][i] = q.y; ph[2][i] = q.z; ph[3][i] = q.w;
    }
    double4 v;
    v.x = wls_eval_var(geo, m1, m2, ph[0]);
    v.y = wls_eval_var(geo, m1, m2, ph[1]);
    v.z = wls_eval_var(geo, m1, m2, ph[2]);
    v.w = wls_eval_var(geo, m1, m2, ph[3]);
    cur[out] = v;
}

// component v (0..3) of hanging-node request r of kind WLS or COPY: the
// four components of a value are independent, so four threads can share a
// request.  geo: the request's geometry block (global memory, or a copy of
// it in shared memory).
__device__ __forceinline__ void request_item_var(const Tables &T, double4 *cur, int64_t r, int v,
                                                 const double *geo) {
    const int64_t out = T.NI + T.NG + T.NC + r;
    const int kind = T.rq_kind[r];
    const int32_t *mem = T.rq_mem + r * WLS_MAXM;
    double *o = reinterpret_cast<double *>(cur + out) + v;
    if (kind == RQ_COPY) {
        *o = reinterpret_cast<const double *>(cur + mem[0])[v];
        return;
    }
    if (kind == RQ_RESTRICT) return;
    const int m1 = T.rq_m[2 * r], m2 = T.rq_m[2 * r + 1];
    const int m = m1 + m2;
    double ph[WLS_MAXM];
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) ph[i] = i < m ? reinterpret_cast<const double *>(cur + mem[i])[v] : 0.0;
    *o = wls_eval_var(geo, m1, m2, ph);
}

// The geometry blocks of the RQ_TILE requests from r0 on (contiguous in
// rq_geo) into shared memory, 16 bytes per cp.async; all BT threads of the
// block call it, and it returns after the copy has landed and the block has
// synchronised.
constexpr int RQ_TILE = 64;
__device__ __forceinline__ void stage_request_geometry(const Tables &T, int64_t r0, double *smem_geo, int nthreads) {
    int64_t nreq = T.NR - r0;
    if (nreq > RQ_TILE) nreq = RQ_TILE;
    const int nch = nreq > 0 ? (int)(nreq * RQ_GEO / 2) : 0;   // 16-byte chunks
    const double *src = T.rq_geo + r0 * RQ_GEO;
    for (int k = threadIdx.x; k < nch; k += nthreads) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(smem_geo + 2 * k);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + 2 * k));
    }
    asm volatile("cp.async.commit_group;\n" ::);
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
}

__device__ __forceinline__ void request_item_var(const Tables &T, double4 *cur, int64_t r, int v) {
    const int64_t out = T.NI + T.NG + T.NC + r;
    const int kind = T.rq_kind[r];
    const int32_t *mem = T.rq_mem + r * WLS_MAXM;
    double *o = reinterpret_cast<double *>(cur + out) + v;
    if (kind == RQ_COPY) {
        *o = reinterpret_cast<const double *>(cur + mem[0])[v];
        return;
    }
    if (kind == RQ_RESTRICT) return;
    const int m1 = T.rq_m[2 * r], m2 = T.rq_m[2 * r + 1];
    const int m = m1 + m2;
    const double *geo = T.rq_geo + r * RQ_GEO;
    double ph[WLS_MAXM];
#pragma unroll
    for (int i = 0; i < WLS_MAXM; ++i) ph[i] = i < m ? reinterpret_cast<const double *>(cur + mem[i])[v] : 0.0;
    *o = wls_eval_var(geo, m1, m2, ph);
}

// interpA fallback of parent_value_weno for request r (whole warp)
__device__ __forceinline__ void request_restrict_warp(const Tables &T, double4 *cur, int64_t r, RestrictSmem &sm) {
    if (T.rq_kind[r] != RQ_RESTRICT) return;
    const double4 v = restrict_warp(T, cur, T.rq_m[2 * r], T.rq_m[2 * r + 1], sm);
    if ((threadIdx.x & 31) == 0) cur[T.NI + T.NG + T.NC + r] = v;
}

// The four stencil slots of face f.  Faces [0, NI) are the right (top) faces
// of the interior leaves; faces [NI, NI+nu) are left (bottom) faces that are
// not shared with a same-level neighbour.
template <int DIR>
__device__ __forceinline__ void face_slots(const Tables &T, int64_t f, int32_t &a, int32_t &b, int32_t &c,
                                           int32_t &d) {
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
}

template <int DIR, bool SPLIT = true>
__device__ __forceinline__ void face_item(const Tables &T, const double4 *__restrict__ cur, double4 *F, double lam,
                                          double g, int64_t f) {
    int32_t a, b, c, d;
    face_slots<DIR>(T, f, a, b, c, d);
    double out[4];
    if constexpr (SPLIT) {   // the records read again for the flux half: fewer live registers
        face_flux_slots<DIR>(cur, a, b, c, d, g, lam, out);
    } else {
        const Prim p0 = load_prim(cur, a), p1 = load_prim(cur, b), p2 = load_prim(cur, c), p3 = load_prim(cur, d);
        face_flux<DIR, false>(p0, p1, p2, p3, g, lam, out);
    }
    F[f] = make_double4(out[0], out[1], out[2], out[3]);
}

// Residual + forward-Euler candidate (LXL) fused with updateRK for leaf i.
// mode 0: write the blended stage value into next; mode 1: write the
// primitive candidate Ut into next (no blend) for the split API.  rm / rs /
// lx / ly receive the leaf's residual norms and (stage 3) wave speeds.
__device__ __forceinline__ void cell_item(const Tables &T, const LevelTab &LT, const double4 *__restrict__ cur,
                                          const double4 *__restrict__ un, double4 *next,
                                          const double4 *__restrict__ Fx, const double4 *__restrict__ Fy,
                                          double tstep, int krk, int mode, double g, int64_t i, double rm[4],
                                          double rs[4], double &lx, double &ly) {
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

// Block reduction of one 256-leaf tile: residual max / sum of squares into
// res_slot[0..7], lambda maxima into the scalars at stage 3.  Called by all
// threads of a 256-thread block; sh / shl are the block's shared scratch.
struct CellsSmem {
    double sh[8][8];
    double shl[8][2];
};
__device__ __forceinline__ void cells_block_reduce(double rm[4], double rs[4], double lx, double ly,
                                                   double *res_slot, DevScalars *sc, bool lam, CellsSmem &S) {
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
        for (int n = 0; n < 4; ++n) { S.sh[wid][n] = rm[n]; S.sh[wid][4 + n] = rs[n]; }
        S.shl[wid][0] = lx;
        S.shl[wid][1] = ly;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        const int n = threadIdx.x;
        double v = S.sh[0][n];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = n < 4 ? fmax(v, S.sh[w][n]) : v + S.sh[w][n];
        res_slot[n] = v;
    }
    if (lam && threadIdx.x == 0) {
        double a = S.shl[0][0], b = S.shl[0][1];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { a = fmax(a, S.shl[w][0]); b = fmax(b, S.shl[w][1]); }
        atomicMax((unsigned long long *)&sc->lam_next_x, (unsigned long long)__double_as_longlong(a));
        atomicMax((unsigned long long *)&sc->lam_next_y, (unsigned long long)__double_as_longlong(b));
    }
    __syncthreads();
}

struct GhostStates {
    double s[6][4];   // bc_state[0..3], dmr_post, dmr_pre
    double x0, cot, speed;
};

// value of a ghost leaf of kind COPY or a boundary state
__device__ __forceinline__ double4 ghost_simple_value(const Tables &T, const double4 *buf, const GhostStates &GS,
                                                      const DevScalars *__restrict__ sc, int j, int64_t gi,
                                                      int kind) {
    if (kind == GH_COPY) return buf[T.gh_a[gi]];
    // boundary time of body_boundary_RK (src/solution.F90:320-326)
    double t = sc->tt;
    if (j == 2) t = sc->tt + sc->tstep;
    else if (j == 3) t = sc->tt + 0.5 * sc->tstep;
    int st = T.gh_a[gi];
    if (kind == GH_DMR_TOP) {
        const double xs = GS.x0 + T.gh_y[gi] * GS.cot + GS.speed * t;
        st = T.gh_x[gi] < xs ? 4 : 5;
    }
    return make_double4(GS.s[st][0], GS.s[st][1], GS.s[st][2], GS.s[st][3]);
}
// mirror (wall) flip and store of a ghost value
__device__ __forceinline__ void ghost_store(const Tables &T, double4 *buf, int64_t gi, double4 v) {
    const int fl = T.gh_flip[gi];
    if (fl == 1) v.y = -v.y;
    else if (fl == 2) v.z = -v.z;
    buf[T.NI + gi] = v;
}

// ghost leaf gi (whole warp: interpA images can span hundreds of leaves)
__device__ __forceinline__ void ghost_warp(const Tables &T, double4 *buf, const GhostStates &GS,
                                           const DevScalars *__restrict__ sc, int j, int64_t gi, RestrictSmem &sm) {
    const int lane = threadIdx.x & 31;
    const int kind = T.gh_kind[gi];
    if (kind == GH_NONE) return;
    double4 v;
    if (kind == GH_RESTRICT) v = restrict_warp(T, buf, T.gh_a[gi], T.gh_b[gi], sm);
    else v = ghost_simple_value(T, buf, GS, sc, j, gi, kind);
    if (lane != 0) return;
    ghost_store(T, buf, gi, v);
}

__host__ inline GhostStates ghost_states(const fdm_params &p) {
    GhostStates GS;
    for (int s = 0; s < 4; ++s)
        for (int k = 0; k < 4; ++k) GS.s[s][k] = p.bc_state[s][k];
    for (int k = 0; k < 4; ++k) { GS.s[4][k] = p.dmr_post[k]; GS.s[5][k] = p.dmr_pre[k]; }
    GS.x0 = p.dmr_x0;
    GS.cot = p.dmr_angle_cot;
    GS.speed = p.dmr_shock_speed;
    return GS;
}

// lambda/time-step control (src/solution.F90:185-201); one thread
__device__ __forceinline__ void step_control_item(DevScalars *sc, const fdm_params &P, int use_dt) {
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

// residual partials -> Res_max / Res_rms sums over a fixed reduction tree,
// so the result is identical run to run; all threads of a 256-thread block
__device__ __forceinline__ void res_finalize_block(const double *__restrict__ res_part, int nb, DevScalars *sc,
                                                   double (*sh)[8]) {
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
    __syncthreads();
}

// end of one solute iteration: tt, rms, NaN stop, t_end
// (src/solution.F90:205-215); one thread
__device__ __forceinline__ void step_end_item(DevScalars *sc, int64_t NI) {
    if (sc->done) return;
    sc->tt = sc->tt + sc->tstep;
    sc->it = sc->it + 1;
    for (int n = 0; n < 4; ++n) {
        sc->res_rms[n] = sqrt(sc->res_rms[n] / (1.0 * (double)NI));
        if (isnan(sc->res_rms[n])) sc->status = FDM_ERR_NAN;
    }
    // the reference stops at t_end and at a NaN residual: later iterations
    // are no-ops
    if (!(sc->tt < sc->t_end) || sc->status == FDM_ERR_NAN) sc->done = 1;
}

}  // namespace fdm
