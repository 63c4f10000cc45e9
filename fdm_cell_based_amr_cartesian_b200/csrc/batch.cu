// batch.cu — many independent meshes advanced together: one persistent
// kernel launch per SSP-RK3 stage covers every member of an ensemble.
//
// No reference counterpart (the reference runs one mesh per process).  Each
// member is an ordinary handle (its own tables, state buffers and scalars);
// the batch only schedules their work.  A launch runs the phases of one
// stage (step control, hanging-node requests, faces, hard faces of the
// learned gate, cells, ghosts and, at stage 3, the residual and the end of
// the step) for all members, separated by a grid barrier.  Inside a phase
// the blocks take (member, tile) pairs from one atomic counter, so members
// of very different sizes share the machine without a static split.  The
// per-item arithmetic is the single-mesh code (items.cuh, gate_items.cuh),
// so a member advanced in a batch matches the same handle advanced alone.
//
// The launch is cooperative (all blocks resident), and every wait in the
// grid barrier has a time limit, measured on the global timer: a barrier
// that does not complete sets an error word and the kernel returns, which
// the host reports as FDM_ERR_TIMEOUT.
#include <algorithm>
#include <atomic>
#include <cstddef>
#include <cstring>
#include <thread>
#include <vector>

#include "gate_items.cuh"
#include "numerics_nr.cuh"

struct fdm_batch;

namespace fdm {

__host__ __device__ __forceinline__ int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

constexpr int BT = 256;        // threads per block
constexpr int BW = BT / 32;    // warps per block
static_assert(BT == 4 * RQ_TILE, "a request tile is one block of four threads per request");

enum { PH_REQ = 0, PH_FACE, PH_HARD, PH_CELL, PH_GHOST, PH_GHOST1, N_PHASE };

struct Member {
    Tables T;
    LevelTab LT;
    double4 *B0, *B1, *B2;
    double4 *Fx, *Fy;
    DevScalars *sc;
    double *res_part;
    GhostStates GS;
    double gama;
    // step control (src/solution.F90:185-201)
    fdm_params p;
    int32_t amr_on;          // body_boundary(1) after each step
    int32_t has_restrict;
    // learned gate
    int32_t gate_on;
    float logit_thr;
    float jump_thr;
    const float *gate_P;
    GateLists GL;
    int64_t nfx, nfy;
    Den gm1;                 // gama - 1 with its correctly rounded reciprocal (branch-free division)
};

struct GridBar {
    unsigned count;
    unsigned gen;
    int err;
    int pad;
    unsigned long long limit_ns;   // wait limit of one barrier; 0: BAR_WAIT_NS
};

struct BatchArgs {
    const Member *mem;
    int nmem;
    int any_gate;
    const int64_t *off;            // [N_PHASE][nmem + 1] tile offsets (PH_HARD filled on the device)
    int64_t *off_hard;             // = off + PH_HARD * (nmem + 1)
    unsigned long long *ctr;       // [N_PHASE] tile counters, zero at launch
    GridBar *bar;
    int32_t *act;                  // member not finished at the start of the step
    const int32_t *skip_j1;        // host: a regrid follows this step (no body_boundary(1) here)
    unsigned long long *stamp;     // [3][16] global-timer stamps at the phase ends of each stage
    Den d2;                        // d2 of WCNS_Z3 with its correctly rounded reciprocal
};

// The full WCNS flux of face f of member M: in the reference's operation
// order (NRF false), or in the split order with the branch-free division
// (NRF true, the same bits; a face with an operand outside its range is
// computed again with the compiler's division).
template <int DIR, bool NRF>
__device__ __forceinline__ void batch_face(const Member &M, const double4 *__restrict__ cur, double4 *F, double lam,
                                           const Den &d2, int64_t f) {
    if constexpr (NRF) {
        int32_t a, b, c, d;
        face_slots<DIR>(M.T, f, a, b, c, d);
        double out[4];
        DivNR dv(M.gm1, d2);
        face_flux_slots_d<DIR>(cur, a, b, c, d, M.gama, dv, lam, out);
        if (!dv.ok) face_flux_slots<DIR>(cur, a, b, c, d, M.gama, lam, out);
        F[f] = make_double4(out[0], out[1], out[2], out[3]);
    } else {
        face_item<DIR, false>(M.T, cur, F, lam, M.gama, f);
    }
}

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// A wait gives up after BAR_WAIT_NS of global-timer time (or the batch's
// own limit), whatever the load on the GPU; the poll count is a second
// bound that holds even if the timer stood still (2^31 polls of >= 64 ns).
constexpr unsigned long long BAR_WAIT_NS = 2000000000ull;   // 2 s
constexpr unsigned long long BAR_POLL_CAP = 1ull << 31;

// Grid-wide barrier among the co-resident blocks of a cooperative launch.
// Returns false when any block gave up waiting; the caller then returns.
__device__ bool grid_bar(GridBar *b, unsigned nblocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *vgen = &b->gen;
        const unsigned g0 = *vgen;
        __threadfence();
        const unsigned arrived = atomicAdd(&b->count, 1u);
        if (arrived == nblocks - 1) {
            b->count = 0;
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            const unsigned long long lim = b->limit_ns ? b->limit_ns : BAR_WAIT_NS;
            const unsigned long long t0 = gtimer();
            unsigned long long polls = 0;
            while (*vgen == g0) {
                if (*(volatile int *)&b->err || gtimer() - t0 > lim || ++polls > BAR_POLL_CAP) {
                    atomicExch(&b->err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int *)&b->err == 0;
}

// Work stealing over the tiles of one phase: fn(member, tile) for every
// tile, each taken by one block from the phase's counter.
constexpr int OFF_CAP = 513;   // tile offsets kept in shared memory (members + 1)
template <class Fn>
__device__ __forceinline__ void run_tiles(const BatchArgs &A, int ph, const int64_t *goff, int64_t *s_t,
                                          int64_t *s_off, Fn &&fn) {
    const int64_t *off = goff;
    if (A.nmem + 1 <= OFF_CAP) {
        for (int k = threadIdx.x; k <= A.nmem; k += blockDim.x) s_off[k] = goff[k];
        __syncthreads();
        off = s_off;
    }
    const int64_t total = off[A.nmem];
    for (;;) {
        if (threadIdx.x == 0) *s_t = (int64_t)atomicAdd(A.ctr + ph, 1ull);
        __syncthreads();
        const int64_t t = *s_t;
        __syncthreads();
        if (t >= total) break;
        int lo = 0, hi = A.nmem;   // off[lo] <= t < off[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (off[mid] <= t) lo = mid;
            else hi = mid;
        }
        fn(lo, t - off[lo]);
    }
    __syncthreads();   // s_off is reloaded by the next phase
}

struct GateSmem {
    GateWeights W;
    XTile xt[BW];
};
union BatchSmem {
    double geo[RQ_TILE * RQ_GEO];   // geometry blocks of a request tile
    GateSmem gate;
    RestrictSmem rs[BW];
    CellsSmem cells;
    double fin[BT][8];
};

// 256 ghost leaves: copies and boundary states one per thread, then the
// interpA images of the tile one per warp
__device__ __forceinline__ void ghost_tile(const Tables &T, double4 *buf, const GhostStates &GS,
                                           const DevScalars *__restrict__ sc, int j, int64_t t, int32_t *rlist,
                                           int *rn, RestrictSmem *rs) {
    const int64_t gi = t * BT + threadIdx.x;
    if (threadIdx.x == 0) *rn = 0;
    __syncthreads();
    if (gi < T.NG) {
        const int kind = T.gh_kind[gi];
        if (kind == GH_RESTRICT) rlist[atomicAdd(rn, 1)] = (int32_t)threadIdx.x;
        else if (kind != GH_NONE) ghost_store(T, buf, gi, ghost_simple_value(T, buf, GS, sc, j, gi, kind));
    }
    __syncthreads();
    const int n = *rn, wid = threadIdx.x >> 5;
    for (int k = wid; k < n; k += BW) ghost_warp(T, buf, GS, sc, j, t * BT + rlist[k], rs[wid]);
    __syncthreads();
}

__device__ __forceinline__ const double4 *stage_cur(const Member &M, int krk) {
    return krk == 1 ? M.B0 : krk == 2 ? M.B1 : M.B2;
}
__device__ __forceinline__ double4 *stage_next(const Member &M, int krk) {
    return krk == 1 ? M.B1 : krk == 2 ? M.B2 : M.B0;
}

// ---- the phases of one stage, each item as the single-mesh code forms it.
// Shared by the persistent kernel (phases separated by grid barriers, tiles
// taken by work stealing) and the phase kernels (one launch per phase).

// step control and per-stage resets of member m (one thread)
__device__ __forceinline__ void ph_begin_member(const BatchArgs &A, int krk, int m) {
    const Member &M = A.mem[m];
    if (krk == 1) {
        A.act[m] = (!M.sc->done && M.sc->tt < M.p.t_end) ? 1 : 0;
        if (A.act[m]) step_control_item(M.sc, M.p, 1);
    }
    if (!A.act[m]) return;
    if (krk == 3) { M.sc->lam_next_x = 0.0; M.sc->lam_next_y = 0.0; }
    if (M.gate_on) {
        if (krk == 1) { M.GL.cnt[0] = 0; M.GL.cnt[1] = 0; }
        else { M.GL.cnt[0] = M.GL.cnt[2]; M.GL.cnt[1] = M.GL.cnt[3]; }
    }
}

// hanging-node requests: tile t of member m (whole block).  WLS tiles hold
// RQ_TILE requests, four threads each; interpA tiles hold BW listed
// fallbacks, one warp each.
__device__ __forceinline__ void ph_request_tile(const BatchArgs &A, int krk, int m, int64_t t, BatchSmem &S) {
    const Member &M = A.mem[m];
    if (!A.act[m]) return;
    double4 *cur = const_cast<double4 *>(stage_cur(M, krk));
    const int64_t nthr = cdiv(4 * M.T.NR, BT);
    const int wid = threadIdx.x >> 5;
    if (t < nthr) {
        // the tile's geometry blocks are contiguous: one staged copy
        // instead of four threads re-reading 768 bytes each
        stage_request_geometry(M.T, t * RQ_TILE, S.geo, BT);
        const int64_t q = t * BT + threadIdx.x;
        if ((q >> 2) < M.T.NR)
            request_item_var(M.T, cur, q >> 2, (int)(q & 3), S.geo + (threadIdx.x >> 2) * RQ_GEO);
        __syncthreads();   // the next tile's copy overwrites S.geo
    } else {
        const int64_t w = (t - nthr) * BW + wid;
        if (w < M.T.NRR) request_restrict_warp(M.T, cur, M.T.rq_rlist[w], S.rs[wid]);
    }
}

// faces: plain flux, or gate / guard with the linear flux (whole block);
// s_loaded names the gate weights held in S.gate
template <bool NRF>
__device__ __forceinline__ void ph_face_tile(const BatchArgs &A, int krk, int m, int64_t t, BatchSmem &S,
                                             const float *&s_loaded) {
    const Member &M = A.mem[m];
    if (!A.act[m]) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const double4 *cur = stage_cur(M, krk);
    const int64_t tx = cdiv(M.nfx, BT);
    const int dir = t < tx ? 0 : 1;
    const int64_t lt = dir == 0 ? t : t - tx;
    const int64_t nf = dir == 0 ? M.nfx : M.nfy;
    const double lam = dir == 0 ? M.sc->lambda_x : M.sc->lambda_y;
    if (!M.gate_on) {
        const int64_t f = lt * BT + threadIdx.x;
        if (f < nf) {
            if (dir == 0) batch_face<0, NRF>(M, cur, M.Fx, lam, A.d2, f);
            else batch_face<1, NRF>(M, cur, M.Fy, lam, A.d2, f);
        }
        return;
    }
    const double ig1 = 1.0 / (M.gama - 1.0);
    const int64_t w = lt * BW + wid;   // warp chunk of 32 faces
    if (krk == 1) {
        if (s_loaded != M.gate_P) {
            __syncthreads();
            load_weights_smem(S.gate.W, M.gate_P);
            for (int k = GF; k < XLD; ++k) S.gate.xt[wid].X[lane][k] = __float2bfloat16_rn(0.f);
            if (threadIdx.x == 0) s_loaded = M.gate_P;
            __syncthreads();
        }
        if (w * 32 < nf) {
            if (dir == 0)
                gate_linear_chunk<0>(M.T, cur, M.Fx, S.gate.W, S.gate.xt[wid], M.logit_thr, M.jump_thr, lam, ig1,
                                     M.gama, M.GL.hx, M.GL.cnt, M.GL.jx, w);
            else
                gate_linear_chunk<1>(M.T, cur, M.Fy, S.gate.W, S.gate.xt[wid], M.logit_thr, M.jump_thr, lam, ig1,
                                     M.gama, M.GL.hy, M.GL.cnt + 1, M.GL.jy, w);
        }
    } else if (w * 32 < nf) {
        if (dir == 0)
            guard_linear_chunk<0>(M.T, cur, M.Fx, M.GL.jx, lam, ig1, M.gama, M.GL.hx, M.GL.cnt, w);
        else
            guard_linear_chunk<1>(M.T, cur, M.Fy, M.GL.jy, lam, ig1, M.gama, M.GL.hy, M.GL.cnt + 1, w);
    }
}

// tile offsets of the hard faces of gated members (one thread)
__device__ __forceinline__ void ph_hard_offsets(const BatchArgs &A, int krk) {
    int64_t acc = 0;
    for (int m = 0; m < A.nmem; ++m) {
        A.off_hard[m] = acc;
        const Member &M = A.mem[m];
        if (!A.act[m] || !M.gate_on) continue;
        if (krk == 1) { M.GL.cnt[2] = M.GL.cnt[0]; M.GL.cnt[3] = M.GL.cnt[1]; }
        acc += cdiv(M.GL.cnt[0], BT) + cdiv(M.GL.cnt[1], BT);
    }
    A.off_hard[A.nmem] = acc;
}

// hard faces (full WCNS flux) of tile t of member m
template <bool NRF>
__device__ __forceinline__ void ph_hard_tile(const BatchArgs &A, int krk, int m, int64_t t) {
    const Member &M = A.mem[m];
    const double4 *cur = stage_cur(M, krk);
    const int64_t tx = cdiv(M.GL.cnt[0], BT);
    if (t < tx) {
        const int64_t i = t * BT + threadIdx.x;
        if (i < M.GL.cnt[0]) batch_face<0, NRF>(M, cur, M.Fx, M.sc->lambda_x, A.d2, M.GL.hx[i]);
    } else {
        const int64_t i = (t - tx) * BT + threadIdx.x;
        if (i < M.GL.cnt[1]) batch_face<1, NRF>(M, cur, M.Fy, M.sc->lambda_y, A.d2, M.GL.hy[i]);
    }
}

// cells: residual, candidate, RK blend, residual partials, lambda (whole block)
__device__ __forceinline__ void ph_cell_tile(const BatchArgs &A, int krk, int m, int64_t t, CellsSmem &S) {
    const Member &M = A.mem[m];
    if (!A.act[m]) return;
    const int64_t i = t * BT + threadIdx.x;
    double rm[4] = {0.0, 0.0, 0.0, 0.0}, rs[4] = {0.0, 0.0, 0.0, 0.0};
    double lx = 0.0, ly = 0.0;
    if (i < M.T.NI)
        cell_item(M.T, M.LT, stage_cur(M, krk), M.B0, stage_next(M, krk), M.Fx, M.Fy, M.sc->tstep, krk, 0, M.gama, i,
                  rm, rs, lx, ly);
    cells_block_reduce(rm, rs, lx, ly, M.res_part + t * 8, M.sc, krk == 3, S);
}

// ghosts of member m, tile t: j = 3 after a stage, j = 1 after a step
__device__ __forceinline__ void ph_ghost_tile(const BatchArgs &A, int krk, int j, int m, int64_t t, int32_t *rlist,
                                              int *rn, RestrictSmem *rs) {
    const Member &M = A.mem[m];
    if (!A.act[m]) return;
    if (j == 1 && (!M.amr_on || A.skip_j1[m])) return;
    ghost_tile(M.T, j == 1 ? M.B0 : stage_next(M, krk), M.GS, M.sc, j, t, rlist, rn, rs);
}

// end of the step of member m: residual norms, tt, it, NaN, t_end (whole block)
__device__ __forceinline__ void ph_end_member(const BatchArgs &A, int m, double (*fin)[8]) {
    const Member &M = A.mem[m];
    if (!A.act[m]) return;
    res_finalize_block(M.res_part, (int)cdiv(M.T.NI, BT), M.sc, fin);
    if (threadIdx.x == 0) step_end_item(M.sc, M.T.NI);
    __syncthreads();
}

// barrier, then block 0 stamps the time (phase k of stage krk ended)
#define BAR_STAMP(k)                                                                   \
    do {                                                                               \
        if (!grid_bar(A.bar, nb)) return;                                              \
        if (blockIdx.x == 0 && threadIdx.x == 0) A.stamp[(krk - 1) * 16 + (k)] = gtimer(); \
    } while (0)

// One RK stage (krk) of every member; MINB resident blocks per SM (the
// register budget follows: 128 per thread at 2, up to 255 at 1).
template <int MINB, bool NRF>
__global__ void __launch_bounds__(BT, MINB) k_batch_stage(BatchArgs A, int krk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem &S = *reinterpret_cast<BatchSmem *>(smem_raw);
    __shared__ int64_t s_t;
    __shared__ int64_t s_off[OFF_CAP];
    __shared__ const float *s_loaded;
    __shared__ int32_t s_rlist[BT];
    __shared__ int s_rn;
    const unsigned nb = gridDim.x;
    const int np1 = A.nmem + 1;
    if (blockIdx.x == 0 && threadIdx.x == 0) A.stamp[(krk - 1) * 16] = gtimer();

    // ---- step control / per-stage resets (one thread per member)
    if (blockIdx.x == 0)
        for (int m = threadIdx.x; m < A.nmem; m += BT) ph_begin_member(A, krk, m);
    BAR_STAMP(1);

    // ---- hanging-node requests
    run_tiles(A, PH_REQ, A.off + PH_REQ * np1, &s_t, s_off,
              [&](int m, int64_t t) { ph_request_tile(A, krk, m, t, S); });
    BAR_STAMP(2);

    // ---- faces: plain flux, or gate / guard with the linear flux
    if (threadIdx.x == 0) s_loaded = nullptr;
    __syncthreads();
    run_tiles(A, PH_FACE, A.off + PH_FACE * np1, &s_t, s_off,
              [&](int m, int64_t t) { ph_face_tile<NRF>(A, krk, m, t, S, s_loaded); });
    BAR_STAMP(3);

    // ---- hard faces of gated members (full WCNS flux)
    if (A.any_gate) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ph_hard_offsets(A, krk);
        BAR_STAMP(4);
        run_tiles(A, PH_HARD, A.off_hard, &s_t, s_off, [&](int m, int64_t t) { ph_hard_tile<NRF>(A, krk, m, t); });
        BAR_STAMP(5);
    }

    // ---- cells: residual, candidate, RK blend, residual partials, lambda
    run_tiles(A, PH_CELL, A.off + PH_CELL * np1, &s_t, s_off,
              [&](int m, int64_t t) { ph_cell_tile(A, krk, m, t, S.cells); });
    BAR_STAMP(6);

    // ---- ghosts of the new stage value (body_boundary_RK)
    run_tiles(A, PH_GHOST, A.off + PH_GHOST * np1, &s_t, s_off,
              [&](int m, int64_t t) { ph_ghost_tile(A, krk, 3, m, t, s_rlist, &s_rn, S.rs); });
    if (krk != 3) return;
    BAR_STAMP(7);

    // ---- end of the step: residual norms, tt, it, NaN, t_end
    for (int m = blockIdx.x; m < A.nmem; m += nb) ph_end_member(A, m, S.fin);
    BAR_STAMP(8);

    // ---- body_boundary(1) after the step on AMR members
    run_tiles(A, PH_GHOST1, A.off + PH_GHOST1 * np1, &s_t, s_off,
              [&](int m, int64_t t) { ph_ghost_tile(A, krk, 1, m, t, s_rlist, &s_rn, S.rs); });
}

// ---- phase kernels: one launch per phase covering every member, no grid
// barrier (the launches are ordered on the batch stream), each with the
// launch shape of its own work.  Blocks take the phase's tiles in a
// grid-stride loop; the member of a tile is found by binary search over the
// phase's tile offsets.
template <class Fn>
__device__ __forceinline__ void flat_tiles(const BatchArgs &A, const int64_t *goff, int64_t *s_off, Fn &&fn) {
    const int64_t *off = goff;
    if (A.nmem + 1 <= OFF_CAP) {
        for (int k = threadIdx.x; k <= A.nmem; k += blockDim.x) s_off[k] = goff[k];
        __syncthreads();
        off = s_off;
    }
    const int64_t total = off[A.nmem];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        int lo = 0, hi = A.nmem;   // off[lo] <= t < off[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (off[mid] <= t) lo = mid;
            else hi = mid;
        }
        fn(lo, t - off[lo]);
    }
}

__global__ void __launch_bounds__(BT) k_bp_begin(BatchArgs A, int krk) {
    for (int m = threadIdx.x; m < A.nmem; m += BT) ph_begin_member(A, krk, m);
}
__global__ void __launch_bounds__(BT) k_bp_requests(BatchArgs A, int krk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem &S = *reinterpret_cast<BatchSmem *>(smem_raw);
    __shared__ int64_t s_off[OFF_CAP];
    flat_tiles(A, A.off + PH_REQ * (A.nmem + 1), s_off, [&](int m, int64_t t) { ph_request_tile(A, krk, m, t, S); });
}
template <bool NRF>
__global__ void __launch_bounds__(BT, 2) k_bp_faces(BatchArgs A, int krk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem &S = *reinterpret_cast<BatchSmem *>(smem_raw);
    __shared__ int64_t s_off[OFF_CAP];
    __shared__ const float *s_loaded;
    if (threadIdx.x == 0) s_loaded = nullptr;
    __syncthreads();
    flat_tiles(A, A.off + PH_FACE * (A.nmem + 1), s_off,
               [&](int m, int64_t t) { ph_face_tile<NRF>(A, krk, m, t, S, s_loaded); });
}
__global__ void k_bp_hard_offsets(BatchArgs A, int krk) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ph_hard_offsets(A, krk);
}
template <bool NRF>
__global__ void __launch_bounds__(BT, 2) k_bp_hard(BatchArgs A, int krk) {
    __shared__ int64_t s_off[OFF_CAP];
    flat_tiles(A, A.off_hard, s_off, [&](int m, int64_t t) { ph_hard_tile<NRF>(A, krk, m, t); });
}
__global__ void __launch_bounds__(BT) k_bp_cells(BatchArgs A, int krk) {
    __shared__ CellsSmem s_cells;
    __shared__ int64_t s_off[OFF_CAP];
    flat_tiles(A, A.off + PH_CELL * (A.nmem + 1), s_off,
               [&](int m, int64_t t) { ph_cell_tile(A, krk, m, t, s_cells); });
}
__global__ void __launch_bounds__(BT) k_bp_ghosts(BatchArgs A, int krk, int j) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RestrictSmem *s_rs = reinterpret_cast<BatchSmem *>(smem_raw)->rs;
    __shared__ int32_t s_rlist[BT];
    __shared__ int s_rn;
    __shared__ int64_t s_off[OFF_CAP];
    flat_tiles(A, A.off + (j == 1 ? PH_GHOST1 : PH_GHOST) * (A.nmem + 1), s_off,
               [&](int m, int64_t t) { ph_ghost_tile(A, krk, j, m, t, s_rlist, &s_rn, s_rs); });
}
__global__ void __launch_bounds__(BT) k_bp_end(BatchArgs A) {
    __shared__ double s_fin[BT][8];
    for (int m = blockIdx.x; m < A.nmem; m += gridDim.x) ph_end_member(A, m, s_fin);
}

// Test of the bounded waits: a grid barrier that waits for one block more
// than the launch has, so every wait runs into its iteration limit, sets the
// error word and returns.
__global__ void k_barrier_timeout(GridBar *b, unsigned expected) { grid_bar(b, expected); }

}  // namespace fdm

using namespace fdm;

struct fdm_batch {
    std::vector<fdm_handle *> mem;
    int device = 0;
    cudaStream_t s = nullptr;
    DevBuf d_mem, d_off, d_ctr, d_bar, d_act, d_skip, d_stamp;
    std::vector<int32_t> h_skip;
    int grid = 0, blocks_per_sm = 0, want_bps = 2;   // want_bps 0: the members' own step graphs,
                                                     // 3: phase kernels (no persistent kernel)
    std::vector<int64_t> h_off;                      // tile offsets per phase (host copy)
    int sms = 0;
    bool face_nr = false;                            // branch-free division in the face phases
    size_t smem = 0;
    bool any_gate = false;
    cudaGraphExec_t graph = nullptr;
    bool graph_stale = false;   // the members changed: re-capture, update the graph in place
    bool use_graph = true;           // off when cooperative launches cannot be captured here
    std::vector<int64_t> versions;   // member table versions the descriptors were built for
    std::vector<bool> gates;
    std::vector<float> thr, jthr;
    cudaEvent_t ev = nullptr;
    unsigned long long wait_ns = 0;  // the grid barrier's wait limit (0: BAR_WAIT_NS)
    std::string err;
};

static int batch_fail(fdm_batch *b, cudaError_t e, const char *what) {
    b->err = std::string(what) + ": " + cudaGetErrorString(e);
    return FDM_ERR_CUDA;
}
#define BCK(b, x)                                             \
    do {                                                      \
        cudaError_t e_ = (x);                                 \
        if (e_ != cudaSuccess) return batch_fail(b, e_, #x);  \
    } while (0)

static void drop_batch_graph(fdm_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

// Member descriptors and tile offsets from the members' current tables.
static int batch_refresh(fdm_batch *b) {
    const int n = (int)b->mem.size();
    std::vector<Member> M(n);
    std::vector<int64_t> off((size_t)N_PHASE * (n + 1), 0);
    b->any_gate = false;
    for (int m = 0; m < n; ++m) {
        fdm_handle *h = b->mem[m];
        Member &d = M[m];
        std::memset(&d, 0, sizeof d);
        d.T = h->tables();
        d.LT = h->lt;
        d.B0 = h->B[0].as<double4>();
        d.B1 = h->B[1].as<double4>();
        d.B2 = h->B[2].as<double4>();
        d.Fx = h->Fx.as<double4>();
        d.Fy = h->Fy.as<double4>();
        d.sc = h->scal.as<DevScalars>();
        d.res_part = h->res_part.as<double>();
        d.GS = ghost_states(h->p);
        d.gama = h->G.gama;
        d.p = h->p;
        d.amr_on = h->p.iflag_amr ? 1 : 0;
        d.has_restrict = h->n_restrict > 0;
        d.nfx = h->NI + h->nux;
        d.nfy = h->NI + h->nuy;
        d.gate_on = h->gate_on;
        d.gm1 = Den{h->G.gama - 1.0, 1.0 / (h->G.gama - 1.0)};   // IEEE division on the host
        if (h->gate_on) {
            b->any_gate = true;
            d.logit_thr = h->gate_logit_thr;
            d.jump_thr = h->gate_jump_thr;
            d.gate_P = h->gate_params.as<float>();
            d.GL = gate_lists(h->gate_flag.p, d.nfx, d.nfy);
        }
        const int64_t tiles[N_PHASE] = {
            cdiv(4 * h->NR, BT) + cdiv(h->n_restrict, BW),               // PH_REQ
            cdiv(d.nfx, BT) + cdiv(d.nfy, BT),                          // PH_FACE
            0,                                                          // PH_HARD (device)
            cdiv(h->NI, BT),                                            // PH_CELL
            cdiv(h->NG, BT),                                            // PH_GHOST
            cdiv(h->NG, BT)};                                           // PH_GHOST1
        for (int ph = 0; ph < N_PHASE; ++ph) off[(size_t)ph * (n + 1) + m + 1] = off[(size_t)ph * (n + 1) + m] + tiles[ph];
    }
    BCK(b, b->d_mem.ensure(sizeof(Member) * n));
    BCK(b, b->d_off.ensure(sizeof(int64_t) * off.size()));
    BCK(b, cudaMemcpyAsync(b->d_mem.p, M.data(), sizeof(Member) * n, cudaMemcpyHostToDevice, b->s));
    BCK(b, cudaMemcpyAsync(b->d_off.p, off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice, b->s));
    b->h_off = off;
    BCK(b, cudaStreamSynchronize(b->s));
    b->versions.resize(n);
    b->gates.resize(n);
    b->thr.resize(n);
    b->jthr.resize(n);
    for (int m = 0; m < n; ++m) {
        b->versions[m] = b->mem[m]->table_version;
        b->gates[m] = b->mem[m]->gate_on;
        b->thr[m] = b->mem[m]->gate_logit_thr;
        b->jthr[m] = b->mem[m]->gate_jump_thr;
    }
    b->graph_stale = true;
    return FDM_OK;
}

static bool batch_stale(const fdm_batch *b) {
    for (size_t m = 0; m < b->mem.size(); ++m)
        if (b->versions[m] != b->mem[m]->table_version || b->gates[m] != b->mem[m]->gate_on ||
            b->thr[m] != b->mem[m]->gate_logit_thr || b->jthr[m] != b->mem[m]->gate_jump_thr)
            return true;
    return false;
}

// the persistent kernel of the batch's launch shape and face flux
static const void *batch_kernel(const fdm_batch *b) {
    if (b->want_bps == 1) return b->face_nr ? (const void *)k_batch_stage<1, true> : (const void *)k_batch_stage<1, false>;
    return b->face_nr ? (const void *)k_batch_stage<2, true> : (const void *)k_batch_stage<2, false>;
}

static int batch_grid(fdm_batch *b) {
    if (b->want_bps == 0) {   // no persistent kernel
        b->blocks_per_sm = 0;
        return FDM_OK;
    }
    if (b->want_bps == 3) {   // phase kernels: each launch sized by its own tiles
        BCK(b, cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
        BCK(b, cudaFuncSetAttribute(k_bp_requests, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        BCK(b, cudaFuncSetAttribute(k_bp_ghosts, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        BCK(b, cudaFuncSetAttribute(k_bp_faces<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        BCK(b, cudaFuncSetAttribute(k_bp_faces<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
        b->blocks_per_sm = 0;
        b->grid = 0;
        return FDM_OK;
    }
    int sms = 0, bps = 0;
    BCK(b, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    const void *fn = batch_kernel(b);
    BCK(b, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem));
    BCK(b, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, BT, b->smem));
    if (bps <= 0) { b->err = "the batch kernel does not fit on an SM"; return FDM_ERR_UNSUPPORTED; }
    b->blocks_per_sm = std::min(bps, b->want_bps);
    b->grid = sms * b->blocks_per_sm;
    return FDM_OK;
}

// One stage as phase kernels on the batch stream: each launch covers every
// member's tiles of one phase, in the order the persistent kernel runs the
// phases (the stream orders them; no grid barrier).
static int enqueue_phase_kernels(fdm_batch *b, const BatchArgs &A, int krk) {
    const int n1 = A.nmem + 1;
    auto total = [&](int ph) { return b->h_off[(size_t)ph * n1 + A.nmem]; };
    auto grid = [](int64_t t) { return (unsigned)std::min<int64_t>(t, 1ll << 30); };
    k_bp_begin<<<1, BT, 0, b->s>>>(A, krk);
    if (total(PH_REQ) > 0) k_bp_requests<<<grid(total(PH_REQ)), BT, b->smem, b->s>>>(A, krk);
    if (total(PH_FACE) > 0) {
        if (b->face_nr) k_bp_faces<true><<<grid(total(PH_FACE)), BT, b->smem, b->s>>>(A, krk);
        else k_bp_faces<false><<<grid(total(PH_FACE)), BT, b->smem, b->s>>>(A, krk);
    }
    if (A.any_gate) {
        // hard-face tiles are known on the device only: a grid-stride launch
        k_bp_hard_offsets<<<1, 32, 0, b->s>>>(A, krk);
        const unsigned g = (unsigned)(4 * b->sms);
        if (b->face_nr) k_bp_hard<true><<<g, BT, 0, b->s>>>(A, krk);
        else k_bp_hard<false><<<g, BT, 0, b->s>>>(A, krk);
    }
    if (total(PH_CELL) > 0) k_bp_cells<<<grid(total(PH_CELL)), BT, 0, b->s>>>(A, krk);
    if (total(PH_GHOST) > 0) k_bp_ghosts<<<grid(total(PH_GHOST)), BT, b->smem, b->s>>>(A, krk, 3);
    if (krk == 3) {
        k_bp_end<<<(unsigned)A.nmem, BT, 0, b->s>>>(A);
        if (total(PH_GHOST1) > 0) k_bp_ghosts<<<grid(total(PH_GHOST1)), BT, b->smem, b->s>>>(A, krk, 1);
    }
    BCK(b, cudaGetLastError());
    return FDM_OK;
}

static int enqueue_batch_stage(fdm_batch *b, int krk) {
    BatchArgs A;
    A.mem = b->d_mem.as<Member>();
    A.nmem = (int)b->mem.size();
    A.any_gate = b->any_gate ? 1 : 0;
    A.off = b->d_off.as<int64_t>();
    A.off_hard = const_cast<int64_t *>(A.off) + PH_HARD * (A.nmem + 1);
    A.ctr = b->d_ctr.as<unsigned long long>();
    A.bar = b->d_bar.as<GridBar>();
    A.act = b->d_act.as<int32_t>();
    A.skip_j1 = b->d_skip.as<int32_t>();
    A.stamp = b->d_stamp.as<unsigned long long>();
    A.d2 = Den{FDM_D2_WCNS, 1.0 / FDM_D2_WCNS};   // IEEE division on the host
    BCK(b, cudaMemsetAsync(A.ctr, 0, sizeof(unsigned long long) * N_PHASE, b->s));
    if (b->want_bps == 3) return enqueue_phase_kernels(b, A, krk);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->grid);
    cfg.blockDim = dim3(BT);
    cfg.dynamicSmemBytes = b->smem;
    cfg.stream = b->s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (b->want_bps == 1) {
        if (b->face_nr) BCK(b, cudaLaunchKernelEx(&cfg, k_batch_stage<1, true>, A, krk));
        else BCK(b, cudaLaunchKernelEx(&cfg, k_batch_stage<1, false>, A, krk));
    } else {
        if (b->face_nr) BCK(b, cudaLaunchKernelEx(&cfg, k_batch_stage<2, true>, A, krk));
        else BCK(b, cudaLaunchKernelEx(&cfg, k_batch_stage<2, false>, A, krk));
    }
    return FDM_OK;
}

// CUDA graph of one step of every member (three cooperative launches);
// captured again whenever a member's tables or gate change, and then
// updated in place when it keeps its shape (instantiated otherwise).  Where
// the capture of a cooperative launch is refused, the three launches are
// issued directly instead.
static int batch_graph(fdm_batch *b) {
    if (batch_stale(b)) {
        int rc = batch_refresh(b);
        if (rc) return rc;
    }
    if (!b->use_graph || (b->graph && !b->graph_stale)) return FDM_OK;
    cudaGraph_t g = nullptr;
    BCK(b, cudaStreamBeginCapture(b->s, cudaStreamCaptureModeThreadLocal));
    int rc = FDM_OK;
    for (int krk = 1; krk <= 3 && !rc; ++krk) rc = enqueue_batch_stage(b, krk);
    cudaError_t e = cudaStreamEndCapture(b->s, &g);
    if (!rc && e == cudaSuccess && b->graph) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(b->graph, g, &info) != cudaSuccess) {
            cudaGetLastError();   // another shape: instantiate it
            drop_batch_graph(b);
        }
    }
    if (!rc && e == cudaSuccess && !b->graph) {
        e = cudaGraphInstantiate(&b->graph, g, 0);
        if (e != cudaSuccess) b->graph = nullptr;
    }
    if (g) cudaGraphDestroy(g);
    b->graph_stale = false;
    if (rc || e != cudaSuccess || !b->graph) {
        cudaGetLastError();
        drop_batch_graph(b);
        b->use_graph = false;
        b->err.clear();
    }
    return FDM_OK;
}

static int launch_step(fdm_batch *b) {
    if (b->graph) {
        BCK(b, cudaGraphLaunch(b->graph, b->s));
        return FDM_OK;
    }
    for (int krk = 1; krk <= 3; ++krk) {
        int rc = enqueue_batch_stage(b, krk);
        if (rc) return rc;
    }
    return FDM_OK;
}

// members' queued work before the batch's, the batch's before theirs after
static int join_members(fdm_batch *b) {
    for (fdm_handle *h : b->mem) {
        BCK(b, cudaEventRecord(b->ev, h->s));
        BCK(b, cudaStreamWaitEvent(b->s, b->ev, 0));
    }
    return FDM_OK;
}
static int release_members(fdm_batch *b) {
    BCK(b, cudaEventRecord(b->ev, b->s));
    for (fdm_handle *h : b->mem) BCK(b, cudaStreamWaitEvent(h->s, b->ev, 0));
    return FDM_OK;
}

// the streams strategy: each active member's step graph on its own stream,
// after the batch stream's queued work and before the batch stream's next
static int launch_member_steps(fdm_batch *b, int64_t nsteps, const std::vector<int32_t> *regrid_next,
                               const std::vector<bool> *active) {
    int rc = release_members(b);
    if (rc) return rc;
    for (size_t m = 0; m < b->mem.size(); ++m) {
        if (active && !(*active)[m]) continue;
        fdm_handle *h = b->mem[m];
        for (int64_t k = 0; k < nsteps; ++k) {
            rc = member_launch_step(h, regrid_next && (*regrid_next)[m] != 0 && k + 1 == nsteps);
            if (rc) { b->err = "member " + std::to_string(m) + ": " + h->err; return rc; }
        }
    }
    return join_members(b);
}

// The regrids of the members due after this step.  They are independent
// (each member's own tables, buffers and stream), so several run at once,
// each from its own host thread with the batch's device current; the
// result of each is the one a serial loop gives.  The first failing member
// (lowest index) is reported.
constexpr int REGRID_THREADS = 16;
static int regrid_due_members(fdm_batch *b) {
    std::vector<int> due;
    for (int m = 0; m < (int)b->mem.size(); ++m)
        if (b->h_skip[m]) due.push_back(m);
    if (due.empty()) return FDM_OK;
    std::vector<int> rcs(due.size(), FDM_OK);
    if (due.size() == 1) {
        rcs[0] = member_regrid(b->mem[due[0]]);
    } else {
        std::atomic<size_t> next{0};
        auto work = [&]() {
            if (cudaSetDevice(b->device) != cudaSuccess) return;
            for (size_t i = next++; i < due.size(); i = next++) rcs[i] = member_regrid(b->mem[due[i]]);
        };
        const int nt = (int)std::min<size_t>(due.size(), REGRID_THREADS);
        std::vector<std::thread> pool;
        pool.reserve(nt);
        for (int t = 0; t < nt; ++t) pool.emplace_back(work);
        for (auto &t : pool) t.join();
        if (next.load() < due.size()) {   // a thread could not select the device
            b->err = "regrid threads could not select the device";
            return FDM_ERR_CUDA;
        }
    }
    for (size_t i = 0; i < due.size(); ++i)
        if (rcs[i]) {
            b->err = "member " + std::to_string(due[i]) + " regrid: " + b->mem[due[i]]->err;
            return rcs[i];
        }
    return FDM_OK;
}

static int check_barrier(fdm_batch *b) {
    if (b->want_bps == 0) {   // no grid barrier: the members' streams
        int rc = join_members(b);
        if (rc) return rc;
        BCK(b, cudaStreamSynchronize(b->s));
        return FDM_OK;
    }
    GridBar gb;
    BCK(b, cudaMemcpyAsync(&gb, b->d_bar.p, sizeof gb, cudaMemcpyDeviceToHost, b->s));
    BCK(b, cudaStreamSynchronize(b->s));
    if (gb.err) {
        // every block has left the kernel (the stream is idle): the barrier
        // starts again from zero for the next launch, its limit kept
        BCK(b, cudaMemsetAsync(b->d_bar.p, 0, offsetof(GridBar, limit_ns), b->s));
        BCK(b, cudaStreamSynchronize(b->s));
        b->err = "a grid barrier of the batch kernel gave up waiting (members' states of this step are undefined)";
        return FDM_ERR_TIMEOUT;
    }
    return FDM_OK;
}

extern "C" {

int fdm_batch_create(fdm_handle *const *members, int32_t n, fdm_batch **out) {
    if (!members || n <= 0 || !out) return FDM_ERR_ARG;
    *out = nullptr;
    int dev = -1;
    for (int m = 0; m < n; ++m) {
        if (!members[m] || !members[m]->loaded) return FDM_ERR_STATE;
        if (members[m]->p.flux_variant != 0) return FDM_ERR_UNSUPPORTED;   // the batch runs the exact flux
        if (dev < 0) dev = members[m]->device;
        if (members[m]->device != dev) return FDM_ERR_ARG;
        for (int k = 0; k < m; ++k)
            if (members[k] == members[m]) return FDM_ERR_ARG;
    }
    fdm_batch *b = new fdm_batch();
    b->mem.assign(members, members + n);
    b->device = dev;
    b->smem = sizeof(BatchSmem);
    cudaSetDevice(dev);
    int rc = FDM_OK;
    if (cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming) != cudaSuccess)
        rc = FDM_ERR_CUDA;
    if (!rc && (b->d_ctr.ensure(sizeof(unsigned long long) * N_PHASE) != cudaSuccess ||
                b->d_bar.ensure(sizeof(GridBar)) != cudaSuccess || b->d_act.ensure(sizeof(int32_t) * n) != cudaSuccess ||
                b->d_skip.ensure(sizeof(int32_t) * n) != cudaSuccess ||
                b->d_stamp.ensure(sizeof(unsigned long long) * 48) != cudaSuccess))
        rc = FDM_ERR_CUDA;
    if (!rc) {
        cudaMemsetAsync(b->d_bar.p, 0, sizeof(GridBar), b->s);
        cudaMemsetAsync(b->d_skip.p, 0, sizeof(int32_t) * n, b->s);
        cudaMemsetAsync(b->d_stamp.p, 0, sizeof(unsigned long long) * 48, b->s);
        b->h_skip.assign(n, 0);
        rc = batch_grid(b);
    }
    if (!rc) rc = batch_refresh(b);
    if (rc) {
        fdm_batch_destroy(b);
        return rc;
    }
    *out = b;
    return FDM_OK;
}

void fdm_batch_destroy(fdm_batch *b) {
    if (!b) return;
    if (b->s) cudaStreamSynchronize(b->s);
    drop_batch_graph(b);
    b->d_mem.release(); b->d_off.release(); b->d_ctr.release(); b->d_bar.release();
    b->d_act.release(); b->d_skip.release(); b->d_stamp.release();
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->s) cudaStreamDestroy(b->s);
    delete b;
}

int fdm_batch_last_error(const fdm_batch *b, char *buf, size_t n) {
    if (!b || !buf || n == 0) return FDM_ERR_ARG;
    const size_t k = std::min(b->err.size(), n - 1);
    std::memcpy(buf, b->err.data(), k);
    buf[k] = 0;
    return FDM_OK;
}

// nsteps solute iterations of every unfinished member, no regrid and no
// host synchronisation (graph replays on the batch stream).
int fdm_batch_advance(fdm_batch *b, int64_t nsteps) {
    fdm::Nvtx range("fdm_batch_advance");
    if (!b || nsteps < 0) return FDM_ERR_ARG;
    cudaSetDevice(b->device);
    for (fdm_handle *h : b->mem) {
        int rc = member_ready(h);
        if (rc) { b->err = "member: " + h->err; return rc; }
    }
    if (b->want_bps == 0) {
        int rc = launch_member_steps(b, nsteps, nullptr, nullptr);
        if (rc) return rc;
        for (fdm_handle *h : b->mem) member_stepped(h);
        return FDM_OK;
    }
    std::fill(b->h_skip.begin(), b->h_skip.end(), 0);
    int rc = join_members(b);
    if (rc) return rc;
    BCK(b, cudaMemcpyAsync(b->d_skip.p, b->h_skip.data(), sizeof(int32_t) * b->h_skip.size(), cudaMemcpyHostToDevice,
                           b->s));
    rc = batch_graph(b);
    if (rc) return rc;
    for (int64_t k = 0; k < nsteps; ++k) {
        rc = launch_step(b);
        if (rc) return rc;
    }
    for (fdm_handle *h : b->mem) member_stepped(h);
    return release_members(b);
}

// nsteps solute iterations with the members' regrids, as fdm_solute_step
// does for one mesh: after each step the scalars are read back; a NaN stops
// the batch (status of the first member that has it), and members whose
// regrid is due are regridded before the next step.  steps_done: steps
// taken.  Members past t_end are left alone.
int fdm_batch_solute(fdm_batch *b, int64_t nsteps, int64_t *steps_done) {
    fdm::Nvtx range("fdm_batch_solute");
    if (!b || nsteps < 0) return FDM_ERR_ARG;
    cudaSetDevice(b->device);
    const int n = (int)b->mem.size();
    int64_t k = 0;
    int rc = FDM_OK;
    std::vector<DevScalars> hs(n);
    for (fdm_handle *h : b->mem) {
        rc = member_ready(h);
        if (rc) { b->err = "member: " + h->err; return rc; }
    }
    for (; k < nsteps; ++k) {
        // a member regridded in the last iteration takes lambda over its new
        // leaves, as the step control of fdm_solute_step does (enqueued on
        // the member's stream, which the join below orders before the step)
        for (fdm_handle *h : b->mem) {
            rc = member_ready(h);
            if (rc) { b->err = "member: " + h->err; break; }
        }
        if (rc) break;
        // scalars before the step: finished members and regrids due after it
        rc = join_members(b);
        if (rc) break;
        for (int m = 0; m < n; ++m)
            BCK(b, cudaMemcpyAsync(&hs[m], b->mem[m]->scal.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, b->s));
        BCK(b, cudaStreamSynchronize(b->s));
        bool any = false;
        std::vector<bool> act(n, false);
        for (int m = 0; m < n; ++m) {
            const bool active = !hs[m].done && hs[m].tt < b->mem[m]->p.t_end;
            act[m] = active;
            any = any || active;
            b->h_skip[m] = active && member_amr_due(b->mem[m], hs[m].it + 1) ? 1 : 0;
        }
        if (!any) break;
        if (b->want_bps == 0) {
            rc = launch_member_steps(b, 1, &b->h_skip, &act);
            if (rc) break;
        } else {
            BCK(b, cudaMemcpyAsync(b->d_skip.p, b->h_skip.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, b->s));
            rc = batch_graph(b);
            if (rc) break;
            rc = launch_step(b);
            if (rc) break;
        }
        rc = check_barrier(b);
        if (rc) break;
        for (int m = 0; m < n; ++m)
            BCK(b, cudaMemcpyAsync(&hs[m], b->mem[m]->scal.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, b->s));
        BCK(b, cudaStreamSynchronize(b->s));
        for (fdm_handle *h : b->mem) member_stepped(h);
        for (int m = 0; m < n && !rc; ++m) {
            if (hs[m].status == FDM_ERR_NAN) {
                b->err = "member " + std::to_string(m) + ": NaN in the residual RMS";
                rc = FDM_ERR_NAN;
            }
        }
        if (rc) { ++k; break; }
        rc = regrid_due_members(b);
        if (rc) { ++k; break; }
    }
    if (steps_done) *steps_done = k;
    if (!rc) rc = release_members(b);
    return rc;
}

int fdm_batch_sync(fdm_batch *b) {
    if (!b) return FDM_ERR_ARG;
    return check_barrier(b);
}

// 1 or 2 resident blocks per SM for the persistent kernel (the next graph
// uses the new grid); 0: no persistent kernel, each member's own step graph
// on its own stream; 3: no persistent kernel, one launch per phase covering
// every member (each phase at the launch shape of its own work).
int fdm_batch_set_blocks_per_sm(fdm_batch *b, int32_t bps) {
    if (!b || bps < 0 || bps > 3) return FDM_ERR_ARG;
    b->want_bps = bps;
    int rc = batch_grid(b);
    if (rc) return rc;
    drop_batch_graph(b);
    return FDM_OK;
}

// Face phases of the persistent kernel: the reference's operation order
// (0) or the split order with the branch-free division (1); the same bits.
int fdm_batch_set_face_flux(fdm_batch *b, int32_t branch_free) {
    if (!b || branch_free < 0 || branch_free > 1) return FDM_ERR_ARG;
    cudaSetDevice(b->device);
    b->face_nr = branch_free != 0;
    int rc = batch_grid(b);
    if (rc) return rc;
    drop_batch_graph(b);
    return FDM_OK;
}

// Wait limit of one grid barrier of the persistent kernel, in seconds
// (default 2 s); the next launch uses it.
int fdm_batch_set_wait_limit(fdm_batch *b, double seconds) {
    if (!b || !(seconds > 0.0) || seconds > 3600.0) return FDM_ERR_ARG;
    cudaSetDevice(b->device);
    b->wait_ns = (unsigned long long)(seconds * 1e9);
    if (b->wait_ns == 0) b->wait_ns = 1;
    BCK(b, cudaMemcpyAsync((char *)b->d_bar.p + offsetof(GridBar, limit_ns), &b->wait_ns, sizeof b->wait_ns,
                           cudaMemcpyHostToDevice, b->s));
    BCK(b, cudaStreamSynchronize(b->s));
    return FDM_OK;
}

int fdm_batch_info(const fdm_batch *b, int32_t *grid, int32_t *blocks_per_sm, int64_t *smem_bytes) {
    if (!b) return FDM_ERR_ARG;
    if (grid) *grid = b->grid;
    if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
    if (smem_bytes) *smem_bytes = (int64_t)b->smem;
    return FDM_OK;
}

// Microseconds spent in each phase of the last step, per stage: row krk-1,
// column k = phase k (0 step control, then requests, faces, [hard-list
// offsets, hard faces,] cells, ghosts, [step end, level-1 ghosts]); unused
// entries are 0.
int fdm_batch_phase_us(fdm_batch *b, double *us) {
    if (!b || !us) return FDM_ERR_ARG;
    unsigned long long st[48];
    BCK(b, cudaMemcpyAsync(st, b->d_stamp.p, sizeof st, cudaMemcpyDeviceToHost, b->s));
    BCK(b, cudaStreamSynchronize(b->s));
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 16; ++k) {
            const unsigned long long a = st[r * 16 + k], c = k < 15 ? st[r * 16 + k + 1] : 0;
            us[r * 16 + k] = (k < 15 && c > a && a) ? (double)(c - a) * 1e-3 : 0.0;
        }
    return FDM_OK;
}

// the batch stream (events, timing)
int fdm_batch_stream(const fdm_batch *b, void **stream) {
    if (!b || !stream) return FDM_ERR_ARG;
    *stream = (void *)b->s;
    return FDM_OK;
}

// 2 blocks in a grid barrier that expects 3: returns FDM_ERR_TIMEOUT when
// the waits gave up (the expected outcome) and their device time in
// *seconds; the context stays usable.
int fdm_debug_barrier_timeout(double *seconds) {
    fdm::GridBar *d = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    fdm::GridBar hb{};
    int rc = FDM_ERR_CUDA;
    if (cudaMalloc((void **)&d, sizeof(fdm::GridBar)) != cudaSuccess) return FDM_ERR_NOMEM;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess && cudaEventCreate(&e0) == cudaSuccess &&
        cudaEventCreate(&e1) == cudaSuccess && cudaMemsetAsync(d, 0, sizeof(fdm::GridBar), s) == cudaSuccess &&
        cudaEventRecord(e0, s) == cudaSuccess) {
        fdm::k_barrier_timeout<<<2, 32, 0, s>>>(d, 3u);
        if (cudaGetLastError() == cudaSuccess && cudaEventRecord(e1, s) == cudaSuccess &&
            cudaMemcpyAsync(&hb, d, sizeof hb, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
            cudaStreamSynchronize(s) == cudaSuccess) {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (seconds) *seconds = ms * 1e-3;
            rc = hb.err ? FDM_ERR_TIMEOUT : FDM_OK;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(d);
    return rc;
}

}  // extern "C"
