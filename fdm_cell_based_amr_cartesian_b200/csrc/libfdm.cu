// libfdm.cu — the extern "C" boundary (include/fdm.h).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "handle.cuh"
#include "topo.cuh"

using namespace fdm;

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

__global__ void k_reset_lam(DevScalars *sc) {
    if (threadIdx.x || blockIdx.x) return;
    sc->lam_next_x = 0.0;
    sc->lam_next_y = 0.0;
}

__global__ void k_out(int64_t NL, const int32_t *lslot, const double4 *B0, double *prim) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    const double4 v = B0[lslot[k]];
    prim[4 * k] = v.x; prim[4 * k + 1] = v.y; prim[4 * k + 2] = v.z; prim[4 * k + 3] = v.w;
}
__global__ void k_in(int64_t NL, const int32_t *lslot, double4 *B0, const double *prim) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    B0[lslot[k]] = make_double4(prim[4 * k], prim[4 * k + 1], prim[4 * k + 2], prim[4 * k + 3]);
}
// halo records of a strip: gather / scatter at caller-given slots; a slot
// outside the leaf slots is skipped and flagged
__global__ void k_pack_slots(int64_t n, const int32_t *__restrict__ slots, int64_t ns, const double4 *B,
                             double *buf, int32_t *bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t s = slots[i];
    if (s < 0 || s >= ns) { atomicExch(bad, 1); return; }
    const double4 v = B[s];
    buf[4 * i] = v.x; buf[4 * i + 1] = v.y; buf[4 * i + 2] = v.z; buf[4 * i + 3] = v.w;
}
__global__ void k_unpack_slots(int64_t n, const int32_t *__restrict__ slots, int64_t ns, double4 *B,
                               const double *buf, int32_t *bad) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t s = slots[i];
    if (s < 0 || s >= ns) { atomicExch(bad, 1); return; }
    B[s] = make_double4(buf[4 * i], buf[4 * i + 1], buf[4 * i + 2], buf[4 * i + 3]);
}
__global__ void k_set_global_lambda(DevScalars *sc, double lx, double ly, int32_t l_max) {
    if (threadIdx.x || blockIdx.x) return;
    sc->lambda_x = lx;
    sc->lambda_y = ly;
    sc->lam_next_x = 0.0;
    sc->lam_next_y = 0.0;
    sc->l_max = l_max;
}
__global__ void k_stencil_out(Tables T, const double4 *B, double *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    for (int s = 0; s < 8; ++s) {
        const double4 v = B[T.ist[i * 8 + s]];
        double *o = out + (i * 8 + s) * 4;
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
}
__global__ void k_neighbors_out(Tables T, Geometry G, uint64_t *out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= T.NL) return;
    NodeRef c;
    c.n = node_of_key(T.lkey[k]);
    c.leaf = (int32_t)k;
    c.valid = 1;
    NodeRef nb[8];
    nb[0] = face_nb(T, G, c, DIR_UP);
    nb[1] = face_nb(T, G, c, DIR_DOWN);
    nb[2] = face_nb(T, G, c, DIR_RIGHT);
    nb[3] = face_nb(T, G, c, DIR_LEFT);
    if (root_cross(G, c.n.root) >= 0) {
        nb[4] = upleft_nb(T, G, c);
        nb[5] = upright_nb(T, G, c);
        nb[6] = downleft_nb(T, G, c);
        nb[7] = downright_nb(T, G, c);
    } else {
        for (int d = 4; d < 8; ++d) nb[d] = null_ref();
    }
    for (int d = 0; d < 8; ++d) out[k * 8 + d] = nb[d].valid ? node_key(nb[d].n) : ~0ull;
}

// hanging-node stencil of every (interior leaf, entry), in the encoding of
// the oracle's gather export: 0 leaf copy, 1 parent WLS, 2 parent interpA,
// 3 child WLS, 4 child copy
__global__ void k_requests_out(Tables T, int32_t *kind, uint64_t *node, double *xy, int32_t *m12,
                               uint64_t *mem) {
    const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= T.NI * 8) return;
    const int32_t s = T.ist[o];
    const int64_t VS0 = T.NI + T.NG + T.NC;
    for (int k = 0; k < 16; ++k) mem[o * 16 + k] = ~0ull;
    if (s < VS0) {
        kind[o] = 0;
        node[o] = T.lkey[T.slot_leaf[s]];
        xy[2 * o] = 0.0; xy[2 * o + 1] = 0.0;
        m12[2 * o] = 0; m12[2 * o + 1] = 0;
        return;
    }
    const int64_t r = s - VS0;
    const double *geo = T.rq_geo + r * RQ_GEO;
    const int k = T.rq_kind[r];
    const bool child = geo[G_ORIGIN] != 0.0;
    kind[o] = child ? (k == RQ_WLS ? 3 : 4) : (k == RQ_WLS ? 1 : 2);
    node[o] = T.rq_node[r];
    xy[2 * o] = geo[G_XX];
    xy[2 * o + 1] = geo[G_YY];
    if (k == RQ_WLS) {
        const int m1 = T.rq_m[2 * r], m2 = T.rq_m[2 * r + 1];
        m12[2 * o] = m1; m12[2 * o + 1] = m2;
        for (int i = 0; i < m1 + m2 && i < 16; ++i) mem[o * 16 + i] = T.lkey[T.slot_leaf[T.rq_mem[r * WLS_MAXM + i]]];
    } else {
        m12[2 * o] = -1; m12[2 * o + 1] = -1;
    }
}

static int sync_scalars_from_device(fdm_handle *h) {
    FDM_CK(h, cudaMemcpyAsync(h->hs, h->scal.p, sizeof(DevScalars), cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}
static int push_scalars(fdm_handle *h) {
    FDM_CK(h, cudaMemcpyAsync(h->scal.p, h->hs, sizeof(DevScalars), cudaMemcpyHostToDevice, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

// the lambda maxima of a leading handle, taken before a step (paired runs)
__global__ void k_take_lambda(const DevScalars *__restrict__ from, DevScalars *to) {
    if (threadIdx.x || blockIdx.x) return;
    to->lambda_x = from->lambda_x;
    to->lambda_y = from->lambda_y;
    to->lam_next_x = from->lam_next_x;
    to->lam_next_y = from->lam_next_y;
}

static int ensure_lambda(fdm_handle *h) {
    if (h->lam_fresh) return FDM_OK;
    k_reset_lam<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>());
    launch_lambda(h, h->B[0].as<double4>());
    h->lam_fresh = true;
    return FDM_OK;
}

// end of a split-API call: wait for it, or (asynchronous mode) only check
// that the launches were accepted
static int split_done(fdm_handle *h) {
    if (h->split_async) {
        FDM_CK(h, cudaGetLastError());
    } else {
        FDM_CK(h, cudaStreamSynchronize(h->s));
    }
    return FDM_OK;
}

// getRKn + 3 x (solution_cell, updateRK, body_boundary_RK)
static void enqueue_rk(fdm_handle *h) {
    launch_stage(h, 1);
    launch_stage(h, 2);
    k_reset_lam<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>());
    launch_stage(h, 3);
}

// one solute iteration without AMR: step control, RK3, tt/residual/NaN
static void enqueue_solute_iteration(fdm_handle *h) {
    launch_step_control(h);
    enqueue_rk(h);
    launch_step_end(h);
}

static int prepare_buffers(fdm_handle *h) {
    const int64_t nb = nblk(h->NI, 256);
    FDM_CK(h, h->res_part.ensure((size_t)(nb > 0 ? nb : 1) * 8 * sizeof(double)));
    FDM_CK(h, h->gate_flag.ensure(gate_list_bytes(h)));
    return FDM_OK;
}

static void drop_graph(fdm_handle *h) {
    if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
    if (h->step_graph_g) cudaGraphExecDestroy(h->step_graph_g);
    h->step_graph = h->step_graph_g = nullptr;
    h->graph_version = -1;
}

// CUDA graph of one solute iteration (ghosts: followed by the j = 1 ghost
// refresh that solute does after an iteration without regrid); both are
// re-captured after every rebuild of the tables (upload / regrid), replayed
// otherwise.  A re-captured graph of the same shape (the usual case after a
// regrid: the same kernels with new sizes and table pointers) updates the
// executable graph in place, which costs far less than instantiating it.
static int step_graph(fdm_handle *h, cudaGraphExec_t *out, bool ghosts = false) {
    if (h->graph_version != h->table_version) {
        h->graph_stale[0] = h->graph_stale[1] = true;
        h->graph_version = h->table_version;
    }
    cudaGraphExec_t &slot = ghosts ? h->step_graph_g : h->step_graph;
    bool &stale = h->graph_stale[ghosts ? 1 : 0];
    if (slot && !stale) {
        *out = slot;
        return FDM_OK;
    }
    cudaGraph_t g = nullptr;
    FDM_CK(h, cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    enqueue_solute_iteration(h);
    if (ghosts) launch_ghosts(h, h->B[0].as<double4>(), 1);
    cudaError_t e = cudaStreamEndCapture(h->s, &g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    if (slot) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(slot, g, &info) == cudaSuccess) {
            cudaGraphDestroy(g);
            stale = false;
            *out = slot;
            return FDM_OK;
        }
        cudaGetLastError();   // another shape: instantiate it
        cudaGraphExecDestroy(slot);
        slot = nullptr;
    }
    e = cudaGraphInstantiate(&slot, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        slot = nullptr;
        return cuda_fail(h, e, "cudaGraphInstantiate");
    }
    stale = false;
    *out = slot;
    return FDM_OK;
}

static bool amr_due(const fdm_handle *h, int64_t it) {
    return h->p.iflag_amr && it >= h->p.nstep_adapt && h->p.pstep_adapt != 0 &&
           (it % h->p.pstep_adapt) == 1;
}

}  // namespace fdm

#define CHECK_H(h)                    \
    do {                              \
        if (!(h)) return FDM_ERR_ARG; \
    } while (0)
#define CHECK_LOADED(h)                                                            \
    do {                                                                           \
        if (!(h)->loaded) { (h)->err = "no leaf set uploaded"; return FDM_ERR_STATE; } \
    } while (0)
#define RC(x)                \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

extern "C" {

int fdm_create(const fdm_params *p, fdm_handle **out) {
    if (!p || !out) return FDM_ERR_ARG;
    *out = nullptr;
    if (!(p->h > 0.0) || !(p->x_factor > 0.0) || p->m < 7 || p->n < 7) return FDM_ERR_ARG;
    const int m = (int)((p->xmax - p->xmin) / (p->x_factor * p->h));
    const int n = (int)((p->ymax - p->ymin) / p->h);
    if (m != p->m || n != p->n) return FDM_ERR_ARG;
    if ((int64_t)p->m * p->n >= (1ll << 30)) return FDM_ERR_ARG;
    if (p->lvl_amr < 0 || p->lvl_amr > MAXLVL_TAB - 2) return FDM_ERR_ARG;
    if (p->flux_variant != 0 && p->flux_variant != 1) return FDM_ERR_UNSUPPORTED;
    // a strip: rows [row0, row0 + rows) of the n padded rows, at least three
    // owned rows between its two three-row margins; a side where the mesh is
    // cut is an exchange side, and only there
    const bool strip = p->window_rows != 0;
    if (strip) {
        if (p->window_row0 < 0 || p->window_rows < 9 || p->window_row0 + p->window_rows > p->n) return FDM_ERR_ARG;
        const bool cut_lo = p->window_row0 > 0, cut_hi = p->window_row0 + p->window_rows < p->n;
        if (cut_lo != (p->kind_ymbc == FDM_BC_EXCHANGE) || cut_hi != (p->kind_ypbc == FDM_BC_EXCHANGE))
            return FDM_ERR_ARG;
        if ((cut_lo || cut_hi) && (p->kind_ymbc == FDM_BC_PERIODIC || p->kind_ypbc == FDM_BC_PERIODIC))
            return FDM_ERR_UNSUPPORTED;   // the periodic image lies in another strip
    } else if (p->window_row0 != 0 || p->kind_ymbc == FDM_BC_EXCHANGE || p->kind_ypbc == FDM_BC_EXCHANGE) {
        return FDM_ERR_ARG;
    }
    if (p->kind_xmbc == FDM_BC_EXCHANGE || p->kind_xpbc == FDM_BC_EXCHANGE) return FDM_ERR_ARG;
    fdm_handle *h = new (std::nothrow) fdm_handle();
    if (!h) return FDM_ERR_NOMEM;
    h->p = *p;
    h->G.xmin = p->xmin; h->G.ymin = p->ymin; h->G.h = p->h; h->G.xf = p->x_factor;
    h->G.gama = p->gama; h->G.cv = p->cv; h->G.m = p->m;
    h->G.n = strip ? p->window_rows : p->n;
    h->G.row0 = strip ? p->window_row0 : 0;
    h->G.nglob = p->n;
    h->G.halo_lo = p->kind_ymbc == FDM_BC_EXCHANGE;
    h->G.halo_hi = p->kind_ypbc == FDM_BC_EXCHANGE;
    for (int l = 0; l < MAXLVL_TAB; ++l) {
        const double dy = p->h / (double)(1ll << l);
        const double dx = p->x_factor * dy;
        h->lt.dx[l] = dx;
        h->lt.dy[l] = dy;
        h->lt.cxa[l] = 4.0 / (3.0 * dx);
        h->lt.cxb[l] = 1.0 / (6.0 * dx);
        h->lt.cya[l] = 4.0 / 3.0 / dy;
        h->lt.cyb[l] = 1.0 / 6.0 / dy;
        h->lt.dxdy[l] = 0.0;
        h->lt.p15[l] = std::pow(dy, 1.5);
    }
    cudaError_t e = cudaGetDevice(&h->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&h->hs, sizeof(DevScalars));
    if (e == cudaSuccess) e = h->scal.ensure(sizeof(DevScalars));
    if (e == cudaSuccess) e = h->flag.ensure(8 * sizeof(int32_t));
    if (e != cudaSuccess) {
        fdm_destroy(h);
        return e == cudaErrorMemoryAllocation ? FDM_ERR_NOMEM : FDM_ERR_CUDA;
    }
    std::memset(h->hs, 0, sizeof(DevScalars));
    h->hs->tstep = p->tstep;
    h->hs->t_end = p->t_end;
    h->hs->done = 0;
    if (push_scalars(h)) {
        fdm_destroy(h);
        return FDM_ERR_CUDA;
    }
    *out = h;
    return FDM_OK;
}

void fdm_destroy(fdm_handle *h) {
    if (!h) return;
    if (h->s) cudaStreamSynchronize(h->s);
    drop_graph(h);
    DevBuf *bufs[] = {&h->lkey, &h->lslot, &h->slot_leaf, &h->lcx, &h->lcy, &h->lcross, &h->rfirst, &h->ist, &h->ilvl,
                      &h->ifxl, &h->ifyl, &h->uxl, &h->uyl, &h->rq_kind, &h->rq_m, &h->rq_mem, &h->rq_geo, &h->rq_node,
                      &h->gh_kind, &h->gh_a, &h->gh_b, &h->gh_flip, &h->gh_x, &h->gh_y, &h->B[0], &h->B[1],
                      &h->B[2], &h->Fx, &h->Fy, &h->Ut, &h->scal, &h->res_part, &h->cub_tmp, &h->flag,
                      &h->gate_params, &h->gate_flag, &h->ikey, &h->ival, &h->io};
    for (DevBuf *b : bufs) b->release();
    for (auto &t : h->tmp) t.release();
    for (cudaEvent_t e : h->amr_ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->gm4_ev)
        if (e) cudaEventDestroy(e);
    for (int b = 0; b < 2; ++b) {
        cudaEvent_t ev[4] = {h->in_ready[b], h->in_free[b], h->out_ready[b], h->out_free[b]};
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);
        h->in_stage[b].release();
        h->out_stage[b].release();
    }
    for (cudaStream_t cs : {h->cs, h->cs_out})
        if (cs) {
            cudaStreamSynchronize(cs);
            cudaStreamDestroy(cs);
        }
    if (h->hs) cudaFreeHost(h->hs);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
}

int fdm_last_error(const fdm_handle *h, char *buf, size_t n) {
    if (!h || !buf || n == 0) return FDM_ERR_ARG;
    size_t k = h->err.size() < n - 1 ? h->err.size() : n - 1;
    std::memcpy(buf, h->err.data(), k);
    buf[k] = 0;
    return FDM_OK;
}

int fdm_upload_leaves(fdm_handle *h, int64_t n, const uint64_t *keys, const double *prim) {
    Nvtx range("fdm_upload_leaves");
    CHECK_H(h);
    if (n <= 0 || !keys || !prim) return arg_fail(h, "empty leaf set");
    DevBuf dk, dp;
    FDM_CK(h, dk.ensure(n * 8));
    FDM_CK(h, dp.ensure(n * 32));
    FDM_CK(h, cudaMemcpyAsync(dk.p, keys, n * 8, cudaMemcpyHostToDevice, h->s));
    FDM_CK(h, cudaMemcpyAsync(dp.p, prim, n * 32, cudaMemcpyHostToDevice, h->s));
    int rc = build_tables(h, n, dk.as<uint64_t>(), dp.as<double>());
    cudaStreamSynchronize(h->s);
    dk.release();
    dp.release();
    if (rc) { h->loaded = false; return rc; }
    rc = prepare_buffers(h);
    if (!rc) rc = init_internal(h);
    if (rc) h->loaded = false;   // tables without their buffers: upload again
    return rc;
}

int64_t fdm_num_leaves(const fdm_handle *h) { return h && h->loaded ? h->NL : 0; }

int fdm_download_leaves(fdm_handle *h, int64_t cap, int64_t *n_out, uint64_t *keys, double *prim) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n_out) *n_out = h->NL;
    if (cap < h->NL) return arg_fail(h, "capacity below the leaf count");
    DevBuf &dp = h->io;
    FDM_CK(h, dp.ensure(h->NL * 32));
    if (keys) FDM_CK(h, cudaMemcpyAsync(keys, h->lkey.p, h->NL * 8, cudaMemcpyDeviceToHost, h->s));
    if (prim) {
        k_out<<<nblk(h->NL, 256), 256, 0, h->s>>>(h->NL, h->lslot.as<int32_t>(), h->B[0].as<double4>(),
                                                  dp.as<double>());
        FDM_CK(h, cudaMemcpyAsync(prim, dp.p, h->NL * 32, cudaMemcpyDeviceToHost, h->s));
    }
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

// Asynchronous value transfers (no reference counterpart): the copies run
// on a copy stream with double-buffered device staging, so the upload of the
// next step's input and the read-back of the last result overlap the steps
// in between.  Host buffers must be pinned and stay untouched until
// fdm_io_sync returns.
static int io_setup(fdm_handle *h) {
    if (h->cs) return FDM_OK;
    FDM_CK(h, cudaStreamCreateWithFlags(&h->cs, cudaStreamNonBlocking));
    FDM_CK(h, cudaStreamCreateWithFlags(&h->cs_out, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
        FDM_CK(h, cudaEventCreateWithFlags(&h->in_ready[b], cudaEventDisableTiming));
        FDM_CK(h, cudaEventCreateWithFlags(&h->in_free[b], cudaEventDisableTiming));
        FDM_CK(h, cudaEventCreateWithFlags(&h->out_ready[b], cudaEventDisableTiming));
        FDM_CK(h, cudaEventCreateWithFlags(&h->out_free[b], cudaEventDisableTiming));
    }
    return FDM_OK;
}

int fdm_set_values_async(fdm_handle *h, int64_t n, const double *prim) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n != h->NL || !prim) return arg_fail(h, "value count differs from the leaf count");
    RC(io_setup(h));
    const int b = h->in_b;
    h->in_b ^= 1;
    if (h->in_stage[b].bytes < (size_t)n * 32) {
        FDM_CK(h, cudaStreamSynchronize(h->s));   // the buffer may still be read
        FDM_CK(h, h->in_stage[b].ensure(n * 32));
    }
    FDM_CK(h, cudaStreamWaitEvent(h->cs, h->in_free[b], 0));
    FDM_CK(h, cudaMemcpyAsync(h->in_stage[b].p, prim, n * 32, cudaMemcpyHostToDevice, h->cs));
    FDM_CK(h, cudaEventRecord(h->in_ready[b], h->cs));
    FDM_CK(h, cudaStreamWaitEvent(h->s, h->in_ready[b], 0));
    k_in<<<nblk(n, 256), 256, 0, h->s>>>(n, h->lslot.as<int32_t>(), h->B[0].as<double4>(), h->in_stage[b].as<double>());
    if (h->NC > 0)
        for (int k = 1; k < 3; ++k)
            FDM_CK(h, cudaMemcpyAsync(h->B[k].as<double4>() + h->NI + h->NG, h->B[0].as<double4>() + h->NI + h->NG,
                                      h->NC * 32, cudaMemcpyDeviceToDevice, h->s));
    FDM_CK(h, cudaEventRecord(h->in_free[b], h->s));
    h->lam_fresh = false;
    return FDM_OK;
}

int fdm_download_values_async(fdm_handle *h, int64_t cap, double *prim) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NL || !prim) return arg_fail(h, "capacity below the leaf count");
    RC(io_setup(h));
    const int b = h->out_b;
    h->out_b ^= 1;
    if (h->out_stage[b].bytes < (size_t)h->NL * 32) {
        FDM_CK(h, cudaStreamSynchronize(h->cs_out));   // the buffer may still be copied out
        FDM_CK(h, h->out_stage[b].ensure(h->NL * 32));
    }
    FDM_CK(h, cudaStreamWaitEvent(h->s, h->out_free[b], 0));
    k_out<<<nblk(h->NL, 256), 256, 0, h->s>>>(h->NL, h->lslot.as<int32_t>(), h->B[0].as<double4>(),
                                              h->out_stage[b].as<double>());
    FDM_CK(h, cudaEventRecord(h->out_ready[b], h->s));
    FDM_CK(h, cudaStreamWaitEvent(h->cs_out, h->out_ready[b], 0));
    FDM_CK(h, cudaMemcpyAsync(prim, h->out_stage[b].p, h->NL * 32, cudaMemcpyDeviceToHost, h->cs_out));
    FDM_CK(h, cudaEventRecord(h->out_free[b], h->cs_out));
    return FDM_OK;
}

// the leaf keys (key order) into pinned host memory on the read-back
// stream, after the work queued so far; complete at fdm_io_sync
int fdm_download_keys_async(fdm_handle *h, int64_t cap, uint64_t *keys) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NL || !keys) return arg_fail(h, "capacity below the leaf count");
    RC(io_setup(h));
    DevBuf &st = h->key_stage[h->out_b];
    if (st.bytes < (size_t)h->NL * 8) {
        FDM_CK(h, cudaStreamSynchronize(h->cs_out));   // the buffer may still be copied out
        FDM_CK(h, st.ensure(h->NL * 8));
    }
    // the copy on the handle's stream keeps the keys of this point of the
    // run even if a regrid follows before the read-back lands
    FDM_CK(h, cudaStreamWaitEvent(h->s, h->out_free[h->out_b], 0));
    FDM_CK(h, cudaMemcpyAsync(st.p, h->lkey.p, h->NL * 8, cudaMemcpyDeviceToDevice, h->s));
    FDM_CK(h, cudaEventRecord(h->out_ready[h->out_b], h->s));
    FDM_CK(h, cudaStreamWaitEvent(h->cs_out, h->out_ready[h->out_b], 0));
    FDM_CK(h, cudaMemcpyAsync(keys, st.p, h->NL * 8, cudaMemcpyDeviceToHost, h->cs_out));
    FDM_CK(h, cudaEventRecord(h->out_free[h->out_b], h->cs_out));
    return FDM_OK;
}

// waits for the read-backs queued so far (the read-back stream only); the
// one call that another host thread may make while the handle is in use
int fdm_readback_wait(fdm_handle *h) {
    CHECK_H(h);
    if (h->cs_out && cudaStreamSynchronize(h->cs_out) != cudaSuccess) return FDM_ERR_CUDA;
    return FDM_OK;
}

int fdm_io_sync(fdm_handle *h) {
    CHECK_H(h);
    if (h->cs) FDM_CK(h, cudaStreamSynchronize(h->cs));
    if (h->cs_out) FDM_CK(h, cudaStreamSynchronize(h->cs_out));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

int fdm_set_values(fdm_handle *h, int64_t n, const double *prim) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n != h->NL || !prim) return arg_fail(h, "value count differs from the leaf count");
    DevBuf &dp = h->io;
    FDM_CK(h, dp.ensure(n * 32));
    FDM_CK(h, cudaMemcpyAsync(dp.p, prim, n * 32, cudaMemcpyHostToDevice, h->s));
    k_in<<<nblk(n, 256), 256, 0, h->s>>>(n, h->lslot.as<int32_t>(), h->B[0].as<double4>(), dp.as<double>());
    if (h->NC > 0)
        for (int b = 1; b < 3; ++b)
            FDM_CK(h, cudaMemcpyAsync(h->B[b].as<double4>() + h->NI + h->NG, h->B[0].as<double4>() + h->NI + h->NG,
                                      h->NC * 32, cudaMemcpyDeviceToDevice, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    h->lam_fresh = false;
    return FDM_OK;
}

int fdm_get_scalars(fdm_handle *h, double *lambda_x, double *lambda_y, double *tstep, double *tt, int64_t *it,
                    int32_t *l_max) {
    CHECK_H(h);
    RC(sync_scalars_from_device(h));
    if (lambda_x) *lambda_x = h->hs->lambda_x;
    if (lambda_y) *lambda_y = h->hs->lambda_y;
    if (tstep) *tstep = h->hs->tstep;
    if (tt) *tt = h->hs->tt;
    if (it) *it = h->hs->it;
    if (l_max) *l_max = h->l_max;
    return FDM_OK;
}

int fdm_set_scalars(fdm_handle *h, double lambda_x, double lambda_y, double tstep, double tt, int64_t it) {
    CHECK_H(h);
    RC(sync_scalars_from_device(h));
    h->hs->lambda_x = lambda_x;
    h->hs->lambda_y = lambda_y;
    h->hs->tstep = tstep;
    h->hs->tt = tt;
    h->hs->it = it;
    h->hs->t_end = h->p.t_end;
    h->hs->done = !(tt < h->p.t_end);
    h->hs->status = 0;
    return push_scalars(h);
}

int fdm_step_control(fdm_handle *h, double *tstep, double *lambda_x, double *lambda_y, int32_t *l_max) {
    CHECK_H(h);
    CHECK_LOADED(h);
    RC(ensure_lambda(h));
    launch_step_control(h);
    RC(sync_scalars_from_device(h));
    if (tstep) *tstep = h->hs->tstep;
    if (lambda_x) *lambda_x = h->hs->lambda_x;
    if (lambda_y) *lambda_y = h->hs->lambda_y;
    if (l_max) *l_max = h->l_max;
    return FDM_OK;
}

int fdm_time_advance_rk(fdm_handle *h, double tstep) {
    Nvtx range("fdm_time_advance_rk");
    CHECK_H(h);
    CHECK_LOADED(h);
    launch_set_tstep(h, tstep);
    enqueue_rk(h);
    h->lam_fresh = true;
    FDM_CK(h, cudaStreamSynchronize(h->s));
    FDM_CK(h, cudaGetLastError());
    return FDM_OK;
}

int fdm_get_rkn(fdm_handle *h) {
    // B0 holds Un for the whole step (stages never overwrite it before
    // stage 3), so getRKn needs no copy.
    CHECK_H(h);
    CHECK_LOADED(h);
    return FDM_OK;
}

// split API: stage krk reads buffer (krk-1) and writes Ut; update_rk blends
// into buffer krk % 3; body_boundary fills its ghosts.
int fdm_solution_cells(fdm_handle *h, int32_t krk) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (krk < 1 || krk > 3) return arg_fail(h, "krk must be 1..3");
    const double4 *cur = h->B[krk - 1].as<double4>();
    launch_requests(h, cur);
    launch_faces(h, cur, krk);
    launch_cells(h, cur, h->B[0].as<double4>(), h->Ut.as<double4>(), krk, 1);
    return split_done(h);
}
int fdm_update_rk(fdm_handle *h, int32_t krk) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (krk < 1 || krk > 3) return arg_fail(h, "krk must be 1..3");
    launch_blend(h, h->B[0].as<double4>(), h->B[krk % 3].as<double4>(), krk);
    h->cur_buf = krk % 3;
    h->lam_fresh = false;
    return split_done(h);
}
int fdm_body_boundary(fdm_handle *h, int32_t j) {
    CHECK_H(h);
    CHECK_LOADED(h);
    // ghosts of the buffer that holds the latest interior values
    launch_ghosts(h, h->B[h->cur_buf].as<double4>(), j);
    return split_done(h);
}

int fdm_residual(fdm_handle *h, double res_max[4], double res_rms[4]) {
    CHECK_H(h);
    RC(sync_scalars_from_device(h));
    for (int n = 0; n < 4; ++n) {
        if (res_max) res_max[n] = h->hs->res_max[n];
        if (res_rms) res_rms[n] = h->hs->res_rms[n];
    }
    return FDM_OK;
}

int fdm_solute_step(fdm_handle *h) {
    Nvtx range("fdm_solute_step");
    CHECK_H(h);
    CHECK_LOADED(h);
    RC(ensure_lambda(h));
    enqueue_solute_iteration(h);
    h->lam_fresh = true;
    RC(sync_scalars_from_device(h));
    FDM_CK(h, cudaGetLastError());
    if (h->hs->status == FDM_ERR_NAN) {
        h->err = "NaN in the residual RMS (the reference stops here)";
        return FDM_ERR_NAN;
    }
    if (amr_due(h, h->hs->it)) {
        RC(fdm_amr(h));
    }
    if (h->p.iflag_amr) {
        launch_ghosts(h, h->B[0].as<double4>(), 1);
        FDM_CK(h, cudaStreamSynchronize(h->s));
    }
    return FDM_OK;
}

// nsteps iterations of solute_step, run as chunks that end at the next
// regrid: the iterations of a chunk are replays of the step graph (with the
// ghost refresh after each, as solute_step does, when AMR is on) and the host
// reads the scalars once per chunk.  The device makes an iteration after
// t_end or after a NaN residual a no-op, so the steps counted are the
// device's own; after a NaN the ghost cells may have been refreshed once more
// than solute_step leaves them.
int fdm_solute(fdm_handle *h, int64_t nsteps, int64_t *steps_done) {
    Nvtx range("fdm_solute");
    CHECK_H(h);
    CHECK_LOADED(h);
    int64_t k = 0;
    int rc = FDM_OK;
    RC(sync_scalars_from_device(h));
    if (h->hs->status == FDM_ERR_NAN) {
        if (steps_done) *steps_done = 0;
        h->err = "NaN in the residual RMS (the reference stops here)";
        return FDM_ERR_NAN;
    }
    while (k < nsteps && h->hs->tt < h->p.t_end) {
        const int64_t it0 = h->hs->it;
        int64_t j = 1;
        while (k + j < nsteps && j < 64 && !amr_due(h, it0 + j)) ++j;   // at most 64 before a look at tt
        const bool regrid = amr_due(h, it0 + j);
        RC(ensure_lambda(h));
        cudaGraphExec_t gs = nullptr, gl = nullptr;   // iterations before the last, the last
        RC(step_graph(h, &gs, h->p.iflag_amr != 0));
        gl = gs;
        if (regrid) RC(step_graph(h, &gl, false));
        for (int64_t s = 0; s < j; ++s) FDM_CK(h, cudaGraphLaunch(s + 1 < j ? gs : gl, h->s));
        h->lam_fresh = true;
        RC(sync_scalars_from_device(h));
        FDM_CK(h, cudaGetLastError());
        const int64_t taken = h->hs->it - it0;
        k += taken;
        if (h->hs->status == FDM_ERR_NAN) {
            h->err = "NaN in the residual RMS (the reference stops here)";
            rc = FDM_ERR_NAN;
            break;
        }
        if (taken < j) break;   // t_end came inside the chunk
        if (regrid) {
            RC(fdm_amr(h));
            launch_ghosts(h, h->B[0].as<double4>(), 1);
            FDM_CK(h, cudaStreamSynchronize(h->s));
        }
    }
    if (steps_done) *steps_done = k;
    return rc;
}

// Device-only loop of solute iterations through the captured step graph:
// no host synchronisation and no regrid inside (the caller keeps the window
// between regrids).  Used for the timed windows of the benchmark.
int fdm_advance(fdm_handle *h, int64_t nsteps) {
    Nvtx range("fdm_advance");
    CHECK_H(h);
    CHECK_LOADED(h);
    RC(ensure_lambda(h));
    cudaGraphExec_t g = nullptr;
    RC(step_graph(h, &g));
    for (int64_t k = 0; k < nsteps; ++k) FDM_CK(h, cudaGraphLaunch(g, h->s));
    h->lam_fresh = true;
    return FDM_OK;
}

// nsteps solute iterations of two handles on the same leaf set in
// lockstep: `follow` takes the time step and the regrid decisions of
// `lead` (its lambda maxima before every step; at a regrid, the refine and
// coarsen flags of lead's indicators), so the two runs keep one leaf set and
// one time axis and differ only by their face fluxes (e.g. follow with the
// learned gate on, lead on the exact flux).  lead advances exactly as
// fdm_solute would advance it.
int fdm_solute_paired(fdm_handle *lead, fdm_handle *follow, int64_t nsteps, int64_t *steps_done) {
    Nvtx range("fdm_solute_paired");
    CHECK_H(lead);
    CHECK_H(follow);
    if (lead == follow || nsteps < 0) return FDM_ERR_ARG;
    CHECK_LOADED(lead);
    CHECK_LOADED(follow);
    if (lead->device != follow->device) { follow->err = "the two handles are on different devices"; return FDM_ERR_ARG; }
    int64_t k = 0;
    RC(sync_scalars_from_device(lead));
    RC(sync_scalars_from_device(follow));
    if (lead->hs->it != follow->hs->it || lead->hs->tt != follow->hs->tt || lead->NL != follow->NL) {
        follow->err = "paired handles must start at the same iteration, time and leaf count";
        return FDM_ERR_STATE;
    }
    int rc = FDM_OK;
    while (k < nsteps && lead->hs->tt < lead->p.t_end) {
        const bool regrid = amr_due(lead, lead->hs->it + 1);
        RC(ensure_lambda(lead));
        RC(ensure_lambda(follow));
        FDM_CK(follow, cudaStreamSynchronize(lead->s));
        k_take_lambda<<<1, 32, 0, follow->s>>>(lead->scal.as<DevScalars>(), follow->scal.as<DevScalars>());
        cudaGraphExec_t gl = nullptr, gf = nullptr;
        RC(step_graph(lead, &gl, lead->p.iflag_amr != 0 && !regrid));
        RC(step_graph(follow, &gf, follow->p.iflag_amr != 0 && !regrid));
        FDM_CK(lead, cudaGraphLaunch(gl, lead->s));
        FDM_CK(follow, cudaGraphLaunch(gf, follow->s));
        lead->lam_fresh = follow->lam_fresh = true;
        RC(sync_scalars_from_device(lead));
        RC(sync_scalars_from_device(follow));
        ++k;
        if (lead->hs->status == FDM_ERR_NAN || follow->hs->status == FDM_ERR_NAN) {
            (lead->hs->status == FDM_ERR_NAN ? lead : follow)->err = "NaN in the residual RMS (the reference stops here)";
            rc = FDM_ERR_NAN;
            break;
        }
        if (follow->hs->tt != lead->hs->tt || follow->hs->it != lead->hs->it) {
            follow->err = "the paired runs took different time steps";
            rc = FDM_ERR_STATE;
            break;
        }
        if (regrid) {
            rc = run_amr(follow, lead);
            if (!rc) rc = prepare_buffers(follow);
            if (rc) break;
            rc = fdm_amr(lead);
            if (rc) break;
            launch_ghosts(lead, lead->B[0].as<double4>(), 1);
            launch_ghosts(follow, follow->B[0].as<double4>(), 1);
            FDM_CK(lead, cudaStreamSynchronize(lead->s));
            FDM_CK(follow, cudaStreamSynchronize(follow->s));
        }
    }
    if (steps_done) *steps_done = k;
    return rc;
}

int fdm_amr(fdm_handle *h) {
    CHECK_H(h);
    CHECK_LOADED(h);
    int rc = run_amr(h);
    if (!rc) rc = prepare_buffers(h);
    return rc;
}

// Allocation-failure injection for tests: the next `after` device buffer
// allocations succeed, the one after fails with FDM_ERR_NOMEM (no cudaMalloc
// is made for it) and so do all later ones; after < 0 turns it off.
int fdm_debug_fail_alloc(int64_t after) {
    fdm::g_alloc_budget.store(after < 0 ? -1 : (long long)after);
    return FDM_OK;
}

int fdm_get_counters(fdm_handle *h, fdm_counters *c) {
    CHECK_H(h);
    if (!c) return FDM_ERR_ARG;
    std::memset(c, 0, sizeof(*c));
    c->n_leaves = h->NL;
    c->n_interior = h->NI;
    c->n_ghost = h->NG;
    c->n_wls_requests = h->NR - h->n_restrict;
    c->n_restrict_requests = h->n_restrict;
    c->n_faces_x = h->NI + h->nux;
    c->n_faces_y = h->NI + h->nuy;
    c->n_singular = h->n_singular;
    c->n_regrids = h->n_regrids;
    c->n_internal = h->NInt;
    c->n_gm1_iterations = h->gm1_iters;
    c->n_gm4_visits = h->gm4_visits;
    c->n_gm4_nonleaf = h->gm4_nonleaf;
    c->n_gm4_triggers = h->gm4_triggers;
    c->n_gm4_refines = h->gm4_refines;
    c->n_gm4_steps = h->gm4_steps;
    c->gm4_replay_us = (int64_t)(h->gm4_ms * 1e3);
    return FDM_OK;
}

int fdm_debug_stencil(fdm_handle *h, int64_t cap, double *out) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NI) return arg_fail(h, "capacity below the interior leaf count");
    launch_requests(h, h->B[0].as<double4>());
    DevBuf d;
    FDM_CK(h, d.ensure(h->NI * 8 * 32));
    k_stencil_out<<<nblk(h->NI, 128), 128, 0, h->s>>>(h->tables(), h->B[0].as<double4>(), d.as<double>());
    FDM_CK(h, cudaMemcpyAsync(out, d.p, h->NI * 8 * 32, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    d.release();
    return FDM_OK;
}

int fdm_debug_requests(fdm_handle *h, int64_t cap, int32_t *kind, uint64_t *node, double *xy, int32_t *m12,
                       uint64_t *mem) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NI) return arg_fail(h, "capacity below the interior leaf count");
    const int64_t ne = h->NI * 8;
    DevBuf d;
    Carve cv;
    cv.add(ne * 4); cv.add(ne * 8); cv.add(ne * 16); cv.add(ne * 8); cv.add(ne * 128);
    FDM_CK(h, d.ensure(cv.total));
    int32_t *dk = cv.at<int32_t>(d, 0);
    uint64_t *dn = cv.at<uint64_t>(d, 1);
    double *dxy = cv.at<double>(d, 2);
    int32_t *dm = cv.at<int32_t>(d, 3);
    uint64_t *dmem = cv.at<uint64_t>(d, 4);
    k_requests_out<<<nblk(ne, 128), 128, 0, h->s>>>(h->tables(), dk, dn, dxy, dm, dmem);
    FDM_CK(h, cudaMemcpyAsync(kind, dk, ne * 4, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(node, dn, ne * 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(xy, dxy, ne * 16, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(m12, dm, ne * 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(mem, dmem, ne * 128, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    d.release();
    return FDM_OK;
}

int fdm_debug_neighbors(fdm_handle *h, int64_t cap, uint64_t *out) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NL) return arg_fail(h, "capacity below the leaf count");
    DevBuf d;
    FDM_CK(h, d.ensure(h->NL * 8 * 8));
    k_neighbors_out<<<nblk(h->NL, 128), 128, 0, h->s>>>(h->tables(), h->G, d.as<uint64_t>());
    FDM_CK(h, cudaMemcpyAsync(out, d.p, h->NL * 64, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    d.release();
    return FDM_OK;
}

// ------------------------------------------------------ checkpoint/restart
int fdm_download_internal(fdm_handle *h, int64_t cap, int64_t *n_out, uint64_t *keys, double *vals) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n_out) *n_out = h->NInt;
    if (cap < h->NInt) return arg_fail(h, "capacity below the internal node count");
    if (h->NInt == 0) return FDM_OK;
    if (keys) FDM_CK(h, cudaMemcpyAsync(keys, h->ikey.p, h->NInt * 8, cudaMemcpyDeviceToHost, h->s));
    if (vals) FDM_CK(h, cudaMemcpyAsync(vals, h->ival.p, h->NInt * 32, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

int fdm_set_internal(fdm_handle *h, int64_t n, const uint64_t *keys, const double *vals) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n != h->NInt) return arg_fail(h, "internal node count differs from the leaf set's");
    if (n == 0) return FDM_OK;
    if (!keys || !vals) return arg_fail(h, "null keys or values");
    std::vector<uint64_t> cur((size_t)n);
    FDM_CK(h, cudaMemcpyAsync(cur.data(), h->ikey.p, n * 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    if (std::memcmp(cur.data(), keys, (size_t)n * 8) != 0)
        return arg_fail(h, "internal node keys differ from the leaf set's");
    FDM_CK(h, cudaMemcpyAsync(h->ival.p, vals, n * 32, cudaMemcpyHostToDevice, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

// ------------------------------------------------------ strips of one mesh
int fdm_leaf_slots(fdm_handle *h, int64_t cap, int32_t *slot) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (cap < h->NL || !slot) return arg_fail(h, "capacity below the leaf count");
    FDM_CK(h, cudaMemcpyAsync(slot, h->lslot.p, h->NL * sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

static int pack_common(fdm_handle *h, int64_t n, const int32_t *slots, const double *buf, bool unpack) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (n < 0 || (n > 0 && (!slots || !buf))) return arg_fail(h, "bad slot list");
    if (n == 0) return FDM_OK;
    // flag word 6: a slot outside the leaf slots (sticky in asynchronous
    // mode, where fdm_step_control_global reports it)
    int32_t *bad = h->flag.as<int32_t>() + 6;
    if (!h->split_async) FDM_CK(h, cudaMemsetAsync(bad, 0, sizeof(int32_t), h->s));
    const int64_t ns = h->NI + h->NG + h->NC;
    double4 *B = h->B[h->cur_buf].as<double4>();
    if (unpack)
        k_unpack_slots<<<nblk(n, 256), 256, 0, h->s>>>(n, slots, ns, B, buf, bad);
    else
        k_pack_slots<<<nblk(n, 256), 256, 0, h->s>>>(n, slots, ns, B, const_cast<double *>(buf), bad);
    FDM_CK(h, cudaGetLastError());
    if (h->split_async) return FDM_OK;
    int32_t hb = 0;
    FDM_CK(h, cudaMemcpyAsync(&hb, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    if (hb) return arg_fail(h, "a slot is outside the leaf slots");
    return FDM_OK;
}

int fdm_set_async(fdm_handle *h, int32_t on) {
    CHECK_H(h);
    CHECK_LOADED(h);
    FDM_CK(h, cudaStreamSynchronize(h->s));
    FDM_CK(h, cudaMemsetAsync(h->flag.as<int32_t>() + 6, 0, sizeof(int32_t), h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    h->split_async = on != 0;
    return FDM_OK;
}
int fdm_pack_slots(fdm_handle *h, int64_t n, const int32_t *slots, double *buf) {
    return pack_common(h, n, slots, buf, false);
}
int fdm_unpack_slots(fdm_handle *h, int64_t n, const int32_t *slots, const double *buf) {
    return pack_common(h, n, slots, buf, true);
}

int fdm_step_control_global(fdm_handle *h, double lambda_x, double lambda_y, int32_t l_max, double *tstep) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (l_max < 0 || l_max > FDM_LMAX) return arg_fail(h, "l_max out of range");
    if (!(lambda_x >= 0.0) || !(lambda_y >= 0.0)) return arg_fail(h, "lambda must be >= 0");
    k_set_global_lambda<<<1, 32, 0, h->s>>>(h->scal.as<DevScalars>(), lambda_x, lambda_y, l_max);
    h->l_max = l_max;
    h->lam_fresh = true;
    launch_step_control(h);
    RC(sync_scalars_from_device(h));
    FDM_CK(h, cudaGetLastError());
    if (h->split_async) {   // sticky halo-slot error of the previous step's copies
        int32_t hb = 0;
        FDM_CK(h, cudaMemcpy(&hb, h->flag.as<int32_t>() + 6, sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (hb) return arg_fail(h, "a halo copy named a slot outside the leaf slots");
    }
    if (tstep) *tstep = h->hs->tstep;
    return FDM_OK;
}

int fdm_device_state(fdm_handle *h, void **stream, double **prim_dev, int64_t *n) {
    CHECK_H(h);
    CHECK_LOADED(h);
    if (stream) *stream = (void *)h->s;
    if (prim_dev) *prim_dev = h->B[0].as<double>();
    if (n) *n = h->NS;
    return FDM_OK;
}

}  // extern "C"

namespace fdm {

// hooks of the batched path (batch.cu): the same host-side bookkeeping as
// fdm_solute_step around steps that the batch kernel takes
int member_ready(fdm_handle *h) {
    if (!h->loaded) { h->err = "no leaf set uploaded"; return FDM_ERR_STATE; }
    return ensure_lambda(h);
}
void member_stepped(fdm_handle *h) {
    h->lam_fresh = true;
    if (h->gate_on) h->gate_stage1_valid = true;
}
bool member_amr_due(const fdm_handle *h, int64_t it) { return amr_due(h, it); }
// One solute iteration of member h on its own stream, through its step
// graph: followed by the j = 1 ghost refresh unless a regrid comes next
// (member_regrid refreshes after it), as fdm_solute does.
int member_launch_step(fdm_handle *h, bool regrid_next) {
    RC(ensure_lambda(h));
    cudaGraphExec_t g = nullptr;
    RC(step_graph(h, &g, h->p.iflag_amr != 0 && !regrid_next));
    FDM_CK(h, cudaGraphLaunch(g, h->s));
    h->lam_fresh = true;
    return FDM_OK;
}
int member_regrid(fdm_handle *h) {
    int rc = fdm_amr(h);
    if (rc) return rc;
    if (h->p.iflag_amr) {
        launch_ghosts(h, h->B[0].as<double4>(), 1);
        FDM_CK(h, cudaStreamSynchronize(h->s));
    }
    return FDM_OK;
}

}  // namespace fdm
