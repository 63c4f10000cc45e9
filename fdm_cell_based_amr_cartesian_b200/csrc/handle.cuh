// handle.cuh — host-side state of one libfdm handle.
#pragma once
#include <atomic>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "fdm_common.cuh"

namespace fdm {

// A named NVTX range over a scope (profilers show the library's phases;
// without a tool attached a push/pop costs a pointer test).
struct Nvtx {
    explicit Nvtx(const char *name) { nvtxRangePushA(name); }
    ~Nvtx() { nvtxRangePop(); }
    Nvtx(const Nvtx &) = delete;
    Nvtx &operator=(const Nvtx &) = delete;
};


// Allocation-failure injection (fdm_debug_fail_alloc): the number of device
// buffer allocations that still succeed before DevBuf::ensure reports
// cudaErrorMemoryAllocation without calling cudaMalloc; negative: off.
inline std::atomic<long long> g_alloc_budget{-1};
inline bool alloc_refused() {
    long long b = g_alloc_budget.load();
    while (b > 0 && !g_alloc_budget.compare_exchange_weak(b, b - 1)) {}
    return b == 0;
}

// Device buffer that only grows; freed with the handle.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    // At least nbytes; a buffer that has to grow takes 25 % + 1 MiB more, and
    // at least twice what it had, so that a mesh growing by a few cells per
    // regrid does not reallocate (a cudaFree synchronises the device) at
    // every regrid, and one growing several-fold (the first regrids of a run
    // from its background mesh) reallocates a few times, not a dozen.
    cudaError_t ensure(size_t nbytes) {
        if (nbytes <= bytes && p) return cudaSuccess;
        const size_t had = p ? bytes : 0;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t nb = nbytes ? nbytes : 16;
        if (nbytes > 0) nb += nbytes / 4 + (1u << 20);
        if (nb < 2 * had) nb = 2 * had;
        if (alloc_refused()) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&p, nb);
        if (e != cudaSuccess && nb > nbytes) {   // no room for headroom
            cudaGetLastError();
            e = cudaMalloc(&p, nb = nbytes);
        }
        if (e == cudaSuccess) bytes = nb;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return (T *)p; }
};

// Carves several arrays out of one scratch buffer: offsets and the total
// size come from the same list, 256-byte aligned.
struct Carve {
    size_t off[16];
    size_t total = 0;
    int n = 0;
    size_t add(size_t bytes) {
        total = (total + 255) & ~size_t(255);
        off[n++] = total;
        total += bytes;
        return off[n - 1];
    }
    template <class T> T *at(const DevBuf &b, int i) const { return (T *)((char *)b.p + off[i]); }
};

}  // namespace fdm

struct fdm_handle {
    fdm_params p{};
    fdm::Geometry G{};
    fdm::LevelTab lt{};
    int device = 0;
    cudaStream_t s = nullptr;
    std::string err;

    // leaf set sizes
    int64_t NL = 0, NI = 0, NG = 0, NC = 0, NR = 0, NS = 0, nux = 0, nuy = 0;
    int32_t l_max = 0;
    bool loaded = false;
    bool lam_fresh = false;
    int cur_buf = 0;         // split API: buffer holding the latest interior values
    bool split_async = false;  // split API and halo copies return after enqueuing
    int face_variant = 0;    // 0: four lanes per face, 1: one thread per face
    int64_t n_singular = 0, n_regrids = 0, n_restrict = 0, n_ghost_restrict = 0;

    // tables
    fdm::DevBuf lkey, lslot, slot_leaf, lcx, lcy, lcross, rfirst;
    fdm::DevBuf ist, ilvl, ifxl, ifyl, uxl, uyl;
    fdm::DevBuf rq_kind, rq_m, rq_mem, rq_geo, rq_node, rq_rlist;
    fdm::DevBuf gh_kind, gh_a, gh_b, gh_flip, gh_x, gh_y;
    // state: three slot arrays (step start / stage 1 / stage 2)
    fdm::DevBuf B[3];
    fdm::DevBuf Fx, Fy, Ut;
    fdm::DevBuf scal;        // DevScalars
    fdm::DevBuf res_part;    // per-block residual partials
    // scratch for table building
    fdm::DevBuf tmp[8];
    fdm::DevBuf cub_tmp;
    fdm::DevBuf flag;        // device error flags (int32[8])
    fdm::DevScalars *hs = nullptr;   // pinned host mirror of the scalars

    // internal nodes of the tree and their values (the reference keeps a
    // stale U in every refined node; gridmodify4 can copy it back)
    fdm::DevBuf ikey, ival;
    int64_t NInt = 0;
    fdm::DevBuf amr[26];     // regrid scratch: [0..5] node sets, [6..19] work arrays, [20, 21] new leaves,
                             // [22] per-cell index of the node set, [23..25] the new nodes of a gridmodify4 pass
    int64_t gm1_iters = 0, gm4_visits = 0, gm4_nonleaf = 0, gm4_triggers = 0, gm4_refines = 0, gm4_steps = 0;
    // device-timeline phases of the last regrid (events recorded on the stream)
    static constexpr int AMR_PHASES = 5;
    cudaEvent_t amr_ev[AMR_PHASES + 1] = {};
    cudaEvent_t gm4_ev[2] = {};   // around the gridmodify4 replay kernel
    double gm4_ms = 0.0;          // its device time, summed over all passes
    double amr_phase_ms[AMR_PHASES] = {};
    double amr_phase_total_ms[AMR_PHASES] = {};   // summed over all regrids

    // learned gate of the face flux
    fdm::DevBuf io;   // staging of fdm_set_values / fdm_download_leaves (grows, kept)
    fdm::DevBuf diag; // per-leaf terms and sums of fdm_output_error
    fdm::DevBuf key_stage[2];   // staging of fdm_download_keys_async
    // asynchronous value transfers: a copy stream each way (uploads, read-
    // backs), two staging buffers each way, and the events that order them
    // with the compute stream
    cudaStream_t cs = nullptr, cs_out = nullptr;
    fdm::DevBuf in_stage[2], out_stage[2];
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
    int in_b = 0, out_b = 0;
    fdm::DevBuf gate_params, gate_flag;   // gate_flag: per-stage hard-face lists
    float gate_logit_thr = 0.f;
    float gate_jump_thr = -1.f;   // >= 0: the plain jump rule instead of the network
    bool gate_on = false;
    bool gate_stage1_valid = false;   // stage-1 decisions exist for the current tables

    // CUDA graph of one RK3 step (captured lazily, dropped at regrid)
    cudaGraphExec_t step_graph = nullptr;     // one solute iteration
    cudaGraphExec_t step_graph_g = nullptr;   // the same followed by the j = 1 ghost refresh
    int64_t graph_version = -1;               // table_version the slots were last checked against
    bool graph_stale[2] = {true, true};       // step_graph / step_graph_g need a re-capture
    int64_t table_version = 0;

    fdm::Tables tables() const {
        fdm::Tables T{};
        T.NL = NL; T.NI = NI; T.NG = NG; T.NC = NC; T.NR = NR; T.NS = NS;
        T.lkey = lkey.as<uint64_t>();
        T.lslot = lslot.as<int32_t>();
        T.slot_leaf = slot_leaf.as<int32_t>();
        T.lcx = lcx.as<double>();
        T.lcy = lcy.as<double>();
        T.rfirst = rfirst.as<int32_t>();
        T.nroots = (int64_t)G.m * G.n;
        T.ist = ist.as<int32_t>();
        T.ilvl = ilvl.as<uint8_t>();
        T.ifxl = ifxl.as<int32_t>();
        T.ifyl = ifyl.as<int32_t>();
        T.uxl = uxl.as<int32_t>();
        T.uyl = uyl.as<int32_t>();
        T.nux = nux; T.nuy = nuy;
        T.rq_kind = rq_kind.as<int32_t>();
        T.rq_rlist = rq_rlist.as<int32_t>();
        T.NRR = n_restrict;
        T.rq_m = rq_m.as<int32_t>();
        T.rq_mem = rq_mem.as<int32_t>();
        T.rq_geo = rq_geo.as<double>();
        T.rq_node = rq_node.as<uint64_t>();
        T.gh_kind = gh_kind.as<int32_t>();
        T.gh_a = gh_a.as<int32_t>();
        T.gh_b = gh_b.as<int32_t>();
        T.gh_flip = gh_flip.as<int32_t>();
        T.gh_x = gh_x.as<double>();
        T.gh_y = gh_y.as<double>();
        return T;
    }
};

namespace fdm {

// error helpers: record a message in the handle and return a status
inline int cuda_fail(fdm_handle *h, cudaError_t e, const char *what) {
    char buf[256];
    snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    h->err = buf;
    return e == cudaErrorMemoryAllocation ? FDM_ERR_NOMEM : FDM_ERR_CUDA;
}
#define FDM_CK(h, call)                                        \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return fdm::cuda_fail(h, e_, #call); \
    } while (0)

inline int arg_fail(fdm_handle *h, const char *msg) {
    h->err = msg;
    return FDM_ERR_ARG;
}

// table construction (build.cu)
// key_bits: the low bits of the keys that the key sort orders (64 for keys
// from a caller, root_bits(h) + 34 for keys the device made itself)
// key_bits: the low bits the sort looks at; 0: the keys are already sorted
// (the regrid emits them in key order), so they are only copied
int build_tables(fdm_handle *h, int64_t n, const uint64_t *keys_dev, const double *prim_dev, int key_bits = 64);
// bits of the largest background-cell (root) index m*n - 1: a leaf key
// (root << 34 | path << 4 | lvl) made on the device has no bit set at or
// above 34 + root_bits, so radix sorts of such keys stop there
inline int root_bits(const fdm_handle *h) {
    const uint64_t top = (uint64_t)h->p.m * (uint64_t)h->p.n;
    int b = 1;
    while (b < 30 && (1ull << b) < top) ++b;
    return b;
}
// per-stage pipeline (stage.cu)
void launch_requests(fdm_handle *h, const double4 *cur);
void launch_faces(fdm_handle *h, const double4 *cur, int krk);
void launch_cells(fdm_handle *h, const double4 *cur, const double4 *un, double4 *next, int krk,
                  int mode);
void launch_ghosts(fdm_handle *h, double4 *next, int j);
void launch_blend(fdm_handle *h, const double4 *un, double4 *cur, int krk);
void launch_lambda(fdm_handle *h, const double4 *cur);
// batched path (batch.cu) <-> single-mesh bookkeeping (libfdm.cu)
int member_ready(fdm_handle *h);
void member_stepped(fdm_handle *h);
bool member_amr_due(const fdm_handle *h, int64_t it);
int member_regrid(fdm_handle *h);
int member_launch_step(fdm_handle *h, bool regrid_next);
void launch_step_control(fdm_handle *h);
void launch_step_end(fdm_handle *h);
void launch_set_tstep(fdm_handle *h, double tstep);
void launch_res_finalize(fdm_handle *h);
int launch_stage(fdm_handle *h, int krk);
void launch_gated_faces(fdm_handle *h, const double4 *cur, int krk);
// flux_variant 1 (fast_flux.cu)
void launch_faces_fast(fdm_handle *h, const double4 *cur);
void launch_faces_list_fast(fdm_handle *h, const double4 *cur, const int32_t *hx, const int32_t *hy,
                            const uint32_t *cnt, int lx, int ly);
size_t gate_list_bytes(const fdm_handle *h);
// AMR (amr.cu)
int run_amr(fdm_handle *h, fdm_handle *lead = nullptr);
int init_internal(fdm_handle *h);

}  // namespace fdm
