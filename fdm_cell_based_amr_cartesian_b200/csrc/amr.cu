// amr.cu — device regrid (src/solution.F90:408-589, src/mesh.F90:199-408).
#include <cub/cub.cuh>

#include "handle.cuh"
#include "ordered_sum.cuh"
#include "topo.cuh"

namespace fdm {

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

void launch_requests(fdm_handle *h, const double4 *cur);

// Urot / Udiv / dux (src/solution.F90:558-589) on the stencil values
// Tip, Tim, Tjp, Tjm of every interior leaf.
__global__ void k_rot_div(Tables T, LevelTab LT, const double4 *__restrict__ B, double *rot, double *div,
                          uint64_t *dfs_key, int32_t *idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int lvl = T.ilvl[i];
    const int32_t *s = T.ist + i * 8;
    const double4 ip = B[s[0]], im = B[s[1]], jp = B[s[2]], jm = B[s[3]];
    const double dy = LT.dy[lvl], dx = LT.dx[lvl], p15 = LT.p15[lvl];
    const double vx = (ip.z - im.z) / (2.0 * dx);
    const double uy = (jp.y - jm.y) / (2.0 * dy);
    rot[i] = fabs(vx - uy) * p15;
    const double ux = (ip.x - im.x) / (2.0 * dx);
    const double vy = (jp.x - jm.x) / (2.0 * dy);
    div[i] = (fabs(ux) + fabs(vy)) * p15;
    // traversal order of solute_div_rot: roots row-major, sons 1,2,3,4
    const uint64_t key = T.lkey[T.slot_leaf[i]];
    const uint64_t path = key_pos(key) & ((1ull << 30) - 1ull);
    dfs_key[i] = ((key >> 34) << 30) | (path ^ ((path & 0x2AAAAAAAull) >> 1));
    idx[i] = (int32_t)i;
}

// Srot = Srot + rot**2 ... in traversal order: one thread, the sum is a
// sequence of roundings that no parallel order reproduces
// squares in traversal order (the products are rounded exactly as in the
// sequential loop: no FMA in this build)
__global__ void k_ordered_squares(int64_t NI, const int32_t *__restrict__ order, const double *__restrict__ rot,
                                  const double *__restrict__ div, double2 *__restrict__ sq) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NI) return;
    const int32_t i = order[k];
    sq[k] = make_double2(rot[i] * rot[i], div[i] * div[i]);
}

// Srot, Sdiv: left-to-right sums in traversal order, as the reference's
// recursive loop forms them (src/solution.F90:430-457), bit for bit, one
// block each (ordered_sum.cuh); launched with 2 blocks
__global__ void __launch_bounds__(OSUM_NT) k_ordered_sums(int64_t NI, const double2 *__restrict__ sq, double *out) {
    __shared__ OSumShared sh;
    const double *x = reinterpret_cast<const double *>(sq) + blockIdx.x;
    const double v = ordered_sum_block<OSUM_NT, OSUM_EPT>([&](int64_t e) { return x[2 * e]; }, NI, sh);
    if (threadIdx.x == 0) {
        out[blockIdx.x] = v;
        if (blockIdx.x == 0) out[2] = (double)NI;
    }
}

// rot/div of the current state into rot/div buffers; ordered sums to out3
static int compute_rot_div(fdm_handle *h, double *rot, double *div, double *out3) {
    Nvtx range("fdm regrid: indicators");
    const int64_t NI = h->NI;
    launch_requests(h, h->B[0].as<double4>());
    Carve cv;
    cv.add(NI * 8); cv.add(NI * 8); cv.add(NI * 4); cv.add(NI * 4); cv.add(NI * 16);
    FDM_CK(h, h->tmp[0].ensure(cv.total));
    uint64_t *k0 = cv.at<uint64_t>(h->tmp[0], 0), *k1 = cv.at<uint64_t>(h->tmp[0], 1);
    int32_t *i0 = cv.at<int32_t>(h->tmp[0], 2), *i1 = cv.at<int32_t>(h->tmp[0], 3);
    double2 *sq = cv.at<double2>(h->tmp[0], 4);
    k_rot_div<<<nblk(NI, 256), 256, 0, h->s>>>(h->tables(), h->lt, h->B[0].as<double4>(), rot, div, k0, i0);
    size_t bytes = 0;
    const int kb = 30 + root_bits(h);   // dfs keys: root << 30 | path
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0, k1, i0, i1, (int)NI, 0, kb, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(h->cub_tmp.p, bytes, k0, k1, i0, i1, (int)NI, 0, kb, h->s));
    k_ordered_squares<<<nblk(NI, 256), 256, 0, h->s>>>(NI, i1, rot, div, sq);
    k_ordered_sums<<<2, OSUM_NT, 0, h->s>>>(NI, sq, out3);
    return FDM_OK;
}

// ===================================================================
// Regrid.  The tree is handled as a node set: every leaf and every internal
// node, sorted by key, each with a value.  Internal nodes carry the value
// the reference leaves in a refined cell (its U when it was refined, or the
// interpA mean when it was coarsened), because gridmodify4 can copy it back
// into new leaves (Refine_cell of a non-leaf, src/mesh.F90:389-392).
// ===================================================================

struct NodeSet {
    int64_t n = 0;
    uint64_t *key = nullptr;
    uint8_t *leaf = nullptr;
    double4 *val = nullptr;
    const int32_t *rf = nullptr;   // per-cell index of key (index_set), or null
    int64_t nroots = 0;
};

enum { D_NONE = 0, D_REFINE = 1, D_COARSEN = 2 };
enum { PF_LEAF = 1, PF_DELETED = 2, PF_VISITED = 4 };

__device__ __forceinline__ int64_t find_key(const uint64_t *__restrict__ keys, int64_t n, uint64_t k) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const uint64_t v = keys[mid];
        if (v < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && keys[lo] == k) ? lo : -1;
}

// find_key within the nodes of k's background cell when the set is indexed
// (every cell holds at least its root node, and its nodes are contiguous)
__device__ __forceinline__ int64_t find_key_set(const NodeSet &A, uint64_t k) {
    const int64_t r = (int64_t)(k >> 34);
    if (!A.rf || r >= A.nroots) return find_key(A.key, A.n, k);
    int64_t lo = __ldg(A.rf + r), hi = __ldg(A.rf + r + 1);
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const uint64_t v = A.key[mid];
        if (v < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < A.n && A.key[lo] == k) ? lo : -1;
}

// find_key on the leaf table, within k's background cell (T.rfirst)
__device__ __forceinline__ int64_t find_key_t(const Tables &T, uint64_t k) {
    const int64_t r = (int64_t)(k >> 34);
    if (!T.rfirst || r >= T.nroots) return find_key_t(T, k);
    int64_t lo = __ldg(T.rfirst + r), hi = __ldg(T.rfirst + r + 1);
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldg(T.lkey + mid) < k) lo = mid + 1;
        else hi = mid;
    }
    return (lo < T.NL && __ldg(T.lkey + lo) == k) ? lo : -1;
}

// The helpers below work on the interleaved path bits directly.  Level j's
// digit (x bit | y bit << 1) sits at key bit 4 + 2 (LMAX - j); the x bits of
// the path occupy the even path positions and the y bits the odd ones.
constexpr uint64_t KEY_PATH_X = 0x15555555ull << 4;   // x bits of the path
constexpr uint64_t KEY_PATH_Y = 0x2AAAAAAAull << 4;   // y bits of the path
constexpr uint64_t KEY_PATH = (KEY_PATH_X | KEY_PATH_Y);
FDM_HD int key_digit_shift(int lvl) { return 4 + 2 * (LMAX - lvl); }

FDM_HD uint64_t parent_key(uint64_t k) {
    const int lvl = (int)(k & 15u);
    return (k & ~(3ull << key_digit_shift(lvl))) - 1u;
}
FDM_HD uint64_t child_key(uint64_t k, int q) {
    const int lvl = (int)(k & 15u);
    return (k | ((uint64_t)q << key_digit_shift(lvl + 1))) + 1u;
}
// The ancestor of key k at level la (0 <= la <= k's level): the path digits
// below level la cleared
FDM_HD uint64_t ancestor_key(uint64_t k, int la) {
    const uint64_t below = ((1ull << (2 * (LMAX - la))) - 1ull) << 4;
    return (k & ~below & ~15ull) | (uint64_t)la;
}
// Row and column of a background cell: q = root / m from a float reciprocal
// (root < 2^24, so the estimate is off by at most one) and one correction
FDM_HD void root_row_col(uint32_t root, uint32_t m, uint32_t &row, uint32_t &col) {
    uint32_t q = (uint32_t)((float)root * (1.0f / (float)m));
    int64_t r = (int64_t)root - (int64_t)q * m;
    q = r < 0 ? q - 1u : (r >= (int64_t)m ? q + 1u : q);
    r = r < 0 ? r + m : (r >= (int64_t)m ? r - m : r);
    row = q;
    col = (uint32_t)r;
}
// same-level neighbour node key across a face; false across the grid edge.
// A step along x (y) is a dilated increment or decrement of the x (y) bits
// at the node's level; a carry out of the path (or a borrow) moves to the
// next root.  Written without branches: the lanes of a warp step in
// different directions.
FDM_HD bool shift_key(const Geometry &G, uint64_t k, int dir, uint64_t &out) {
    const int lvl = (int)(k & 15u);
    const uint64_t unit = 1ull << key_digit_shift(lvl);
    const bool alongx = dir == DIR_RIGHT || dir == DIR_LEFT;
    const bool inc = dir == DIR_RIGHT || dir == DIR_UP;
    const uint64_t mask = alongx ? KEY_PATH_X : KEY_PATH_Y;
    const uint64_t u = alongx ? unit : unit << 1;
    const uint64_t bits = k & mask;
    // carries skip the other coordinate's bits; a borrow from zero leaves all
    // ones down to the node's level, the first node of the next root back
    const uint64_t path = inc ? (((bits | ~mask) + u) & mask) : ((bits - u) & mask);
    const bool wrap = inc ? (((bits | ~mask | (u - 1)) & KEY_PATH) == KEY_PATH) : bits == 0;
    const uint32_t root = (uint32_t)(k >> 34);
    const uint32_t m = (uint32_t)G.m;
    uint32_t row, col;
    root_row_col(root, m, row, col);
    const uint32_t rc = alongx ? col : row, lim = alongx ? m : (uint32_t)G.n;
    const bool edge = inc ? rc + 1u >= lim : rc == 0u;
    const uint32_t step = alongx ? 1u : m;
    const uint32_t nroot = wrap ? (inc ? root + step : root - step) : root;
    out = ((uint64_t)nroot << 34) | (k & ~mask & ((1ull << 34) - 1ull)) | path;
    return !(wrap && edge);
}
// traversal rank of gridmodify4 / solute_div_rot (sons 1,2,3,4): Morton path
// with the digits of son3 and son4 swapped
FDM_HD uint64_t dfs_rank(uint64_t k) {
    const uint64_t path = key_pos(k) & ((1ull << 30) - 1ull);
    return ((k >> 34) << 30) | (path ^ ((path & 0x2AAAAAAAull) >> 1));
}
// Visit order of gridmodify4's traversal (sons 1,2,3,4 of every node): the
// traversal rank of the node's position, then its level, so a node comes
// before its first son, which starts at the same position.  The node's key
// is recovered from it.  Below 2^53 for up to 2^19 background cells.
FDM_HD uint64_t visit_rank(uint64_t k) { return (dfs_rank(k) << 4) | (k & 15u); }
FDM_HD uint64_t key_of_visit_rank(uint64_t r) {
    const uint64_t pr = r >> 4;
    const uint64_t path = pr & ((1ull << 30) - 1ull);
    return ((pr >> 30) << 34) | ((path ^ ((path & 0x2AAAAAAAull) >> 1)) << 4) | (r & 15u);
}
// post-order rank of gridmodify1 (a node after all of its descendants):
// 3 bits per level, sons 1,2,3,4 -> 0,1,2,3 and 4 below the node's level
FDM_HD uint64_t post_rank(uint64_t k) {
    const Node n = node_of_key(k);
    const uint64_t path = key_pos(k) & ((1ull << 30) - 1ull);
    uint64_t r = 0;
    for (int l = 1; l <= LMAX; ++l) {
        uint64_t dgt = 4;
        if (l <= n.lvl) {
            const uint64_t q = (path >> (2 * (LMAX - l))) & 3u;
            dgt = q ^ (q >> 1);
        }
        r = (r << 3) | dgt;
    }
    return ((uint64_t)n.root << 45) | r;
}

__device__ __forceinline__ double4 mean4(const double4 &c0, const double4 &c1, const double4 &c2, const double4 &c3) {
    // interpA: 0.25*(son1 + son2 + son3 + son4) with son3 = q3, son4 = q2
    double4 v;
    v.x = 0.25 * (c0.x + c1.x + c3.x + c2.x);
    v.y = 0.25 * (c0.y + c1.y + c3.y + c2.y);
    v.z = 0.25 * (c0.z + c1.z + c3.z + c2.z);
    v.w = 0.25 * (c0.w + c1.w + c3.w + c2.w);
    return v;
}

// ---------------------------------------------------- internal node values
__global__ void k_anc_count(int64_t NL, const uint64_t *lkey, int32_t *cnt) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < NL) cnt[k] = (int32_t)(lkey[k] & 15u);
}
__global__ void k_anc_emit(int64_t NL, const uint64_t *lkey, const int32_t *off, uint64_t *out) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    uint64_t a = lkey[k];
    const int l = (int)(a & 15u);
    for (int j = 0; j < l; ++j) {
        a = parent_key(a);
        out[off[k] + j] = a;
    }
}
// interpA of internal nodes at one level from their children (leaves or
// deeper internal nodes, already done)
__global__ void k_internal_vals(int64_t NInt, const uint64_t *ikey, double4 *ival, int lvl, const uint64_t *lkey,
                                int64_t NL, const int32_t *lslot, const double4 *B0) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= NInt) return;
    const uint64_t k = ikey[i];
    if ((int)(k & 15u) != lvl) return;
    double4 c[4];
    for (int q = 0; q < 4; ++q) {
        const uint64_t ck = child_key(k, q);
        const int64_t li = find_key(lkey, NL, ck);
        if (li >= 0) c[q] = B0[lslot[li]];
        else {
            const int64_t ii = find_key(ikey, NInt, ck);
            c[q] = ii >= 0 ? ival[ii] : make_double4(0, 0, 0, 0);
        }
    }
    ival[i] = mean4(c[0], c[1], c[2], c[3]);
}

// ------------------------------------------------------------- sorting
__global__ void k_iota(int64_t n, int32_t *o) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) o[i] = (int32_t)i;
}
__global__ void k_gather_nodes(int64_t n, const int32_t *perm, const uint8_t *leaf_in, const double4 *val_in,
                               uint8_t *leaf_out, double4 *val_out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    leaf_out[i] = leaf_in[perm[i]];
    val_out[i] = val_in[perm[i]];
}

struct AmrCtx {
    fdm_handle *h;
    NodeSet A, B;          // current / next node set
    int a = 0;             // which buffer triple (amr[0..2] or amr[3..5]) holds A
    int64_t cap = 0;       // capacity of both triples
};

static void bind_sets(fdm_handle *h, AmrCtx &X) {
    const int64_t na = X.A.n, nb = X.B.n;
    NodeSet *S[2] = {&X.A, &X.B};
    for (int s = 0; s < 2; ++s) {
        const int b = s == 0 ? X.a : 1 - X.a;
        S[s]->key = h->amr[3 * b + 0].as<uint64_t>();
        S[s]->leaf = h->amr[3 * b + 1].as<uint8_t>();
        S[s]->val = h->amr[3 * b + 2].as<double4>();
        S[s]->rf = nullptr;
    }
    X.A.n = na;
    X.B.n = nb;
}
static void swap_sets(fdm_handle *h, AmrCtx &X) {
    X.a = 1 - X.a;
    std::swap(X.A.n, X.B.n);
    bind_sets(h, X);
}
// room for n nodes in both triples; the contents of both are dropped when
// they have to grow (callers grow only before writing into B, after A's last
// reader has finished)
static int grow_nodes(fdm_handle *h, AmrCtx &X, int64_t n) {
    if (n <= X.cap) return FDM_OK;
    FDM_CK(h, cudaStreamSynchronize(h->s));
    int64_t c = n + n / 2 + 1024;
    if (c < 2 * X.cap) c = 2 * X.cap;   // geometric growth while a run refines from its background mesh
    for (int s = 0; s < 2; ++s) {
        FDM_CK(h, h->amr[3 * s + 0].ensure(c * 8));
        FDM_CK(h, h->amr[3 * s + 1].ensure(c));
        FDM_CK(h, h->amr[3 * s + 2].ensure(c * 32));
    }
    X.cap = c;
    bind_sets(h, X);
    return FDM_OK;
}

// Merge of two key-sorted runs (keys distinct) into the node set out: an
// entry's place is its index in its run plus the number of keys of the
// other run below it.
__global__ void k_merge_runs(const uint64_t *__restrict__ ka, const uint8_t *__restrict__ la,
                             const double4 *__restrict__ va, int64_t na, const uint64_t *__restrict__ kb,
                             const uint8_t *__restrict__ lb, const double4 *__restrict__ vb, int64_t nb, NodeSet out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= na + nb) return;
    const bool in_a = i < na;
    const int64_t j = in_a ? i : i - na;
    const uint64_t k = in_a ? ka[j] : kb[j];
    const uint64_t *other = in_a ? kb : ka;
    int64_t lo = 0, hi = in_a ? nb : na;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (other[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    const int64_t o = j + lo;
    out.key[o] = k;
    out.leaf[o] = in_a ? la[j] : lb[j];
    out.val[o] = in_a ? va[j] : vb[j];
}
// the runs [0, m) and [m, n) of (keys, leaf, val), each sorted, into out
static void merge_into(fdm_handle *h, const uint64_t *keys, const uint8_t *leaf, const double4 *val, int64_t m,
                       int64_t n, NodeSet &out) {
    if (n > 0)
        k_merge_runs<<<nblk(n, 256), 256, 0, h->s>>>(keys, leaf, val, m, keys + m, leaf + m, val + m, n - m, out);
    out.n = n;
}
// (keys, leaf, val) of length n, already in key order, into out
static int copy_into(fdm_handle *h, int64_t n, const uint64_t *keys, const uint8_t *leaf, const double4 *val,
                     NodeSet &out) {
    if (n > 0) {
        FDM_CK(h, cudaMemcpyAsync(out.key, keys, n * 8, cudaMemcpyDeviceToDevice, h->s));
        FDM_CK(h, cudaMemcpyAsync(out.leaf, leaf, n, cudaMemcpyDeviceToDevice, h->s));
        FDM_CK(h, cudaMemcpyAsync(out.val, val, n * 32, cudaMemcpyDeviceToDevice, h->s));
    }
    out.n = n;
    return FDM_OK;
}

// per-cell index of A's keys (amr[22]) for the root-confined searches
static int index_set(fdm_handle *h, NodeSet &A) {
    const int64_t nroots = (int64_t)h->G.m * h->G.n;
    FDM_CK(h, h->amr[22].ensure((nroots + 1) * 4));
    k_root_first<<<nblk(A.n + 1, 256), 256, 0, h->s>>>(A.n, A.key, nroots, h->amr[22].as<int32_t>());
    A.rf = h->amr[22].as<int32_t>();
    A.nroots = nroots;
    return FDM_OK;
}


// exclusive scan of n counts and their total; *at_val: the prefix at index
// at (0 <= at < n), read back in the same round trip
static int scan_total32(fdm_handle *h, const int32_t *in, int32_t *out, int64_t n, int64_t &total,
                        int64_t at = -1, int64_t *at_val = nullptr) {
    size_t bytes = 0;
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(h->cub_tmp.p, bytes, in, out, (int)n, h->s));
    int32_t a = 0, b = 0, c = 0;
    FDM_CK(h, cudaMemcpyAsync(&a, in + n - 1, 4, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(&b, out + n - 1, 4, cudaMemcpyDeviceToHost, h->s));
    if (at_val && at >= 0 && at < n) FDM_CK(h, cudaMemcpyAsync(&c, out + at, 4, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    total = (int64_t)a + b;
    if (at_val) *at_val = at >= n ? total : (int64_t)c;
    return FDM_OK;
}

// exclusive scan without reading the total back
static int scan_i32_only(fdm_handle *h, const int32_t *in, int32_t *out, int64_t n) {
    size_t bytes = 0;
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(h->cub_tmp.p, bytes, in, out, (int)n, h->s));
    return FDM_OK;
}

// internal nodes and their interpA values from the current leaf set
// (values as the reference's import of a leaf set would give them)
int init_internal(fdm_handle *h) {
    const int TB = 256;
    const int64_t NL = h->NL;
    Carve cv;
    cv.add(NL * 4); cv.add(NL * 4);
    FDM_CK(h, h->amr[8].ensure(cv.total));
    int32_t *cnt = cv.at<int32_t>(h->amr[8], 0), *off = cv.at<int32_t>(h->amr[8], 1);
    k_anc_count<<<nblk(NL, TB), TB, 0, h->s>>>(NL, h->lkey.as<uint64_t>(), cnt);
    int64_t na = 0;
    int rc = scan_total32(h, cnt, off, NL, na);
    if (rc) return rc;
    h->NInt = 0;
    if (na == 0) return FDM_OK;
    FDM_CK(h, h->amr[9].ensure(na * 8 * 2 + 64));
    uint64_t *anc = h->amr[9].as<uint64_t>(), *srt = anc + na;
    k_anc_emit<<<nblk(NL, TB), TB, 0, h->s>>>(NL, h->lkey.as<uint64_t>(), off, anc);
    size_t bytes = 0;
    const int kb = 34 + root_bits(h);   // ancestor node keys
    FDM_CK(h, cub::DeviceRadixSort::SortKeys(nullptr, bytes, anc, srt, (int)na, 0, kb, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceRadixSort::SortKeys(h->cub_tmp.p, bytes, anc, srt, (int)na, 0, kb, h->s));
    FDM_CK(h, h->ikey.ensure(na * 8));
    FDM_CK(h, h->amr[10].ensure(16));
    int64_t *nsel = h->amr[10].as<int64_t>();
    bytes = 0;
    FDM_CK(h, cub::DeviceSelect::Unique(nullptr, bytes, srt, h->ikey.as<uint64_t>(), nsel, (int)na, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceSelect::Unique(h->cub_tmp.p, bytes, srt, h->ikey.as<uint64_t>(), nsel, (int)na, h->s));
    int64_t ni = 0;
    FDM_CK(h, cudaMemcpyAsync(&ni, nsel, 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    h->NInt = ni;
    FDM_CK(h, h->ival.ensure(ni * 32 + 32));
    for (int l = MAXLVL_TAB - 2; l >= 0; --l)
        k_internal_vals<<<nblk(ni, TB), TB, 0, h->s>>>(ni, h->ikey.as<uint64_t>(), h->ival.as<double4>(), l,
                                                      h->lkey.as<uint64_t>(), NL, h->lslot.as<int32_t>(),
                                                      h->B[0].as<double4>());
    FDM_CK(h, cudaGetLastError());
    return FDM_OK;
}

// ----------------------------------------------------------- solute_ref
// refine flags of the leaves (solute_ref_sub, src/solution.F90:519-535)
__global__ void k_refine_flags(Tables T, Geometry G, fdm_params P, const double *rot_slot, const double *div_slot,
                               const double *sums, int8_t *rflag) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= T.NL) return;
    const uint64_t key = T.lkey[k];
    const int lvl = (int)(key & 15u);
    const int cr = root_cross(G, (int64_t)(key >> 34));
    const int32_t s = T.lslot[k];
    rflag[k] = 0;
    if ((cr == 0 || cr == 1) && lvl < P.lvl_amr && s < T.NI) {
        const double arot = sqrt(sums[0] / sums[2]);
        const double adiv = sqrt(sums[1] / sums[2]);
        if (rot_slot[s] > P.refine_goal_rot * arot || div_slot[s] > P.refine_goal_div * adiv) rflag[k] = 1;
    }
}
// coarsen flags of internal nodes (solute_coarse_sub, src/solution.F90:490-517):
// all four sons are leaves, none refined in this pass, means below the goals
__global__ void k_coarsen_flags(int64_t NInt, const uint64_t *ikey, Tables T, fdm_params P, const double *rot_slot,
                                const double *div_slot, const double *sums, const int8_t *rflag, int8_t *cflag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= NInt) return;
    cflag[i] = 0;
    const uint64_t k = ikey[i];
    if ((int)(k & 15u) >= P.lvl_amr) return;
    double r[4], d[4];
    for (int q = 0; q < 4; ++q) {
        const int64_t li = find_key_t(T, child_key(k, q));
        if (li < 0 || rflag[li]) return;
        const int32_t s = T.lslot[li];
        r[q] = s < T.NI ? rot_slot[s] : 0.0;
        d[q] = s < T.NI ? div_slot[s] : 0.0;
    }
    const double arot = sqrt(sums[0] / sums[2]);
    const double adiv = sqrt(sums[1] / sums[2]);
    // son1 + son2 + son3 + son4 = q0 + q1 + q3 + q2
    if ((r[0] + r[1] + r[3] + r[2]) / 4 < P.coarse_goal_rot * arot &&
        (d[0] + d[1] + d[3] + d[2]) / 4 < P.coarse_goal_div * adiv)
        cflag[i] = 1;
}
__global__ void k_ref_count(Tables T, const int8_t *rflag, const uint64_t *ikey, int64_t NInt, const int8_t *cflag,
                            int32_t *cnt) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < T.NL) {
        const uint64_t key = T.lkey[k];
        int c = rflag[k] ? 5 : 1;
        if ((key & 15u) > 0) {
            const int64_t pi = find_key(ikey, NInt, parent_key(key));
            if (pi >= 0 && cflag[pi]) c = 0;
        }
        cnt[k] = c;
    } else if (k < T.NL + NInt) {
        cnt[k] = 1;
    }
}
__global__ void k_ref_emit(Tables T, const double4 *B0, const int8_t *rflag, const uint64_t *ikey, const double4 *ival,
                           int64_t NInt, const int8_t *cflag, const int32_t *off, uint64_t *okey, uint8_t *oleaf,
                           double4 *oval) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < T.NL) {
        const uint64_t key = T.lkey[k];
        if ((key & 15u) > 0) {
            const int64_t pi = find_key(ikey, NInt, parent_key(key));
            if (pi >= 0 && cflag[pi]) return;
        }
        const double4 v = B0[T.lslot[k]];
        int64_t o = off[k];
        okey[o] = key; oleaf[o] = rflag[k] ? 0 : 1; oval[o] = v;
        if (rflag[k]) {   // Refine_cell: sons copy U (src/mesh.F90:210-252)
            for (int q = 0; q < 4; ++q) {
                okey[o + 1 + q] = child_key(key, q); oleaf[o + 1 + q] = 1; oval[o + 1 + q] = v;
            }
        }
    } else if (k < T.NL + NInt) {
        const int64_t i = k - T.NL;
        const uint64_t key = ikey[i];
        const int64_t o = off[k];
        okey[o] = key;
        if (cflag[i]) {   // Coarse_cell: interpA of the four leaf sons (src/mesh.F90:397-408)
            double4 c[4];
            for (int q = 0; q < 4; ++q) c[q] = B0[T.lslot[find_key_t(T, child_key(key, q))]];
            oleaf[o] = 1;
            oval[o] = mean4(c[0], c[1], c[2], c[3]);
        } else {
            oleaf[o] = 0;
            oval[o] = ival[i];
        }
    }
}

// ----------------------------------------------------------- gridmodify1
struct Links {
    int32_t *parent, *child, *nb;   // child[4 n], nb[4 n] (up, down, right, left)
    uint64_t *rank;                 // post-order rank key of the visit (post_rank): compared, never indexed
    uint8_t *leaf0;
    int8_t *cross;
};
__global__ void k_gm1_links(NodeSet A, Geometry G, Links L, int32_t *max_lvl) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const uint64_t k = A.key[i];
    const int lvl = (int)(k & 15u);
    if (!A.leaf[i]) atomicMax(max_lvl, lvl);   // the deepest internal node
    L.parent[i] = lvl > 0 ? (int32_t)find_key_set(A, parent_key(k)) : -1;
    L.leaf0[i] = A.leaf[i];
    L.cross[i] = (int8_t)root_cross(G, (int64_t)(k >> 34));
    for (int q = 0; q < 4; ++q)
        L.child[4 * i + q] = A.leaf[i] ? -1 : (int32_t)find_key_set(A, child_key(k, q));
    for (int d = 0; d < 4; ++d) {
        uint64_t nk;
        L.nb[4 * i + d] = shift_key(G, k, d, nk) ? (int32_t)find_key_set(A, nk) : -1;
    }
    L.rank[i] = post_rank(k);
}
// "the same-level node N exists and has sons" when x is visited: decisions
// of earlier-visited nodes applied
__device__ __forceinline__ bool gm1_has_son(const Links &L, const int8_t *d, int32_t N, uint64_t rx) {
    if (N < 0) return false;
    for (int32_t a = L.parent[N]; a >= 0; a = L.parent[a])
        if (d[a] == D_COARSEN && L.rank[a] < rx) return false;
    if (!L.leaf0[N]) return !(d[N] == D_COARSEN && L.rank[N] < rx);
    return d[N] == D_REFINE && L.rank[N] < rx;
}
// gridmodify1 decision of one node (src/mesh.F90:305-353) given the current
// estimate of all decisions; a decision only reads decisions of nodes that
// are visited earlier, so iterating to a fixpoint gives the sequential result.
// The estimate is updated in place: a decision may read others already
// updated in the same sweep (never older than the last sweep's), which only
// shortens the chains; a sweep that changes nothing wrote nothing, so every
// decision in it read final values and the fixpoint (unique: the
// dependencies follow the visit order) is reached.
__global__ void k_gm1_decide(int64_t n, Links L, int8_t *d, int32_t *changed, int32_t *any) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= n) return;
    int8_t r = D_NONE;
    if (L.cross[x] == 0) {
        const uint64_t rx = L.rank[x];
        const bool up = gm1_has_son(L, d, L.nb[4 * x + DIR_UP], rx);
        const bool down = gm1_has_son(L, d, L.nb[4 * x + DIR_DOWN], rx);
        const bool left = gm1_has_son(L, d, L.nb[4 * x + DIR_LEFT], rx);
        const bool right = gm1_has_son(L, d, L.nb[4 * x + DIR_RIGHT], rx);
        if (L.leaf0[x]) {
            if ((left && right) || (up && down)) r = D_REFINE;
        } else {
            bool all_leaf = true;
            for (int q = 0; q < 4; ++q) {
                const int32_t c = L.child[4 * x + q];
                const bool lf = c >= 0 && ((L.leaf0[c] && d[c] != D_REFINE) || (!L.leaf0[c] && d[c] == D_COARSEN));
                all_leaf = all_leaf && lf;
            }
            if (all_leaf && ((!left && !right) || (!up && !down))) r = D_COARSEN;
        }
    }
    if (r != d[x]) {
        d[x] = r;
        atomicExch(changed, 1);
    }
    if (any && r != D_NONE) atomicExch(any, 1);
}
// values of coarsened nodes, deepest level first (interpA of the sons as they
// are at the node's visit)
__global__ void k_gm1_vals(NodeSet A, Links L, const int8_t *d, int lvl) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= A.n || d[x] != D_COARSEN || (int)(A.key[x] & 15u) != lvl) return;
    const int32_t *c = L.child + 4 * x;
    A.val[x] = mean4(A.val[c[0]], A.val[c[1]], A.val[c[2]], A.val[c[3]]);
}
__device__ __forceinline__ bool ancestor_coarsened(const Links &L, const int8_t *d, int32_t x) {
    for (int32_t a = L.parent[x]; a >= 0; a = L.parent[a])
        if (d[a] == D_COARSEN) return true;
    return false;
}
__global__ void k_gm1_count(int64_t n, Links L, const int8_t *d, int32_t *cnt) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= n) return;
    cnt[x] = ancestor_coarsened(L, d, (int32_t)x) ? 0 : (d[x] == D_REFINE ? 5 : 1);
}
__global__ void k_gm1_emit(NodeSet A, Links L, const int8_t *d, const int32_t *off, uint64_t *okey, uint8_t *oleaf,
                           double4 *oval) {
    const int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (x >= A.n || ancestor_coarsened(L, d, (int32_t)x)) return;
    const int64_t o = off[x];
    const uint64_t k = A.key[x];
    const double4 v = A.val[x];
    okey[o] = k;
    oval[o] = v;
    if (d[x] == D_REFINE) {
        oleaf[o] = 0;
        for (int q = 0; q < 4; ++q) { okey[o + 1 + q] = child_key(k, q); oleaf[o + 1 + q] = 1; oval[o + 1 + q] = v; }
    } else if (d[x] == D_COARSEN) {
        oleaf[o] = 1;
    } else {
        oleaf[o] = A.leaf[x];
    }
}

// ----------------------------------------------------------- gridmodify4
// live neighbour (src/neighbor.F90:65-196) on a sorted node set: the
// same-level node, else the deepest existing ancestor of it (a leaf)
__device__ int64_t live_nb_set(const NodeSet &A, const Geometry &G, uint64_t k, int dir) {
    uint64_t t;
    if (!shift_key(G, k, dir, t)) return -1;
    for (;;) {
        const int64_t i = find_key_set(A, t);
        if (i >= 0) return i;
        if ((t & 15u) == 0) return -1;
        t = parent_key(t);
    }
}
// leaves that can act in gridmodify4 (a neighbour, or the neighbour's
// neighbour, two or more levels coarser).  Later refinements of leaves only
// make neighbours finer; the one way a region gets coarser during the pass
// (a non-leaf refinement dropping a deep subtree) queues the leaves around
// it (push_ring)
__global__ void k_gm4_triggers(NodeSet A, Geometry G, int32_t *flag, uint64_t *rank, int32_t *idx) {
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= A.n) return;
    int f = 0;
    if (A.leaf[c]) {
        const uint64_t k = A.key[c];
        const int lc = (int)(k & 15u);
        const int dirs[4] = {DIR_RIGHT, DIR_LEFT, DIR_UP, DIR_DOWN};
        for (int t = 0; t < 4 && !f; ++t) {
            const int64_t nb = live_nb_set(A, G, k, dirs[t]);
            if (nb < 0) continue;
            if ((int)(A.key[nb] & 15u) <= lc - 2) { f = 1; break; }
            const int64_t nn = live_nb_set(A, G, A.key[nb], dirs[t]);
            if (nn >= 0 && (int)(A.key[nn] & 15u) <= lc - 2) f = 1;
        }
    }
    flag[c] = f;
    rank[c] = visit_rank(A.key[c]);
    idx[c] = (int32_t)c;
}

// An item of the replay: mk = visit rank * 2, + 1 for a leaf queued ahead of
// the traversal (so that on equal rank the initial trigger comes first), its
// pool index and the generation it was queued with.
struct __align__(16) HEnt {
    uint64_t mk;
    int32_t idx, gen;
};
// Hash table of the pool: open addressing over buckets of 8 entries, one
// 128-byte line each (8 keys, then 8 slot words).  A key's probe sequence is
// its home bucket's entries in order, then the next buckets' (linear
// probing from a bucket boundary), so at the table's load (a quarter or
// less) one bucket read settles a lookup but about once in a thousand.
constexpr int HB = 8;
struct __align__(128) HBucket {
    uint64_t key[HB];
    int32_t slot[HB];    // pool index (| SLOT_DEL when deleted), -1 empty
    int32_t pad[HB];
};
constexpr int HB_COPY = 96;   // the bytes of a bucket that a probe reads (keys and slots)
struct Pool {
    uint64_t *key;
    uint8_t *flags;
    int32_t *gen;
    double4 *val;
    HBucket *tab;
    uint64_t bmask;      // buckets - 1
    int64_t cap;         // pool capacity
    int64_t *n;          // pool size (device counter)
    HEnt *heap;          // heap of leaves to visit ahead of the traversal (spill)
    int64_t hcap;
    int32_t *err;        // [0] capacity exceeded, [1] visits, [2] non-leaf refines, [3] step limit,
                         // [4] refines, [5] replay steps
};
constexpr int32_t SLOT_DEL = 0x40000000;
// Home bucket hash: the key folded to 32 bits, then MurmurHash3's 32-bit
// finaliser (A. Appleby, public domain); 32-bit multiplies only
__device__ __forceinline__ uint64_t hmix(uint64_t k) {
    uint32_t x = (uint32_t)k ^ ((uint32_t)(k >> 32) * 0x9E3779B1u);
    x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13; x *= 0xC2B2AE35u; x ^= x >> 16;
    return x;
}
__device__ __forceinline__ uint64_t hhome(const Pool &P, uint64_t k) { return hmix(k) & P.bmask; }
__device__ __forceinline__ int32_t *hslot(const Pool &P, uint64_t pos) { return &P.tab[pos >> 3].slot[pos & 7]; }
__device__ __forceinline__ uint64_t *hkey(const Pool &P, uint64_t pos) { return &P.tab[pos >> 3].key[pos & 7]; }
// the entry after pos in every probe sequence through it
__device__ __forceinline__ uint64_t hnext(const Pool &P, uint64_t pos) {
    return (pos & 7) == 7 ? (((pos >> 3) + 1) & P.bmask) << 3 : pos + 1;
}
// key k in bucket b, read from memory: 1 found at entry e (slot word s),
// 0 absent (e = the first empty entry), -1 every entry holds another key
__device__ __forceinline__ int hscan_mem(const Pool &P, uint64_t b, uint64_t k, int &e, int32_t &s) {
    for (int j = 0; j < HB; ++j) {
        s = P.tab[b].slot[j];
        if (s == -1) { e = j; return 0; }
        if (P.tab[b].key[j] == k) { e = j; return 1; }
    }
    return -1;
}
// the same on the copy of a bucket in shared memory, without branches: bit
// masks of the empty entries and of the entries holding k, then the first of
// each
__device__ __forceinline__ int hscan_copy(const unsigned char *c, uint64_t k, int &e, int32_t &s) {
    const ulonglong2 *kp = reinterpret_cast<const ulonglong2 *>(c);
    const int4 *sp = reinterpret_cast<const int4 *>(c + HB * 8);
    unsigned em = 0, mm = 0;
#pragma unroll
    for (int j = 0; j < HB / 2; ++j) {
        const ulonglong2 v = kp[j];
        mm |= (v.x == k ? 1u : 0u) << (2 * j);
        mm |= (v.y == k ? 1u : 0u) << (2 * j + 1);
    }
#pragma unroll
    for (int j = 0; j < HB / 4; ++j) {
        const int4 v = sp[j];
        em |= (v.x == -1 ? 1u : 0u) << (4 * j);
        em |= (v.y == -1 ? 1u : 0u) << (4 * j + 1);
        em |= (v.z == -1 ? 1u : 0u) << (4 * j + 2);
        em |= (v.w == -1 ? 1u : 0u) << (4 * j + 3);
    }
    // entries fill in order, so the key can only sit before the first empty one
    const unsigned live = em ? (em & (0u - em)) - 1u : 0xFFu;   // entries before the first empty
    mm &= live;
    const int fe = em ? __ffs(em) - 1 : HB, fm = mm ? __ffs(mm) - 1 : HB;
    e = mm ? fm : fe;
    s = mm ? reinterpret_cast<const int32_t *>(c + HB * 8)[fm] : -1;
    return mm ? 1 : (em ? 0 : -1);
}
// key k's entry from bucket b on: 1 found at pos (slot word s), 0 absent
// (pos = the first empty entry of its sequence), -1 the table is full
__device__ __forceinline__ int hlocate_from(const Pool &P, uint64_t k, uint64_t b, uint64_t &pos, int32_t &s) {
    for (uint64_t probe = 0; probe <= P.bmask; ++probe) {
        int e = 0;
        const int r = hscan_mem(P, b, k, e, s);
        if (r >= 0) { pos = b * HB + (uint64_t)e; return r; }
        b = (b + 1) & P.bmask;
    }
    return -1;
}
__device__ __forceinline__ int hlocate(const Pool &P, uint64_t k, uint64_t &pos, int32_t &s) {
    return hlocate_from(P, k, hhome(P, k), pos, s);
}
// asynchronous copy of a bucket's keys and slot words into shared memory
__device__ __forceinline__ void hfetch(const Pool &P, uint64_t b, unsigned char *dst) {
    const unsigned char *src = reinterpret_cast<const unsigned char *>(&P.tab[b]);
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
#pragma unroll
    for (int q = 0; q < HB_COPY / 16; ++q)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d + 16 * q), "l"(src + 16 * q) : "memory");
}
__device__ __forceinline__ void hfetch_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__global__ void k_pool_init(NodeSet A, Pool P) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    const uint64_t k = A.key[i];
    P.key[i] = k;
    P.flags[i] = A.leaf[i] ? PF_LEAF : 0;
    P.gen[i] = 0;
    P.val[i] = A.val[i];
    // claim the first free entry of the sequence (entries only fill up here)
    uint64_t b = hhome(P, k);
    for (uint64_t probe = 0; probe <= P.bmask; ++probe) {
        for (int j = 0; j < HB; ++j) {
            if (P.tab[b].slot[j] != -1) continue;
            if (atomicCAS(&P.tab[b].slot[j], -1, (int32_t)i) == -1) {
                P.tab[b].key[j] = k;
                return;
            }
        }
        b = (b + 1) & P.bmask;
    }
}
// entry position of key k (live or deleted), or -1
__device__ __forceinline__ int64_t hpos(const Pool &P, uint64_t k, int32_t &s) {
    uint64_t pos = 0;
    s = -1;
    return hlocate(P, k, pos, s) == 1 ? (int64_t)pos : -1;
}
// pool index of the live node with key k, or -1
__device__ __forceinline__ int32_t hfind(const Pool &P, uint64_t k) {
    int32_t s;
    if (hpos(P, k, s) < 0) return -1;
    return (s & SLOT_DEL) ? -1 : s;
}
// insert or revive a leaf with value v (one lane); pn is the pool size.
// Returns its pool index or -1
__device__ int32_t hinsert(const Pool &P, uint64_t k, const double4 &v, int64_t &pn) {
    int32_t s;
    uint64_t pos;
    const int r = hlocate(P, k, pos, s);
    if (r < 0) return -1;
    if (r == 1) {
        const int32_t i = s & ~SLOT_DEL;
        *hslot(P, pos) = i;
        P.flags[i] = PF_LEAF;
        P.gen[i] = P.gen[i] + 1;
        P.val[i] = v;
        return i;
    }
    const int64_t i = pn;
    if (i >= P.cap) return -1;
    pn = i + 1;
    P.key[i] = k; P.flags[i] = PF_LEAF; P.gen[i] = 0; P.val[i] = v;
    *hslot(P, pos) = (int32_t)i;
    *hkey(P, pos) = k;
    return (int32_t)i;
}

constexpr int GM4_BATCH = 8;      // items looked at together
constexpr int GM4_TWIN = 64;      // trigger window in shared memory
constexpr int GM4_SQ = 4096;      // sorted queue in shared memory (16 B entries)

// Leaves to visit ahead of the traversal, ordered by mk: a sorted array
// q[head, tail) in shared memory that the warp inserts into and consumes
// from the front, and a binary min-heap in global memory for what does not
// fit there and for the (rare) entries that one lane queues alone.  The
// sizes are kept uniform across the warp.
struct Heap {
    HEnt *e;
    int64_t cap, n;
};
struct Queue {
    HEnt *q;
    int head, tail;
    Heap g;
};
__device__ __forceinline__ bool hpush(Heap &H, const HEnt &x) {
    if (H.n >= H.cap) return false;
    int64_t i = H.n++;
    while (i > 0) {
        const int64_t pa = (i - 1) >> 1;
        const HEnt p = H.e[pa];
        if (p.mk <= x.mk) break;
        H.e[i] = p;
        i = pa;
    }
    H.e[i] = x;
    return true;
}
__device__ __forceinline__ HEnt hpop(Heap &H) {
    const HEnt top = H.e[0];
    const int64_t hn = --H.n;
    const HEnt last = H.e[hn];
    int64_t i = 0;
    for (;;) {
        int64_t c = 2 * i + 1;
        if (c >= hn) break;
        HEnt a = H.e[c];
        if (c + 1 < hn) {
            const HEnt b = H.e[c + 1];
            if (b.mk < a.mk) { a = b; ++c; }
        }
        if (a.mk >= last.mk) break;
        H.e[i] = a;
        i = c;
    }
    if (hn > 0) H.e[i] = last;
    return top;
}
__device__ __forceinline__ HEnt queued_leaf(uint64_t key, int32_t idx, int32_t gen) {
    HEnt x;
    x.mk = visit_rank(key) * 2 + 1;
    x.idx = idx;
    x.gen = gen;
    return x;
}
// one lane: into the global heap
__device__ __forceinline__ bool gpush_leaf(Heap &H, uint64_t key, int32_t idx, int32_t gen) {
    return hpush(H, queued_leaf(key, idx, gen));
}

// The warp inserts the entries x of the lanes with has (at most 4, lanes
// 0..3) into the sorted array: entries at or above each new one move up by
// the number of new ones below them, top chunk first; each new entry lands
// after the old entries with mk not above its own.  When the array is full
// its upper half moves to the global heap first.  Returns false when the
// global heap overflowed.
__device__ __forceinline__ bool sq_insert(Queue &Q, const HEnt &x, bool has) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned hm = __ballot_sync(FULL, has);
    const int k = __popc(hm);
    if (k == 0) return true;
    bool ok = true;
    if (Q.tail + k > GM4_SQ) {
        // move [head, tail) down to 0, ascending chunks (the target lies below the source)
        const int n = Q.tail - Q.head;
        if (Q.head > 0) {
            for (int b = 0; b < n; b += 32) {
                HEnt y;
                if (b + lane < n) y = Q.q[Q.head + b + lane];
                __syncwarp();
                if (b + lane < n) Q.q[b + lane] = y;
                __syncwarp();
            }
            Q.head = 0;
            Q.tail = n;
        }
        if (Q.tail + k > GM4_SQ) {   // the upper half goes to the global heap
            int e = 0;
            if (lane == 0)
                for (int j = n / 2; j < n; ++j)
                    if (!hpush(Q.g, Q.q[j])) e = 1;
            Q.tail = n / 2;
            Q.g.n = __shfl_sync(FULL, Q.g.n, 0);
            ok = __shfl_sync(FULL, e, 0) == 0;
            __syncwarp();
        }
    }
    uint64_t m[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) m[j] = __shfl_sync(FULL, x.mk, j);
    // rank among the new entries (equal keys by lane) and place among the old ones
    int rank = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        rank += ((hm >> j) & 1u) && (m[j] < x.mk || (m[j] == x.mk && j < lane)) ? 1 : 0;
    int ub = Q.head;
    if (has) {
        int hi = Q.tail;
        while (ub < hi) {
            const int mid = (ub + hi) >> 1;
            if (Q.q[mid].mk <= x.mk) ub = mid + 1;
            else hi = mid;
        }
    }
    for (int b = Q.tail - 32;; b -= 32) {
        const int p = b + lane;
        const bool in = p >= Q.head;
        HEnt y;
        int s = 0;
        if (in) {
            y = Q.q[p];
#pragma unroll
            for (int j = 0; j < 4; ++j) s += ((hm >> j) & 1u) && m[j] < y.mk ? 1 : 0;
        }
        __syncwarp();
        if (in && s > 0) Q.q[p + s] = y;
        __syncwarp();
        if (b <= Q.head || __any_sync(FULL, in && s == 0)) break;
    }
    if (has) Q.q[ub + rank] = x;
    Q.tail += k;
    __syncwarp();
    return ok;
}
// Entries of the global heap that belong among the first GM4_BATCH come
// into the sorted array before a merge
__device__ __forceinline__ bool sq_pull(Queue &Q) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    bool ok = true;
    while (Q.g.n > 0 && ok) {
        const uint64_t kth = Q.tail - Q.head >= GM4_BATCH ? Q.q[Q.head + GM4_BATCH - 1].mk : ~0ull;
        if (Q.g.e[0].mk >= kth) break;
        HEnt x;
        if (lane == 0) x = hpop(Q.g);
        Q.g.n = __shfl_sync(FULL, Q.g.n, 0);
        __syncwarp();
        ok = sq_insert(Q, x, lane == 0);
    }
    return ok;
}

// After a non-leaf Refine_cell dropped a subtree two or more levels deep,
// the region of pk (level l0) is coarser than before: leaves at level
// >= l0 + 3 in the four edge-adjacent level-l0 cells can now find one of the
// new sons as a neighbour (or neighbour's neighbour) two levels coarser.  The
// reference visits every leaf, so those ahead of the traversal are queued.
__device__ __noinline__ bool push_ring(const Pool &P, const Geometry &G, Heap &H, uint64_t pk, uint64_t cur_rank) {
    const int l0 = (int)(pk & 15u);
    const int dirs[4] = {DIR_RIGHT, DIR_LEFT, DIR_UP, DIR_DOWN};
    bool ok = true;
    for (int d = 0; d < 4; ++d) {
        uint64_t t;
        if (!shift_key(G, pk, dirs[d], t)) continue;
        const int32_t s0 = hfind(P, t);
        if (s0 < 0 || (P.flags[s0] & PF_LEAF)) continue;
        uint64_t st[64];
        int sp = 0;
        st[sp++] = t;
        while (sp > 0) {
            const uint64_t k = st[--sp];
            for (int q = 0; q < 4; ++q) {
                const uint64_t ck = child_key(k, q);
                const int32_t c = hfind(P, ck);
                if (c < 0) continue;
                if (P.flags[c] & PF_LEAF) {
                    if ((int)(ck & 15u) >= l0 + 3 && visit_rank(ck) > cur_rank) ok = gpush_leaf(H, ck, c, P.gen[c]) && ok;
                } else if (sp < 64) {
                    st[sp++] = ck;
                } else {
                    ok = false;
                }
            }
        }
    }
    return ok;
}
// Refine_cell (src/mesh.F90:199-260) of a non-leaf whose old subtree is
// dropped and whose new sons copy its stale value (counted in nl); one lane.
// cur_rank is the visit rank of the leaf being visited.
__device__ __noinline__ bool refine_nonleaf(const Pool &P, const Geometry &G, Heap &H, int32_t p, uint64_t cur_rank,
                                            int32_t &nl, int64_t &pn) {
    const uint64_t pk = P.key[p];
    bool deep = false, ok = true;
    nl += 1;
    uint64_t st[64];
    int sp = 0;
    st[sp++] = pk;
    while (sp > 0) {
        const uint64_t k = st[--sp];
        for (int q = 0; q < 4; ++q) {
            int32_t s;
            const int64_t pos = hpos(P, child_key(k, q), s);
            if (pos < 0 || (s & SLOT_DEL)) continue;
            if (!(P.flags[s] & PF_LEAF)) {
                if (k != pk) deep = true;
                if (sp < 64) st[sp++] = P.key[s];
                else ok = false;
            }
            P.flags[s] |= PF_DELETED;
            *hslot(P, (uint64_t)pos) = s | SLOT_DEL;
        }
    }
    P.flags[p] = 0;   // internal, value kept
    const double4 v = P.val[p];
    for (int q = 0; q < 4; ++q) {
        const uint64_t ck = child_key(pk, q);
        const int32_t c = hinsert(P, ck, v, pn);
        if (c < 0) return false;
        if (visit_rank(ck) > cur_rank) ok = gpush_leaf(H, ck, c, P.gen[c]) && ok;
    }
    if (deep) ok = push_ring(P, G, H, pk, cur_rank) && ok;
    return ok;
}
// Is the node with key s (or the position s stands for) inside node r?
__device__ __forceinline__ bool key_inside(uint64_t r, uint64_t s) {
    const int lr = (int)(r & 15u), ls = (int)(s & 15u);
    if (lr > ls || (r >> 34) != (s >> 34)) return false;
    const uint64_t path_mask = (1ull << 30) - 1ull;
    const uint64_t keep = lr == 0 ? 0ull : (path_mask & ~((1ull << (30 - 2 * lr)) - 1ull));
    return (((s >> 4) & path_mask) & keep) == ((r >> 4) & path_mask);
}

// A lookup from key k towards d starts at the shifted key S and walks up to
// the first existing node; refining or dropping node R changes it only when
// S lies inside R.  sk = S (or ~0 when the shift leaves the grid).  It is
// made by a group of 4 consecutive lanes (mask gm, first lane g0): lane
// g0 + j probes the j-th ancestor of the walk's current start, copying its
// home bucket into the lane's shared-memory area lk (HB_COPY bytes), and
// the deepest node found ends the walk; otherwise the walk moves up 4
// levels.  Every lane of the group returns the result.
__device__ __forceinline__ int32_t group_lookup(const Pool &P, const Geometry &G, uint64_t k, int d, uint64_t &nk,
                                                uint64_t &sk, unsigned char *lk, unsigned gm, int g0) {
    const int j = (int)(threadIdx.x & 3);
    uint64_t t;
    if (!shift_key(G, k, d, t)) { sk = ~0ull; return -1; }
    sk = t;
    for (;;) {
        const int lt = (int)(t & 15u);
        const uint64_t c = ancestor_key(t, lt > j ? lt - j : 0);
        bool found = false;
        int32_t s = -1;
        if (j <= lt) {
            const uint64_t b = hhome(P, c);
            hfetch(P, b, lk);
            hfetch_wait();
            int e = 0;
            int r = hscan_copy(lk, c, e, s);
            if (r < 0) {   // a full bucket: the sequence goes on in the next ones
                uint64_t pos;
                r = hlocate_from(P, c, (b + 1) & P.bmask, pos, s);
            }
            found = r == 1 && !(s & SLOT_DEL);
        }
        const unsigned fm = (__ballot_sync(gm, found) >> g0) & 0xFu;
        if (fm) {
            const int w = g0 + __ffs(fm) - 1;
            nk = __shfl_sync(gm, c, w);
            return __shfl_sync(gm, s, w);
        }
        if (lt < 4) return -1;   // level 0 was probed
        t = ancestor_key(t, lt - 4);
    }
}
// the reference's direction order of gridmodify4: right, left, up, down
__device__ __forceinline__ int gm4_dir(int t) { return (t + DIR_RIGHT) & 3; }
// the neighbour of leaf k in direction t of that order and the neighbour's
// neighbour, by a group of 4 lanes
struct Look {
    int32_t nb, nn;
    uint64_t nbk, nnk, snb, snn;
};
__device__ __forceinline__ void group_dir_lookups(const Pool &P, const Geometry &G, uint64_t k, int t, Look &L,
                                                  unsigned char *lk, unsigned gm, int g0) {
    L.nn = -1;
    L.snn = ~0ull;
    L.nnk = 0;
    L.nb = group_lookup(P, G, k, gm4_dir(t), L.nbk, L.snb, lk, gm, g0);
    if (L.nb >= 0) L.nn = group_lookup(P, G, L.nbk, gm4_dir(t), L.nnk, L.snn, lk, gm, g0);
}

// Refine_cell of pool node p (key pk) by the warp.  Lanes 0..3 read the
// node's flags and value and make the first probe for their son's key at
// once.  A leaf's sons are then stored by those lanes: a son found in the
// table (dropped earlier) is revived, the others take new pool entries and
// the first empty slot of their probe sequence.  Sons whose sequences share
// that slot take it one at a time, lowest lane first, the others probing on
// past it.  A non-leaf (rare) is refined by lane 0 alone.  pn (the pool
// size) is uniform.  Returns false when the pool or the queue overflowed.
__device__ __forceinline__ bool refine_warp(Pool &P, const Geometry &G, Queue &Q, int32_t p, uint64_t pk, uint64_t cur_rank,
                            int32_t &nonleaf, int64_t &pn, unsigned char *lk) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const bool son = lane < 4;
    int fp = 0;
    double4 v = make_double4(0.0, 0.0, 0.0, 0.0);
    uint64_t ck = 0, b = 0;
    if (son) {
        ck = child_key(pk, lane);
        b = hhome(P, ck);
        hfetch(P, b, lk);
        fp = P.flags[p];
        v = P.val[p];
        hfetch_wait();
    }
    fp = __shfl_sync(FULL, fp, 0);
    bool ok = true;
    if (!(fp & PF_LEAF)) {
        int e = 0;
        if (lane == 0) {
            // out of line on copies, so that the queue and counters stay in registers
            Heap g = Q.g;
            int32_t nl = nonleaf;
            int64_t pn1 = pn;
            e = refine_nonleaf(P, G, g, p, cur_rank, nl, pn1) ? 0 : 1;
            Q.g.n = g.n;
            nonleaf = nl;
            pn = pn1;
        }
        ok = __shfl_sync(FULL, e, 0) == 0;
        pn = __shfl_sync(FULL, pn, 0);
    } else {
        // the son's own entry (a dropped node), or the first empty entry
        bool found = false;
        uint64_t h = 0;
        int32_t s = -1;
        int r = 0;
        if (son) {
            int e = 0;
            r = hscan_copy(lk, ck, e, s);
            if (r >= 0) h = b * HB + (uint64_t)e;
            else r = hlocate_from(P, ck, (b + 1) & P.bmask, h, s);
            found = r == 1;
        }
        const unsigned nm = __ballot_sync(FULL, son && !found);
        int32_t i = -1, gen = 0;
        if (found) {
            i = s & ~SLOT_DEL;
            gen = P.gen[i] + 1;
        } else if (son) {
            i = (int32_t)(pn + __popc(nm & ((1u << lane) - 1u)));
        }
        pn += __popc(nm);
        ok = pn <= P.cap && !__any_sync(FULL, r < 0);   // the pool, or the table, is full
        if (ok) {
            bool need = son && !found;
            for (;;) {
                const unsigned pend = __ballot_sync(FULL, need);
                if (!pend) break;
                if (need) {
                    const unsigned peers = __match_any_sync(pend, h);
                    if (__ffs(peers) - 1 == lane) {
                        *hslot(P, h) = i;
                        *hkey(P, h) = ck;
                        need = false;
                    }
                }
                __syncwarp();
                bool lost = false;
                if (need) {   // a lower lane took the entry: probe on to the next empty one
                    lost = true;
                    for (uint64_t probe = 0; probe <= P.bmask * HB && lost; ++probe) {
                        h = hnext(P, h);
                        lost = *hslot(P, h) != -1;
                    }
                }
                if (__any_sync(FULL, lost)) { ok = false; break; }
            }
        }
        if (ok) {
            if (son) {
                if (found) *hslot(P, h) = i;
                else P.key[i] = ck;
                P.flags[i] = PF_LEAF;
                P.gen[i] = gen;
                P.val[i] = v;
            }
            if (lane == 0) P.flags[p] = 0;   // internal, value kept
            // the sons ahead of the traversal are queued
            ok = sq_insert(Q, queued_leaf(ck, i, gen), son && visit_rank(ck) > cur_rank);
        }
    }
    Q.g.n = __shfl_sync(FULL, Q.g.n, 0);
    if (!ok && lane == 0) P.err[0] = 1;
    __syncwarp();
    return ok;
}

__device__ __forceinline__ Look shfl_look(const Look &L, int src) {
    const unsigned FULL = 0xffffffffu;
    Look o;
    o.nb = __shfl_sync(FULL, L.nb, src);
    o.nn = __shfl_sync(FULL, L.nn, src);
    o.nbk = __shfl_sync(FULL, L.nbk, src);
    o.nnk = __shfl_sync(FULL, L.nnk, src);
    o.snb = __shfl_sync(FULL, L.snb, src);
    o.snn = __shfl_sync(FULL, L.snn, src);
    return o;
}

constexpr int GM4_THREADS = 128;   // 8 leaves x 4 directions x 4 probing lanes

// gridmodify4 (src/mesh.F90:355-395) over one pass of the tree, by one
// block.  The leaves that can act (the initial triggers, sorted by visit
// rank, and every leaf queued ahead of the traversal) are visited in
// traversal order.  Warp 0 merges the next 8 of them from the sorted queue
// and the trigger window (its lanes at once); then the whole block looks at
// them together: 16 threads per leaf find its right/left/up/down neighbour
// and that neighbour's neighbour, 4 per direction.  Warp 0 then tells which
// directions would refine something.  The leaves before the first one that
// refines have no effect but being visited, so they are marked in
// parallel; the first one that refines is then applied alone, in order, by
// warp 0, and the batch ends there (the leaves after it stay where they are
// for the next batch).  Within that leaf a lookup starts at a shifted key
// and walks up to the first existing node, so a refinement (or a dropped
// subtree) of node R can change a later lookup only when its start lies
// inside R: those lookups, and only those, are repeated.  A leaf that is
// both a trigger and queued is looked at twice; the second look finds it
// visited.
__global__ void __launch_bounds__(GM4_THREADS) k_gm4_block(Pool P, Geometry G, const uint64_t *__restrict__ trank,
                                                           const int32_t *__restrict__ tidx, int64_t ntrig,
                                                           int64_t max_steps) {
    extern __shared__ __align__(16) unsigned char gm4_smem[];
    __shared__ HEnt items[GM4_BATCH];
    __shared__ uint64_t twr[GM4_TWIN];
    __shared__ int32_t twx[GM4_TWIN];
    __shared__ __align__(16) unsigned char lkbuf[GM4_THREADS][HB_COPY];   // each thread's bucket copy
    __shared__ Look looks[GM4_BATCH][4];
    __shared__ uint8_t s_fl[GM4_BATCH], s_valid[GM4_BATCH];
    __shared__ int s_cnt;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned char *lk = lkbuf[tid];
    const unsigned FULL = 0xffffffffu;
    // this thread's part of the block-wide lookups
    const int bi = tid >> 4, bd = (tid >> 2) & 3, g0 = lane & ~3;
    const unsigned gmask = 0xFu << g0;
    // warp 0's state (uniform in warp 0)
    Queue Q;
    Q.q = reinterpret_cast<HEnt *>(gm4_smem);
    Q.head = Q.tail = 0;
    Q.g.e = P.heap;
    Q.g.cap = P.hcap;
    Q.g.n = 0;
    int64_t pn = *P.n;     // pool size (stored at the end)
    int64_t tg = 0;        // next trigger to bring into the window
    int tw_n = 0, tp = 0;  // triggers in the window, next one to merge
    int64_t step = 0;
    int32_t visits = 0, nonleaf = 0, refines = 0;   // lane 0's counts, stored at the end
    bool ok = true;
    bool take = false;     // warp 0: this lane's merged entry is an item ...
    int pos = 0;           // ... at this place
    for (;; ++step) {
        // warp 0 reaches here from lane-level branches of the refinement;
        // reconverge it before the lane-parallel merge, or its lanes can run
        // the merge in separate groups
        __syncwarp();
        if (warp == 0) {
            int c = 0;
            if (step >= max_steps) {
                if (lane == 0) P.err[3] = 1;
            } else if (ok) {
                // keep at least a batch of triggers in the window
                if (tw_n - tp < GM4_BATCH && tg < ntrig) {
                    const int rem = tw_n - tp;
                    uint64_t rr = 0;
                    int32_t rx = 0;
                    if (lane < rem) { rr = twr[tp + lane]; rx = twx[tp + lane]; }
                    __syncwarp();
                    if (lane < rem) { twr[lane] = rr; twx[lane] = rx; }
                    const int nl = (int)min((int64_t)(GM4_TWIN - rem), ntrig - tg);
                    for (int j = lane; j < nl; j += 32) { twr[rem + j] = trank[tg + j]; twx[rem + j] = tidx[tg + j]; }
                    tg += nl;
                    tw_n = rem + nl;
                    tp = 0;
                    __syncwarp();
                }
                if (Q.g.n > 0 && !sq_pull(Q)) ok = false;
            }
            if (step < max_steps && ok) {
                // the next items in traversal order: lanes 0..7 hold the first
                // queued leaves, lanes 8..15 the first triggers; each finds its
                // place among the other list's eight (a trigger's mk is even, a
                // queued leaf's odd: no ties)
                HEnt x;
                x.mk = ~0ull; x.idx = -1; x.gen = 0;
                if (lane < GM4_BATCH) {
                    if (Q.head + lane < Q.tail) x = Q.q[Q.head + lane];
                } else if (lane < 2 * GM4_BATCH) {
                    const int j = tp + lane - GM4_BATCH;
                    if (j < tw_n) { x.mk = twr[j] * 2; x.idx = twx[j]; }
                }
                pos = lane & (GM4_BATCH - 1);
                const int other = lane < GM4_BATCH ? GM4_BATCH : 0;
#pragma unroll
                for (int j = 0; j < GM4_BATCH; ++j) {
                    const uint64_t o = __shfl_sync(FULL, x.mk, other + j);
                    pos += o < x.mk ? 1 : 0;
                }
                take = lane < 2 * GM4_BATCH && x.mk != ~0ull && pos < GM4_BATCH;
                if (take) items[pos] = x;
                c = __popc(__ballot_sync(FULL, take));
            }
            if (lane == 0) s_cnt = c;
        }
        __syncthreads();
        const int cnt = s_cnt;
        if (cnt == 0) break;
        // lookups: 16 threads per item, 4 per direction; the item's key comes
        // from its rank, so its flags and generation load meanwhile
        if (bi < cnt) {
            const HEnt it = items[bi];
            const uint64_t ck = key_of_visit_rank(it.mk >> 1);
            uint8_t fl = 0;
            int32_t gc = 0;
            const bool lead = (tid & 15) == 0;
            if (lead) { fl = P.flags[it.idx]; gc = P.gen[it.idx]; }
            Look L;
            group_dir_lookups(P, G, ck, bd, L, lk, gmask, g0);
            if ((tid & 3) == 0) looks[bi][bd] = L;
            if (lead) {
                s_fl[bi] = fl;
                s_valid[bi] = gc == it.gen && (fl & (PF_LEAF | PF_DELETED | PF_VISITED)) == PF_LEAF;
            }
        }
        __syncthreads();
        if (warp != 0) continue;
        // decisions: lane (grp, tl) tells whether direction tl of item grp refines
        const int grp = lane >> 2, tl = lane & 3;
        bool valid = false, acts = false;
        uint8_t fl = 0;
        HEnt it;
        it.mk = 0; it.idx = -1; it.gen = 0;
        if (grp < cnt) {
            it = items[grp];
            valid = s_valid[grp] != 0;
            fl = s_fl[grp];
            const Look L = looks[grp][tl];
            const int lc = (int)(it.mk >> 1) & 15;
            acts = valid &&
                   ((L.nb >= 0 && (int)(L.nbk & 15u) <= lc - 2) || (L.nn >= 0 && (int)(L.nnk & 15u) <= lc - 2));
        }
        const unsigned am = __ballot_sync(FULL, acts);
        const int fa = am ? (__ffs(am) - 1) >> 2 : cnt;   // first item that refines
        // items before it: visited, nothing else
        const unsigned vm = __ballot_sync(FULL, valid && tl == 0 && grp < fa);
        if (valid && tl == 0 && grp < fa) P.flags[it.idx] = fl | PF_VISITED;
        if (lane == 0) visits += __popc(vm);
        const int consumed = fa < cnt ? fa + 1 : cnt;
        // the consumed items leave the front of their lists (the sons queued
        // below all rank after the item being visited)
        const int cq = __popc(__ballot_sync(FULL, take && lane < GM4_BATCH && pos < consumed));
        Q.head += cq;
        tp += consumed - cq;
        if (fa < cnt) {
            const HEnt ib = items[fa];
            const uint64_t rb = ib.mk >> 1;
            const uint64_t kb = key_of_visit_rank(rb);
            const int lc = (int)(kb & 15u);
            if (lane == 0) {
                P.flags[ib.idx] = s_fl[fa] | PF_VISITED;
                ++visits;
            }
            uint64_t refined[8];   // uniform: nodes refined by this leaf
            int nref = 0;
            for (int t = 0; t < 4 && ok; ++t) {
                Look Lt = looks[fa][t];
                // repeat the lookups whose start lies inside a node refined earlier
                bool re_nb = false, re_nn = false;
                for (int k = 0; k < nref; ++k) {
                    re_nb = re_nb || key_inside(refined[k], Lt.snb);
                    re_nn = re_nn || key_inside(refined[k], Lt.snn);
                }
                if (re_nb || re_nn) {
                    if (lane < 4) {
                        if (re_nb) group_dir_lookups(P, G, kb, t, Lt, lk, 0xFu, 0);
                        else Lt.nn = group_lookup(P, G, Lt.nbk, gm4_dir(t), Lt.nnk, Lt.snn, lk, 0xFu, 0);
                    }
                    Lt = shfl_look(Lt, 0);
                }
                if (Lt.nb < 0) continue;
                // a neighbour two levels coarser is a leaf (every internal node
                // has four sons), and refining it leaves the lookup of its own
                // neighbour unchanged (that start lies outside it)
                if ((int)(Lt.nbk & 15u) <= lc - 2) {
                    ok = refine_warp(P, G, Q, Lt.nb, Lt.nbk, rb, nonleaf, pn, lk);
                    refined[nref++] = Lt.nbk;
                    ++refines;
                }
                if (ok && Lt.nn >= 0 && (int)(Lt.nnk & 15u) <= lc - 2) {
                    ok = refine_warp(P, G, Q, Lt.nn, Lt.nnk, rb, nonleaf, pn, lk);
                    refined[nref++] = Lt.nnk;
                    ++refines;
                }
            }
        }
    }
    if (tid == 0) {
        if (!ok) P.err[0] = 1;
        *P.n = pn;
        P.err[1] = visits;
        P.err[2] = nonleaf;
        P.err[4] = refines;
        P.err[5] = (int32_t)step;
    }
}

__global__ void k_pool_live(int64_t n, const uint8_t *flags, int32_t *live) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) live[i] = !(flags[i] & PF_DELETED);
}
__global__ void k_pool_emit(int64_t n, const uint8_t *flags, const uint64_t *key, const double4 *val,
                            const int32_t *off, uint64_t *okey, uint8_t *oleaf, double4 *oval) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n || (flags[i] & PF_DELETED)) return;
    okey[off[i]] = key[i];
    oleaf[off[i]] = (flags[i] & PF_LEAF) ? 1 : 0;
    oval[off[i]] = val[i];
}

// ------------------------------------------------------------ extraction
__global__ void k_split_count(int64_t n, const uint8_t *leaf, int32_t *fl, int32_t *fi) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) { fl[i] = leaf[i] ? 1 : 0; fi[i] = leaf[i] ? 0 : 1; }
}
__global__ void k_split_emit(NodeSet A, const int32_t *ol, const int32_t *oi, uint64_t *lk, double4 *lv, uint64_t *ik,
                             double4 *iv) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= A.n) return;
    if (A.leaf[i]) { lk[ol[i]] = A.key[i]; lv[ol[i]] = A.val[i]; }
    else { ik[oi[i]] = A.key[i]; iv[oi[i]] = A.val[i]; }
}

// emission helper: count kernel already ran into cnt; scan; emit kernel fills
// the unsorted arrays (B's storage); sort into the other set
struct Emit {
    uint64_t *key;
    uint8_t *leaf;
    double4 *val;
};
static int emit_buffers(fdm_handle *h, int64_t n, Emit &E) {
    FDM_CK(h, h->amr[11].ensure(n * 8 + 16));
    FDM_CK(h, h->amr[12].ensure(n + 16));
    FDM_CK(h, h->amr[13].ensure(n * 32 + 32));
    E.key = h->amr[11].as<uint64_t>();
    E.leaf = h->amr[12].as<uint8_t>();
    E.val = h->amr[13].as<double4>();
    return FDM_OK;
}

#define AMR_RC(x)            \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

// one gridmodify1 pass over the node set A -> A
// One gridmodify1 pass over the node set A -> A; *did: a node was refined
// or coarsened (otherwise A is left as it is).
static int gridmodify1_pass(fdm_handle *h, AmrCtx &X, bool *did) {
    Nvtx range("fdm regrid: gridmodify1");
    const int TB = 256;
    const int64_t n = X.A.n;
    Carve cv;
    cv.add(n * 4); cv.add(n * 16); cv.add(n * 16); cv.add(n * 8); cv.add(n); cv.add(n);
    cv.add(n); cv.add(n); cv.add(16); cv.add(n * 4); cv.add(n * 4);
    FDM_CK(h, h->amr[14].ensure(cv.total));
    DevBuf &b = h->amr[14];
    Links L;
    L.parent = cv.at<int32_t>(b, 0); L.child = cv.at<int32_t>(b, 1); L.nb = cv.at<int32_t>(b, 2);
    L.rank = cv.at<uint64_t>(b, 3); L.leaf0 = cv.at<uint8_t>(b, 4); L.cross = cv.at<int8_t>(b, 5);
    int8_t *d0 = cv.at<int8_t>(b, 6);   // the decisions (slot 7 unused)
    int32_t *changed = cv.at<int32_t>(b, 8);
    int32_t *cnt = cv.at<int32_t>(b, 9), *off = cv.at<int32_t>(b, 10);
    AMR_RC(index_set(h, X.A));
    FDM_CK(h, cudaMemsetAsync(changed, 0, 16, h->s));
    k_gm1_links<<<nblk(n, TB), TB, 0, h->s>>>(X.A, h->G, L, changed + 2);
    FDM_CK(h, cudaMemsetAsync(d0, 0, n, h->s));
    int8_t *cur = d0;
    // Sweeps are enqueued GM1_SWEEPS at a time and the change flag of the
    // last one is read: once the decisions are settled a sweep changes
    // nothing, so the extra sweeps leave the fixpoint as it is.
    constexpr int GM1_SWEEPS = 4;
    int64_t it = 0;
    int deepest = MAXLVL_TAB - 2;   // a coarsened node is internal: no deeper than the deepest internal node
    for (;;) {
        if (it > n + 2 + GM1_SWEEPS) { h->err = "gridmodify1 decisions did not settle"; return FDM_ERR_UNSUPPORTED; }
        int32_t hc[3] = {0, 0, 0};   // last sweep: changed, any decision; deepest internal node
        for (int k = 0; k < GM1_SWEEPS; ++k) {
            const bool last = k == GM1_SWEEPS - 1;
            if (last) FDM_CK(h, cudaMemsetAsync(changed, 0, 8, h->s));   // the level stays
            k_gm1_decide<<<nblk(n, TB), TB, 0, h->s>>>(n, L, cur, changed, last ? changed + 1 : nullptr);
        }
        it += GM1_SWEEPS;
        FDM_CK(h, cudaMemcpyAsync(hc, changed, 12, cudaMemcpyDeviceToHost, h->s));
        FDM_CK(h, cudaStreamSynchronize(h->s));
        if (!hc[0]) {
            *did = hc[1] != 0;
            deepest = hc[2];
            break;
        }
    }
    h->gm1_iters += it;
    if (!*did) return FDM_OK;   // every decision is "nothing": A stays
    for (int l = deepest < MAXLVL_TAB - 2 ? deepest : MAXLVL_TAB - 2; l >= 0; --l)
        k_gm1_vals<<<nblk(n, TB), TB, 0, h->s>>>(X.A, L, cur, l);
    k_gm1_count<<<nblk(n, TB), TB, 0, h->s>>>(n, L, cur, cnt);
    int64_t total = 0;
    AMR_RC(scan_total32(h, cnt, off, n, total));
    Emit E;
    AMR_RC(emit_buffers(h, total, E));
    k_gm1_emit<<<nblk(n, TB), TB, 0, h->s>>>(X.A, L, cur, off, E.key, E.leaf, E.val);
    AMR_RC(grow_nodes(h, X, total));
    // the emit keeps key order: a refined leaf's sons follow it directly and
    // lie before every later node (they fill the leaf's own span)
    AMR_RC(copy_into(h, total, E.key, E.leaf, E.val, X.B));
    swap_sets(h, X);
    return FDM_OK;
}

// One gridmodify4 pass over the node set A -> A; *did: something was
// refined (otherwise A is left as it is).
static int gridmodify4_pass(fdm_handle *h, AmrCtx &X, bool *did) {
    Nvtx range("fdm regrid: gridmodify4");
    const int TB = 256;
    const int64_t n = X.A.n;
    Carve cv;
    cv.add(n * 4); cv.add(n * 8); cv.add(n * 4); cv.add(n * 8); cv.add(n * 4); cv.add(n * 4); cv.add(16);
    FDM_CK(h, h->amr[15].ensure(cv.total));
    DevBuf &b = h->amr[15];
    int32_t *flag = cv.at<int32_t>(b, 0), *idx = cv.at<int32_t>(b, 2), *sidx = cv.at<int32_t>(b, 4);
    uint64_t *rk = cv.at<uint64_t>(b, 1), *srk = cv.at<uint64_t>(b, 3);
    int32_t *foff = cv.at<int32_t>(b, 5);
    int64_t *nsel = cv.at<int64_t>(b, 6);
    AMR_RC(index_set(h, X.A));
    k_gm4_triggers<<<nblk(n, TB), TB, 0, h->s>>>(X.A, h->G, flag, rk, idx);
    // keep the triggering leaves, sorted by traversal rank
    size_t bytes = 0;
    FDM_CK(h, cub::DeviceSelect::Flagged(nullptr, bytes, rk, flag, srk, nsel, (int)n, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceSelect::Flagged(h->cub_tmp.p, bytes, rk, flag, srk, nsel, (int)n, h->s));
    FDM_CK(h, cub::DeviceSelect::Flagged(nullptr, bytes, idx, flag, sidx, nsel + 1, (int)n, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceSelect::Flagged(h->cub_tmp.p, bytes, idx, flag, sidx, nsel + 1, (int)n, h->s));
    int64_t ntrig = 0;
    FDM_CK(h, cudaMemcpyAsync(&ntrig, nsel, 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    *did = false;
    if (ntrig == 0) return FDM_OK;
    // key order is Morton order (son4 before son3); the traversal visits
    // son3 first, so sort the triggers by traversal rank
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(nullptr, bytes, srk, rk, sidx, idx, (int)ntrig, 0, 56, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceRadixSort::SortPairs(h->cub_tmp.p, bytes, srk, rk, sidx, idx, (int)ntrig, 0, 56, h->s));
    // pool + hash of all nodes, room for new ones
    const int64_t cap = 2 * n + 4096;
    uint64_t slots = 1;
    while (slots < (uint64_t)(2 * cap)) slots <<= 1;
    Carve cp;
    cp.add(cap * 8); cp.add(cap); cp.add(cap * 4); cp.add(cap * 32); cp.add(slots / HB * sizeof(HBucket)); cp.add(16);
    cp.add(cap * sizeof(HEnt)); cp.add(32);
    FDM_CK(h, h->amr[16].ensure(cp.total));
    DevBuf &pb = h->amr[16];
    Pool P;
    P.key = cp.at<uint64_t>(pb, 0); P.flags = cp.at<uint8_t>(pb, 1); P.gen = cp.at<int32_t>(pb, 2);
    P.val = cp.at<double4>(pb, 3); P.tab = cp.at<HBucket>(pb, 4); P.n = cp.at<int64_t>(pb, 5);
    P.heap = cp.at<HEnt>(pb, 6);
    P.err = cp.at<int32_t>(pb, 7);
    P.bmask = slots / HB - 1;
    P.cap = cap;
    P.hcap = cap;
    FDM_CK(h, cudaMemsetAsync(P.tab, 0xff, slots / HB * sizeof(HBucket), h->s));
    FDM_CK(h, cudaMemsetAsync(P.err, 0, 32, h->s));
    FDM_CK(h, cudaMemcpyAsync(P.n, &n, 8, cudaMemcpyHostToDevice, h->s));
    k_pool_init<<<nblk(n, TB), TB, 0, h->s>>>(X.A, P);
    // every step consumes a trigger or a queued leaf, or ends the pass
    const size_t gm4_smem = (size_t)GM4_SQ * sizeof(HEnt);
    FDM_CK(h, cudaFuncSetAttribute(k_gm4_block, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gm4_smem));
    for (cudaEvent_t &e : h->gm4_ev)
        if (!e) FDM_CK(h, cudaEventCreate(&e));
    FDM_CK(h, cudaEventRecord(h->gm4_ev[0], h->s));
    k_gm4_block<<<1, GM4_THREADS, gm4_smem, h->s>>>(P, h->G, rk, idx, ntrig, 2 * ntrig + 2 * P.hcap + 16);
    FDM_CK(h, cudaEventRecord(h->gm4_ev[1], h->s));
    int32_t herr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int64_t pn = 0;
    FDM_CK(h, cudaMemcpyAsync(herr, P.err, 32, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaMemcpyAsync(&pn, P.n, 8, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    float gm4_t = 0.f;
    if (cudaEventElapsedTime(&gm4_t, h->gm4_ev[0], h->gm4_ev[1]) == cudaSuccess) h->gm4_ms += gm4_t;
    if (herr[0]) { h->err = "gridmodify4 cascade exceeded its node pool"; return FDM_ERR_UNSUPPORTED; }
    if (herr[3]) { h->err = "gridmodify4 replay did not finish"; return FDM_ERR_UNSUPPORTED; }
    h->gm4_visits += herr[1];
    h->gm4_nonleaf += herr[2];
    h->gm4_refines += herr[4];
    h->gm4_steps += herr[5];
    h->gm4_triggers += ntrig;
    *did = herr[4] != 0;
    if (!*did) return FDM_OK;   // no Refine_cell: the pool holds A unchanged
    // live nodes back into a sorted node set
    Carve ce;
    ce.add(pn * 4); ce.add(pn * 4);
    FDM_CK(h, h->amr[17].ensure(ce.total));
    int32_t *live = ce.at<int32_t>(h->amr[17], 0), *loff = ce.at<int32_t>(h->amr[17], 1);
    k_pool_live<<<nblk(pn, TB), TB, 0, h->s>>>(pn, P.flags, live);
    int64_t total = 0, m = 0;   // m: live nodes of A (pool entries below n, in key order)
    AMR_RC(scan_total32(h, live, loff, pn, total, n, &m));
    Emit E;
    AMR_RC(emit_buffers(h, total, E));
    k_pool_emit<<<nblk(pn, TB), TB, 0, h->s>>>(pn, P.flags, P.key, P.val, loff, E.key, E.leaf, E.val);
    // the new nodes (in the order they were made) sorted by key, then merged
    // with the survivors of A
    const int64_t nb = total - m;
    FDM_CK(h, h->amr[23].ensure(nb * 8 + 16));
    FDM_CK(h, h->amr[24].ensure(nb + 16));
    FDM_CK(h, h->amr[25].ensure(nb * 32 + 32));
    uint64_t *bk = h->amr[23].as<uint64_t>();
    uint8_t *bl = h->amr[24].as<uint8_t>();
    double4 *bv = h->amr[25].as<double4>();
    if (nb > 0) {
        FDM_CK(h, h->amr[6].ensure(nb * 4 + 16));
        FDM_CK(h, h->amr[7].ensure(nb * 4 + 16));
        int32_t *iota = h->amr[6].as<int32_t>(), *perm = h->amr[7].as<int32_t>();
        k_iota<<<nblk(nb, TB), TB, 0, h->s>>>(nb, iota);
        size_t bytes = 0;
        const int kb = 34 + root_bits(h);
        FDM_CK(h, cub::DeviceRadixSort::SortPairs(nullptr, bytes, E.key + m, bk, iota, perm, (int)nb, 0, kb, h->s));
        FDM_CK(h, h->cub_tmp.ensure(bytes));
        FDM_CK(h, cub::DeviceRadixSort::SortPairs(h->cub_tmp.p, bytes, E.key + m, bk, iota, perm, (int)nb, 0, kb, h->s));
        k_gather_nodes<<<nblk(nb, TB), TB, 0, h->s>>>(nb, perm, E.leaf + m, E.val + m, bl, bv);
    }
    AMR_RC(grow_nodes(h, X, total));
    if (total > 0)
        k_merge_runs<<<nblk(total, TB), TB, 0, h->s>>>(E.key, E.leaf, E.val, m, bk, bl, bv, nb, X.B);
    X.B.n = total;
    swap_sets(h, X);
    return FDM_OK;
}

// AMR (src/solution.F90:408-421) after the trigger test: indicators,
// refine/coarsen, lvlAMR rounds of gridmodify1 + gridmodify4, new tables.
static int run_amr_impl(fdm_handle *h, fdm_handle *lead);

// A regrid that fails part way (an allocation, a CUDA call) leaves the node
// set and the tables out of step: the handle then counts as not loaded, so
// every stage call returns FDM_ERR_STATE until the next upload.  With a
// leader (lead != nullptr), the refine/coarsen decisions come from the
// leader's indicators on the leader's state; both must hold the same leaf
// set, which is checked on the device.
int run_amr(fdm_handle *h, fdm_handle *lead) {
    const int rc = run_amr_impl(h, lead);
    if (rc && rc != FDM_ERR_UNSUPPORTED && rc != FDM_ERR_ARG) h->loaded = false;
    return rc;
}

__global__ void k_keys_differ(int64_t n, const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                              int32_t *flag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n && a[i] != b[i]) *flag = 1;
}

// the same leaf set (keys in the same order) in both handles
static int same_leaves(fdm_handle *h, fdm_handle *lead, bool *same) {
    *same = false;
    if (h->NL != lead->NL || h->NI != lead->NI || h->NInt != lead->NInt) return FDM_OK;
    FDM_CK(h, cudaStreamSynchronize(lead->s));
    int32_t *flag = h->flag.as<int32_t>() + 7;
    FDM_CK(h, cudaMemsetAsync(flag, 0, 4, h->s));
    k_keys_differ<<<nblk(h->NL, 256), 256, 0, h->s>>>(h->NL, h->lkey.as<uint64_t>(), lead->lkey.as<uint64_t>(), flag);
    int32_t f = 1;
    FDM_CK(h, cudaMemcpyAsync(&f, flag, 4, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    *same = f == 0;
    return FDM_OK;
}

static int run_amr_impl(fdm_handle *h, fdm_handle *lead) {
    Nvtx range("fdm regrid");
    const int TB = 256;
    const int64_t NL = h->NL, NI = h->NI, NInt = h->NInt;
    if (h->p.window_rows != 0) {
        h->err = "a strip of a mesh takes no regrid: regrid the whole mesh";
        return FDM_ERR_UNSUPPORTED;
    }
    if ((int64_t)h->p.m * h->p.n >= (1ll << 19)) {
        h->err = "device regrid supports up to 2^19 background cells";
        return FDM_ERR_UNSUPPORTED;
    }
    for (int k = 0; k <= fdm_handle::AMR_PHASES; ++k)
        if (!h->amr_ev[k]) FDM_CK(h, cudaEventCreate(&h->amr_ev[k]));
    FDM_CK(h, cudaEventRecord(h->amr_ev[0], h->s));
    // 1. indicators and their ordered sums
    Carve ci;
    ci.add(NI * 8); ci.add(NI * 8); ci.add(32); ci.add(NL); ci.add((NInt > 0 ? NInt : 1));
    FDM_CK(h, h->amr[18].ensure(ci.total));
    double *rot = ci.at<double>(h->amr[18], 0), *div = ci.at<double>(h->amr[18], 1), *sums = ci.at<double>(h->amr[18], 2);
    int8_t *rflag = ci.at<int8_t>(h->amr[18], 3), *cflag = ci.at<int8_t>(h->amr[18], 4);
    if (lead) {
        bool same = false;
        AMR_RC(same_leaves(h, lead, &same));
        if (!same) {
            h->err = "the leader's leaf set differs from this handle's";
            return FDM_ERR_ARG;
        }
        const int rc = compute_rot_div(lead, rot, div, sums);
        if (rc) { h->err = "leader's indicators: " + lead->err; return rc; }
        FDM_CK(h, cudaStreamSynchronize(lead->s));
    } else {
        AMR_RC(compute_rot_div(h, rot, div, sums));
    }
    FDM_CK(h, cudaEventRecord(h->amr_ev[1], h->s));
    // 2. solute_ref: refine and coarsen flags, applied at once
    const Tables T = h->tables();
    k_refine_flags<<<nblk(NL, TB), TB, 0, h->s>>>(T, h->G, h->p, rot, div, sums, rflag);
    if (NInt > 0)
        k_coarsen_flags<<<nblk(NInt, TB), TB, 0, h->s>>>(NInt, h->ikey.as<uint64_t>(), T, h->p, rot, div, sums, rflag,
                                                        cflag);
    const int64_t nn = NL + NInt;
    FDM_CK(h, h->amr[19].ensure(nn * 8 + 16));
    int32_t *cnt = h->amr[19].as<int32_t>(), *off = cnt + nn;
    k_ref_count<<<nblk(nn, TB), TB, 0, h->s>>>(T, rflag, h->ikey.as<uint64_t>(), NInt, cflag, cnt);
    int64_t total = 0, split = 0;   // the leaves' entries (sorted) come first, then the internal nodes' (sorted)
    AMR_RC(scan_total32(h, cnt, off, nn, total, NL, &split));
    Emit E;
    AMR_RC(emit_buffers(h, total, E));
    k_ref_emit<<<nblk(nn, TB), TB, 0, h->s>>>(T, h->B[0].as<double4>(), rflag, h->ikey.as<uint64_t>(),
                                              h->ival.as<double4>(), NInt, cflag, off, E.key, E.leaf, E.val);
    AmrCtx X;
    X.h = h;
    AMR_RC(grow_nodes(h, X, total));
    bind_sets(h, X);
    merge_into(h, E.key, E.leaf, E.val, split, total, X.B);
    swap_sets(h, X);
    FDM_CK(h, cudaEventRecord(h->amr_ev[2], h->s));
    // 3. solute_gridmodify: lvlAMR rounds (src/solution.F90:537-556)
    // A round that changes nothing leaves the node set as it found it, so
    // the rounds after it would change nothing either.
    for (int k = 1; k <= h->p.lvl_amr; ++k) {
        bool did1 = false, did4 = false;
        AMR_RC(gridmodify1_pass(h, X, &did1));
        AMR_RC(gridmodify4_pass(h, X, &did4));
        if (!did1 && !did4) break;
    }
    FDM_CK(h, cudaEventRecord(h->amr_ev[3], h->s));
    // 4. split leaves / internal nodes, rebuild the tables (idneighbor + IDgrid)
    const int64_t n = X.A.n;
    Carve cs;
    cs.add(n * 4); cs.add(n * 4); cs.add(n * 4); cs.add(n * 4);
    FDM_CK(h, h->amr[8].ensure(cs.total));
    int32_t *fl = cs.at<int32_t>(h->amr[8], 0), *fi = cs.at<int32_t>(h->amr[8], 1);
    int32_t *ol = cs.at<int32_t>(h->amr[8], 2), *oi = cs.at<int32_t>(h->amr[8], 3);
    k_split_count<<<nblk(n, TB), TB, 0, h->s>>>(n, X.A.leaf, fl, fi);
    int64_t nleaf = 0, nint = 0;
    AMR_RC(scan_i32_only(h, fi, oi, n));
    AMR_RC(scan_total32(h, fl, ol, n, nleaf));
    nint = n - nleaf;   // every node is one or the other
    DevBuf &lk = h->amr[20], &lv = h->amr[21];   // kept between regrids
    FDM_CK(h, lk.ensure(nleaf * 8 + 8));
    FDM_CK(h, lv.ensure(nleaf * 32 + 32));
    FDM_CK(h, h->ikey.ensure(nint * 8 + 8));
    FDM_CK(h, h->ival.ensure(nint * 32 + 32));
    k_split_emit<<<nblk(n, TB), TB, 0, h->s>>>(X.A, ol, oi, lk.as<uint64_t>(), lv.as<double4>(),
                                               h->ikey.as<uint64_t>(), h->ival.as<double4>());
    FDM_CK(h, cudaEventRecord(h->amr_ev[4], h->s));
    h->NInt = nint;   // the rebuild is ordered after the split on the stream
    const int rc = build_tables(h, nleaf, lk.as<uint64_t>(), lv.as<double>(), 0);   // split keeps key order
    if (rc) return rc;
    FDM_CK(h, cudaEventRecord(h->amr_ev[5], h->s));
    FDM_CK(h, cudaEventSynchronize(h->amr_ev[5]));
    for (int k = 0; k < fdm_handle::AMR_PHASES; ++k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, h->amr_ev[k], h->amr_ev[k + 1]);
        h->amr_phase_ms[k] = t;
        h->amr_phase_total_ms[k] += t;
    }
    h->n_regrids++;
    return FDM_OK;
}

}  // namespace fdm

// Device-timeline milliseconds of the regrid phases: indicators and
// ordered sums, refine/coarsen flags and the first node sort, the lvlAMR
// gridmodify rounds, the leaf/internal split, the table rebuild; ms[0..4]
// for the last regrid, ms[5..9] summed over all regrids of the handle.
extern "C" int fdm_amr_phase_ms(const fdm_handle *h, double *ms) {
    if (!h || !ms) return FDM_ERR_ARG;
    for (int k = 0; k < fdm_handle::AMR_PHASES; ++k) {
        ms[k] = h->amr_phase_ms[k];
        ms[fdm_handle::AMR_PHASES + k] = h->amr_phase_total_ms[k];
    }
    return FDM_OK;
}

extern "C" int fdm_debug_rot_div(fdm_handle *h, int64_t cap, double *rot, double *div, double *sums) {
    using namespace fdm;
    if (!h) return FDM_ERR_ARG;
    if (!h->loaded) return FDM_ERR_STATE;
    if (cap < h->NI) return arg_fail(h, "capacity below the interior leaf count");
    DevBuf d;
    Carve cv;
    cv.add(h->NI * 8); cv.add(h->NI * 8); cv.add(3 * 8);
    FDM_CK(h, d.ensure(cv.total));
    double *dr = cv.at<double>(d, 0), *dd = cv.at<double>(d, 1), *ds = cv.at<double>(d, 2);
    int rc = compute_rot_div(h, dr, dd, ds);
    if (rc) return rc;
    if (rot) FDM_CK(h, cudaMemcpyAsync(rot, dr, h->NI * 8, cudaMemcpyDeviceToHost, h->s));
    if (div) FDM_CK(h, cudaMemcpyAsync(div, dd, h->NI * 8, cudaMemcpyDeviceToHost, h->s));
    if (sums) FDM_CK(h, cudaMemcpyAsync(sums, ds, 24, cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    d.release();
    return FDM_OK;
}

namespace fdm {
__global__ void k_interleave2(int64_t n, const double *__restrict__ a, const double *__restrict__ b, double2 *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_double2(a[i], b[i]);
}
}  // namespace fdm

extern "C" int fdm_debug_ordered_sum(const double *a, const double *b, int64_t n, double *sums) {
    using namespace fdm;
    if (!a || !b || !sums || n < 0 || n >= (1ll << 31)) return FDM_ERR_ARG;
    double *da = nullptr, *db = nullptr, *dout = nullptr;
    double2 *dq = nullptr;
    const size_t bytes = (size_t)(n > 0 ? n : 1) * 8;
    cudaError_t e = cudaMalloc(&da, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&db, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dq, 2 * bytes);
    if (e == cudaSuccess) e = cudaMalloc(&dout, 32);
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(da, a, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n > 0) e = cudaMemcpy(db, b, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (n > 0) k_interleave2<<<nblk(n, 256), 256>>>(n, da, db, dq);
        k_ordered_sums<<<2, OSUM_NT>>>(n, dq, dout);
        e = cudaGetLastError();
    }
    double out[3] = {0.0, 0.0, 0.0};
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, 24, cudaMemcpyDeviceToHost);
    cudaFree(da); cudaFree(db); cudaFree(dq); cudaFree(dout);
    if (e != cudaSuccess) return FDM_ERR_CUDA;
    sums[0] = out[0];
    sums[1] = out[1];
    return FDM_OK;
}
