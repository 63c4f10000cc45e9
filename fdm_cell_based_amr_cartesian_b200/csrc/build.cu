// build.cu — device construction of the leaf order, neighbour, stencil,
// hanging-node and ghost tables of a leaf set.
//
// Replaces, for the GPU path, what the reference rebuilds after every
// change of the tree: idneighbor (src/neighbor.F90:399-449), the leaf lists
// of IDgrid (src/solution.F90:593-693), and the per-call stencil search of
// parent_value_weno / child_value_weno / search_cell_5 / WLSI_US_WENO's
// geometry (src/XuanGua.F90:45-356), which the reference redoes inside
// every stage for every hanging face.
#include <cub/cub.cuh>

#include "handle.cuh"
#include "topo.cuh"

namespace fdm {

#define FDM_ATAN_BIAS 1.000000013351432e-10   /* REAL(4) 1e-10, src/XuanGua.F90:40 */
#define FDM_PI_REF 3.1415926535897932

enum BuildErr { BE_PARTITION = 0, BE_NULLNB = 1, BE_OVERFLOW = 2, BE_ROOT = 3, BE_LEVEL = 4, BE_INDEX = 5 };

static inline int nblk(int64_t n, int t) { return (int)((n + t - 1) / t); }

// get_direction (src/XuanGua.F90:33-43): 45-degree sector 1..8 (1 = east,
// counter-clockwise) of (xx,yy) seen from (x,y).
__device__ __noinline__ int get_direction_atan(double dx, double dy) {
    const double angle = (atan2(dy, dx) + FDM_ATAN_BIAS) * 180.0 / FDM_PI_REF;
    const int f = (int)floor((angle + 22.5) / 45.0 + 8);
    return ((f % 8) + 8) % 8 + 1;
}
// The sector follows from |dy| against tan(22.5) |dx| and tan(67.5) |dx|
// except next to a sector boundary: a relative margin of 1e-9 on the
// tangent keeps the point more than 3.5e-10 rad from the boundary, which
// is more than the 1e-10 rad shift of the bias plus the rounding of atan2
// and of the angle arithmetic, so the sector is the one the formula above
// gives; the points within the margin (and dx = dy = 0) take the formula.
__device__ __forceinline__ int get_direction(double xx, double yy, double x, double y) {
    const double dx = xx - x;
    const double dy = yy - y;
    const double a = fabs(dx), b = fabs(dy);
    constexpr double T1 = 0.41421356237309503, T2 = 2.414213562373095;   // tan(22.5), tan(67.5)
    constexpr double LO = 1.0 - 1e-9, HI = 1.0 + 1e-9;
    if (b < a * (T1 * LO)) return dx > 0.0 ? 1 : 5;
    if (b > a * (T2 * HI)) return dy > 0.0 ? 3 : 7;
    if (b > a * (T1 * HI) && b < a * (T2 * LO)) return dx > 0.0 ? (dy > 0.0 ? 2 : 8) : (dy > 0.0 ? 4 : 6);
    return get_direction_atan(dx, dy);
}

// ------------------------------------------------------------ classify
__global__ void k_classify(const uint64_t *__restrict__ lkey, int64_t NL, Geometry G,
                           int32_t *fI, int32_t *fG, int32_t *fC, int8_t *cross, int32_t *err) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    const int64_t total = (int64_t)G.m * G.n;
    const uint64_t key = lkey[k];
    const int lvl = (int)(key & 15u);
    const int64_t root = (int64_t)(key >> 34);
    const uint64_t pos = key_pos(key);
    if (root >= total) { atomicExch(err + BE_ROOT, 1); return; }
    if (lvl >= MAXLVL_TAB - 1) atomicExch(err + BE_LEVEL, 1);
    if (pos & (span_of_level(lvl) - 1)) atomicExch(err + BE_PARTITION, 1);
    const uint64_t prev_end = k == 0 ? 0ull : key_pos(lkey[k - 1]) + span_of_level((int)(lkey[k - 1] & 15u));
    if (pos != prev_end) atomicExch(err + BE_PARTITION, 1);
    if (k == NL - 1 && pos + span_of_level(lvl) != ((uint64_t)total << 30)) atomicExch(err + BE_PARTITION, 1);
    const int c = root_cross(G, root);
    cross[k] = (int8_t)c;
    // halo leaves of a strip take ghost slots (not advanced, not filled)
    const bool halo = root_in_halo(G, root);
    fI[k] = c == 0 && !halo;
    fC[k] = c == -5 && !halo;
    fG[k] = !fI[k] && !fC[k];
}

__global__ void k_slots(int64_t NL, int64_t NI, int64_t NG, const int32_t *fI, const int32_t *fG,
                        const int32_t *sI, const int32_t *sG, const int32_t *sC, int32_t *lslot,
                        int32_t *slot_leaf) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    const int32_t s = fI[k] ? sI[k] : fG[k] ? (int32_t)(NI + sG[k]) : (int32_t)(NI + NG + sC[k]);
    lslot[k] = s;
    slot_leaf[s] = (int32_t)k;
}

__global__ void k_scatter(int64_t NL, const int32_t *perm, const int32_t *lslot,
                          const double *__restrict__ prim, double4 *B0) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    const int64_t src = perm[k];
    B0[lslot[k]] = make_double4(prim[4 * src], prim[4 * src + 1], prim[4 * src + 2], prim[4 * src + 3]);
}

__global__ void k_centers(int64_t NL, const uint64_t *lkey, Geometry G, double *cx, double *cy) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k >= NL) return;
    double x, y;
    node_center(G, node_of_key(lkey[k]), x, y);
    cx[k] = x;
    cy[k] = y;
}

// ------------------------------------------------------- stencil resolve
// Tip/Tim/Tjp/Tjm and Tipp/Timm/Tjpp/Tjmm (src/XuanGua.F90:401-590):
// each of the 8 stencil entries of an interior leaf is either a same-level
// leaf (its slot) or a request: parent_value_weno on a same-level internal
// node, or child_value_weno on a coarser leaf at a target point.
struct ResolveOut {
    int32_t *slot;    // >= 0 direct slot, -1 request
    int32_t *kind;    // 0 parent, 1 child
    int64_t *ref;     // parent: node key; child: sorted leaf index
    double *tx, *ty;  // target point
};

__device__ __forceinline__ void target_point(const Geometry &G, double cx, double cy, int lvl, int dir,
                                             int k2, double &xx, double &yy) {
    if (k2 == 1) {
        switch (dir) {
            case DIR_RIGHT: xx = cx + G.xf * G.h / ipow2d(lvl); yy = cy; break;
            case DIR_LEFT: xx = cx - G.xf * G.h / ipow2d(lvl); yy = cy; break;
            case DIR_UP: xx = cx; yy = cy + G.h / ipow2d(lvl); break;
            default: xx = cx; yy = cy - G.h / ipow2d(lvl); break;
        }
    } else {
        switch (dir) {
            case DIR_RIGHT: xx = cx + 2.0 * G.xf * G.h / ipow2d(lvl); yy = cy; break;
            case DIR_LEFT: xx = cx - 2.0 * G.xf * G.h / ipow2d(lvl); yy = cy; break;
            case DIR_UP: xx = cx; yy = cy + 2.0 * G.h / ipow2d(lvl); break;
            default: xx = cx; yy = cy - 2.0 * G.h / ipow2d(lvl); break;
        }
    }
}

__global__ void k_resolve(Tables T, Geometry G, ResolveOut O, uint8_t *ilvl, int32_t *err) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int32_t k = T.slot_leaf[i];
    NodeRef c;
    c.n = node_of_key(T.lkey[k]);
    c.leaf = k;
    c.valid = 1;
    ilvl[i] = (uint8_t)c.n.lvl;
    const double cx = T.lcx[k], cy = T.lcy[k];
    const int dirs[4] = {DIR_RIGHT, DIR_LEFT, DIR_UP, DIR_DOWN};
    for (int q = 0; q < 4; ++q) {
        const int d = dirs[q];
        const NodeRef cn = face_nb(T, G, c, d);
        if (!cn.valid) { atomicExch(err + BE_NULLNB, 1); return; }
        // T1
        int64_t e = i * 8 + q;
        if (cn.n.lvl == c.n.lvl) {
            if (cn.leaf >= 0) O.slot[e] = T.lslot[cn.leaf];
            else { O.slot[e] = -1; O.kind[e] = 0; O.ref[e] = (int64_t)node_key(cn.n); }
        } else {
            O.slot[e] = -1; O.kind[e] = 1; O.ref[e] = cn.leaf;
            target_point(G, cx, cy, c.n.lvl, d, 1, O.tx[e], O.ty[e]);
        }
        // T2
        e = i * 8 + 4 + q;
        if (cn.n.lvl == c.n.lvl) {
            const NodeRef cnn = face_nb(T, G, cn, d);
            if (!cnn.valid) { atomicExch(err + BE_NULLNB, 1); return; }
            if (cnn.n.lvl == cn.n.lvl) {
                if (cnn.leaf >= 0) O.slot[e] = T.lslot[cnn.leaf];
                else { O.slot[e] = -1; O.kind[e] = 0; O.ref[e] = (int64_t)node_key(cnn.n); }
            } else {
                O.slot[e] = -1; O.kind[e] = 1; O.ref[e] = cnn.leaf;
                target_point(G, cx, cy, c.n.lvl, d, 2, O.tx[e], O.ty[e]);
            }
        } else {
            O.slot[e] = -1; O.kind[e] = 1; O.ref[e] = cn.leaf;
            target_point(G, cx, cy, c.n.lvl, d, 2, O.tx[e], O.ty[e]);
        }
    }
}

__global__ void k_req_flags(int64_t n, const int32_t *slot, int32_t *flag) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    flag[e] = slot[e] < 0;
}

struct ReqDesc {
    int32_t *kind;
    int64_t *ref;
    double *tx, *ty;
};

__global__ void k_emit(int64_t n, int64_t VS0, ResolveOut O, const int32_t *ridx, int32_t *ist, ReqDesc R) {
    const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int32_t s = O.slot[e];
    if (s >= 0) { ist[e] = s; return; }
    const int32_t r = ridx[e];
    ist[e] = (int32_t)(VS0 + r);
    R.kind[r] = O.kind[e];
    R.ref[r] = O.ref[e];
    R.tx[r] = O.tx[e];
    R.ty[r] = O.ty[e];
}

// ---------------------------------------------------------- WLS gather
struct Gather {
    int32_t m1, m2;
    int32_t n1[WLS_MAXM], n2[WLS_MAXM];  // sorted leaf indices
    bool used[8];
    int32_t overflow;
};

__device__ __forceinline__ void g_add(Gather &g, int32_t leaf, int dir) {
    g.used[dir - 1] = true;
    const bool axis = (dir == 1 || dir == 3 || dir == 5 || dir == 7);
    if (axis) {
        for (int t = 0; t < g.m1; ++t) if (g.n1[t] == leaf) return;
        if (g.m1 >= WLS_MAXM) { g.overflow = 1; return; }
        g.n1[g.m1++] = leaf;
    } else {
        for (int t = 0; t < g.m2; ++t) if (g.n2[t] == leaf) return;
        if (g.m2 >= WLS_MAXM) { g.overflow = 1; return; }
        g.n2[g.m2++] = leaf;
    }
}

// search_cell_5 (src/XuanGua.F90:152-177) on a node: its leaves in DFS
// order son1, son2, son3, son4; the first leaf of every still-unused
// sector joins the stencil.  The DFS rank of a leaf is its Morton path with
// each digit mapped 0,1,2,3 -> 0,1,3,2 (son1, son2, son4, son3).
__device__ void g_search(const Tables &T, const NodeRef &X, double x, double y, Gather &g) {
    if (!X.valid) return;
    if (X.leaf >= 0) {
        const int dir = get_direction(T.lcx[X.leaf], T.lcy[X.leaf], x, y);
        if (!g.used[dir - 1]) g_add(g, X.leaf, dir);
        return;
    }
    const uint64_t p0 = node_pos(X.n);
    const int64_t lo = lower_bound_pos_t(T, p0);
    const int64_t hi = lower_bound_pos_t(T, p0 + span_of_level(X.n.lvl));
    uint64_t best_rank[8];
    int32_t best_leaf[8];
    for (int s = 0; s < 8; ++s) { best_rank[s] = ~0ull; best_leaf[s] = -1; }
    for (int64_t k = lo; k < hi; ++k) {
        const int dir = get_direction(T.lcx[k], T.lcy[k], x, y);
        if (g.used[dir - 1]) continue;
        const uint64_t path = key_pos(T.lkey[k]) & ((1ull << 30) - 1ull);
        const uint64_t rank = path ^ ((path & 0x2AAAAAAAull) >> 1);
        if (rank < best_rank[dir - 1]) { best_rank[dir - 1] = rank; best_leaf[dir - 1] = (int32_t)k; }
    }
    for (;;) {
        int bs = -1;
        uint64_t br = ~0ull;
        for (int s = 0; s < 8; ++s)
            if (best_leaf[s] >= 0 && best_rank[s] < br) { br = best_rank[s]; bs = s; }
        if (bs < 0) break;
        g_add(g, best_leaf[bs], bs + 1);
        best_leaf[bs] = -1;
    }
}

// brinv (src/XuanGua.F90:593-660): full-pivot Gauss-Jordan in place;
// returns false on the singular test (the partially reduced matrix stays).
// The matrix lives in registers: every loop is unrolled, and the row and
// column exchanges with the pivot (whose indices are data) are selects over
// the rows and columns at or after the step, so the arithmetic is the
// reference's, operation for operation.
template <int N>
__device__ __forceinline__ void brinv_swap_rows(double (&r)[N][N], int k, int p) {
#pragma unroll
    for (int q = 0; q < N; ++q)
        if (q > k) {   // q == p > k: exchange rows k and q
#pragma unroll
            for (int j = 0; j < N; ++j) {
                const double a = r[k][j], b = r[q][j];
                const bool sw = q == p;
                r[k][j] = sw ? b : a;
                r[q][j] = sw ? a : b;
            }
        }
}
template <int N>
__device__ __forceinline__ void brinv_swap_cols(double (&r)[N][N], int k, int p) {
#pragma unroll
    for (int q = 0; q < N; ++q)
        if (q > k) {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double a = r[i][k], b = r[i][q];
                const bool sw = q == p;
                r[i][k] = sw ? b : a;
                r[i][q] = sw ? a : b;
            }
        }
}
template <int N>
__device__ __forceinline__ bool brinv_reg(double (&r)[N][N]) {
    int is[N], js[N];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        is[k] = 0; js[k] = 0;
        if (ok) {
            double d = 0.0;
            int pi = 0, pj = 0;
#pragma unroll
            for (int i = 0; i < N; ++i)
#pragma unroll
                for (int j = 0; j < N; ++j)
                    if (i >= k && j >= k && fabs(r[i][j]) > d) { d = fabs(r[i][j]); pi = i; pj = j; }
            is[k] = pi; js[k] = pj;
            if (d + 1.0 == 1.0) {
                ok = false;
            } else {
                brinv_swap_rows<N>(r, k, pi);
                brinv_swap_cols<N>(r, k, pj);
                r[k][k] = 1.0 / r[k][k];
#pragma unroll
                for (int j = 0; j < N; ++j) if (j != k) r[k][j] = r[k][j] * r[k][k];
#pragma unroll
                for (int i = 0; i < N; ++i)
                    if (i != k)
#pragma unroll
                        for (int j = 0; j < N; ++j)
                            if (j != k) r[i][j] = r[i][j] - r[i][k] * r[k][j];
#pragma unroll
                for (int i = 0; i < N; ++i) if (i != k) r[i][k] = -r[i][k] * r[k][k];
            }
        }
    }
    if (!ok) return false;
    // undo the exchanges: row k with row js[k], column k with column is[k]
#pragma unroll
    for (int k = N - 1; k >= 0; --k) {
        brinv_swap_rows<N>(r, k, js[k]);
        brinv_swap_cols<N>(r, k, is[k]);
    }
    return true;
}

struct ReqOut {
    int32_t *kind;
    int32_t *m;
    int32_t *mem;
    double *geo;
    uint64_t *node;
    unsigned long long *counts;   // [0] singular, [1] wls, [2] restrict, [3] copy
};

// One hanging-node request: stencil gather of parent_value_weno /
// child_value_weno (src/XuanGua.F90:45-150), then either the WLS geometry
// (P^T W P and its three brinv inverses, src/XuanGua.F90:206-255) or the
// reference's fallback when fewer than 7 points were found.
__global__ void k_gather(Tables T, Geometry G, ReqDesc D, ReqOut O, int32_t *err) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= T.NR) return;
    Gather g;
    g.m1 = 0; g.m2 = 0; g.overflow = 0;
    for (int s = 0; s < 8; ++s) g.used[s] = false;
    NodeRef c;
    double x, y, xx, yy;
    int32_t *mem = O.mem + r * WLS_MAXM;
    double *geo = O.geo + r * RQ_GEO;
    if (D.kind[r] == 0) {
        // parent_value_weno on the internal node
        c.n = node_of_key((uint64_t)D.ref[r]);
        c.leaf = -1;
        c.valid = 1;
        node_center(G, c.n, x, y);
        xx = x; yy = y;
        O.node[r] = node_key(c.n);
        geo[G_ORIGIN] = 0.0;
        geo[G_XX] = xx;
        geo[G_YY] = yy;
        const int qs[4] = {0, 1, 3, 2};
        for (int t = 0; t < 4; ++t) g_search(T, child_ref(T, c, qs[t]), x, y, g);
        if (g.m1 + g.m2 < 8) {
            g_search(T, face_nb(T, G, c, DIR_LEFT), x, y, g);
            g_search(T, face_nb(T, G, c, DIR_RIGHT), x, y, g);
            g_search(T, face_nb(T, G, c, DIR_DOWN), x, y, g);
            g_search(T, face_nb(T, G, c, DIR_UP), x, y, g);
        }
        if (g.m1 + g.m2 < 7) {
            const uint64_t p0 = node_pos(c.n);
            O.kind[r] = RQ_RESTRICT;
            O.m[2 * r] = (int32_t)lower_bound_pos_t(T, p0);
            O.m[2 * r + 1] = (int32_t)lower_bound_pos_t(T, p0 + span_of_level(c.n.lvl));
            geo[G_LVL] = (double)c.n.lvl;
            atomicAdd(O.counts + 2, 1ull);
            return;
        }
    } else {
        // child_value_weno on the coarse leaf at the target point
        const int32_t L = (int32_t)D.ref[r];
        c.n = node_of_key(T.lkey[L]);
        c.leaf = L;
        c.valid = 1;
        x = T.lcx[L]; y = T.lcy[L];
        xx = D.tx[r]; yy = D.ty[r];
        O.node[r] = T.lkey[L];
        geo[G_ORIGIN] = 1.0;
        geo[G_XX] = xx;
        geo[G_YY] = yy;
        g.n1[g.m1++] = L;
        const bool diag = root_cross(G, c.n.root) >= 0;
        const NodeRef nul = null_ref();
        g_search(T, diag ? downleft_nb(T, G, c) : nul, x, y, g);
        g_search(T, face_nb(T, G, c, DIR_LEFT), x, y, g);
        g_search(T, diag ? upleft_nb(T, G, c) : nul, x, y, g);
        g_search(T, face_nb(T, G, c, DIR_DOWN), x, y, g);
        g_search(T, face_nb(T, G, c, DIR_UP), x, y, g);
        g_search(T, diag ? downright_nb(T, G, c) : nul, x, y, g);
        g_search(T, face_nb(T, G, c, DIR_RIGHT), x, y, g);
        g_search(T, diag ? upright_nb(T, G, c) : nul, x, y, g);
        if (g.m1 + g.m2 < 7) {
            O.kind[r] = RQ_COPY;
            mem[0] = T.lslot[L];
            O.m[2 * r] = 1;
            O.m[2 * r + 1] = 0;
            atomicAdd(O.counts + 3, 1ull);
            return;
        }
    }
    if (g.overflow) atomicExch(err + BE_OVERFLOW, 1);
    // WLSI_US_WENO geometry
    const int m1 = g.m1, m2 = g.m2, m = m1 + m2;
    O.kind[r] = RQ_WLS;
    O.m[2 * r] = m1;
    O.m[2 * r + 1] = m2;
    double *gx = geo + G_X, *gy = geo + G_Y, *gw = geo + G_W;
    for (int i = 0; i < m; ++i) {
        const int32_t leaf = i < m1 ? g.n1[i] : g.n2[i - m1];
        mem[i] = T.lslot[leaf];
        const double xi = T.lcx[leaf], yi = T.lcy[leaf];
        gx[i] = xi;
        gy[i] = yi;
        const double d = sqrt((xi - xx) * (xi - xx) + (yi - yy) * (yi - yy));
        gw[i] = 1.0 / (d + 1.e-6);
    }
    geo[G_XX] = xx;
    geo[G_YY] = yy;
    double P[WLS_MAXM][6];
    for (int i = 0; i < m; ++i) {
        P[i][0] = 1.0; P[i][1] = gx[i]; P[i][2] = gy[i];
        P[i][3] = gx[i] * gy[i]; P[i][4] = gx[i] * gx[i]; P[i][5] = gy[i] * gy[i];
    }
    double *L = geo + G_L, *A = geo + G_A, *B = geo + G_B;
    unsigned long long ns = 0;
    {
        double R[6][6];
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = 0; b < 6; ++b) R[a][b] = 0.0;
        for (int i = 0; i < m; ++i) {
            const double pw[6] = {gw[i] * P[i][0], gw[i] * P[i][1], gw[i] * P[i][2],
                                  gw[i] * P[i][3], gw[i] * P[i][4], gw[i] * P[i][5]};
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int b = 0; b < 6; ++b) R[a][b] = R[a][b] + P[i][a] * pw[b];
        }
        if (!brinv_reg<6>(R)) ++ns;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = 0; b < 6; ++b) L[a * 6 + b] = R[a][b];
    }
    {
        double RA[3][3], RB[3][3];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) { RA[a][b] = 0.0; RB[a][b] = 0.0; }
        for (int i = 0; i < m1; ++i) {
            const double pw[3] = {gw[i] * P[i][0], gw[i] * P[i][1], gw[i] * P[i][2]};
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) RA[a][b] = RA[a][b] + P[i][a] * pw[b];
        }
        for (int i = m1; i < m; ++i) {
            const double pw[3] = {gw[i] * P[i][0], gw[i] * P[i][1], gw[i] * P[i][2]};
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) RB[a][b] = RB[a][b] + P[i][a] * pw[b];
        }
        if (!brinv_reg<3>(RA)) ++ns;
        if (!brinv_reg<3>(RB)) ++ns;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) { A[a * 3 + b] = RA[a][b]; B[a * 3 + b] = RB[a][b]; }
    }
    if (ns) atomicAdd(O.counts + 0, ns);
    atomicAdd(O.counts + 1, 1ull);
    // smoothness box of the node (compute_smoothness, src/XuanGua.F90:318-323)
    double ncx, ncy;
    node_center(G, c.n, ncx, ncy);
    if (c.leaf >= 0) { ncx = T.lcx[c.leaf]; ncy = T.lcy[c.leaf]; }
    const double hx = G.xf * G.h / ipow2d(c.n.lvl + 1);
    const double hy = G.h / ipow2d(c.n.lvl + 1);
    geo[G_BOX + 0] = ncx - hx;
    geo[G_BOX + 1] = ncx + hx;
    geo[G_BOX + 2] = ncy - hy;
    geo[G_BOX + 3] = ncy + hy;
}

// ------------------------------------------------------------- ghosts
struct GhostOut {
    int32_t *kind, *a, *b, *flip;
    double *x, *y;
    unsigned long long *n_restrict;   // ghosts imaged by a subtree restriction
};

__device__ __forceinline__ void ghost_from_ref(const Tables &T, const NodeRef &img, GhostOut &O, int64_t g) {
    if (img.leaf >= 0) {
        O.kind[g] = GH_COPY;
        O.a[g] = T.lslot[img.leaf];
        O.b[g] = 0;
    } else {
        const uint64_t p0 = node_pos(img.n);
        O.kind[g] = GH_RESTRICT;
        atomicAdd(O.n_restrict, 1ull);
        O.a[g] = (int32_t)lower_bound_pos_t(T, p0);
        O.b[g] = (int32_t)lower_bound_pos_t(T, p0 + span_of_level(img.n.lvl));
    }
}

// image node for the extension kinds: root (row1, col1) 1-based, descent along
// the ghost's path from the root with the quadrant bits transformed
// (mode 0 keep, 1 force x, 2 force y, 3 mirror y, 4 mirror x)
__device__ NodeRef ext_image(const Tables &T, const Geometry &G, const Node &gn, int row1, int col1,
                             int mode, int bit) {
    Node r0;
    r0.root = (int64_t)(row1 - 1) * G.m + (col1 - 1);
    r0.lvl = 0; r0.ix = 0; r0.iy = 0;
    NodeRef cur = resolve(T, r0);
    for (int j = 1; j <= gn.lvl; ++j) {
        if (cur.leaf >= 0) break;
        int q = (int)(((gn.ix >> (gn.lvl - j)) & 1u) | (((gn.iy >> (gn.lvl - j)) & 1u) << 1));
        if (mode == 1) q = (q & 2) | bit;
        else if (mode == 2) q = (q & 1) | (bit << 1);
        else if (mode == 3) q ^= 2;
        else if (mode == 4) q ^= 1;
        cur = child_ref(T, cur, q);
    }
    return cur;
}

__global__ void k_ghosts(Tables T, Geometry G, fdm_params P, GhostOut O) {
    const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= T.NG) return;
    const int32_t k = T.slot_leaf[T.NI + g];
    const Node gn = node_of_key(T.lkey[k]);
    if (root_in_halo(G, gn.root)) {   // written by the strip's caller
        O.kind[g] = GH_NONE; O.a[g] = 0; O.b[g] = 0; O.flip[g] = 0;
        O.x[g] = T.lcx[k]; O.y[g] = T.lcy[k];
        return;
    }
    const int a = root_cross(G, gn.root);
    const int row = (int)(gn.root / G.m) + 1, col = (int)(gn.root % G.m) + 1;
    const int m = G.m, n = G.n;
    int kind;
    if (a == -4) kind = P.kind_xmbc;
    else if (a == -2) kind = P.kind_xpbc;
    else if (a == -3) kind = P.kind_ypbc;
    else kind = P.kind_ymbc;
    O.flip[g] = 0;
    O.x[g] = T.lcx[k];
    O.y[g] = T.lcy[k];
    if (kind == FDM_BC_PERIODIC) {
        // BC_cyc (src/solution.F90:116-166): image root by index arithmetic,
        // descent along the ghost's sp list taken deepest level first
        const int num1 = row, num2 = col;
        int i1;
        if (a == -4) i1 = num1 * m + num2 - 6;
        else if (a == -2) i1 = num1 * m + num2 - 2 * m + 6;
        else if (a == -3) i1 = num1 * m + num2 - (n - 5) * m;
        else i1 = num1 * m + num2 - (7 - n) * m;
        Node r0;
        r0.root = i1 - 1; r0.lvl = 0; r0.ix = 0; r0.iy = 0;
        NodeRef cur = resolve(T, r0);
        for (int j = 0; j < gn.lvl; ++j) {
            if (cur.leaf >= 0) break;
            // sp(j+1) = sp of the ancestor j levels above the ghost
            const int l = gn.lvl - j;
            const int q = (int)(((gn.ix >> (gn.lvl - l)) & 1u) | (((gn.iy >> (gn.lvl - l)) & 1u) << 1));
            cur = child_ref(T, cur, q);
        }
        ghost_from_ref(T, cur, O, g);
        return;
    }
    if (kind == FDM_BC_TRANSMISSIVE) {
        NodeRef img;
        if (a == -4) img = ext_image(T, G, gn, row, 4, 1, 0);
        else if (a == -2) img = ext_image(T, G, gn, row, m - 3, 1, 1);
        else if (a == -1) img = ext_image(T, G, gn, 4, col, 2, 0);
        else img = ext_image(T, G, gn, n - 3, col, 2, 1);
        ghost_from_ref(T, img, O, g);
        return;
    }
    if (kind == FDM_BC_WALL || kind == FDM_BC_DMR_BOTTOM) {
        if (kind == FDM_BC_DMR_BOTTOM && T.lcx[k] <= P.dmr_x0) {
            O.kind[g] = GH_STATE; O.a[g] = 4; O.b[g] = 0;
            return;
        }
        NodeRef img;
        if (a == -1) img = ext_image(T, G, gn, 7 - row, col, 3, 0);
        else if (a == -3) img = ext_image(T, G, gn, 2 * n - 5 - row, col, 3, 0);
        else if (a == -4) img = ext_image(T, G, gn, row, 7 - col, 4, 0);
        else img = ext_image(T, G, gn, row, 2 * m - 5 - col, 4, 0);
        ghost_from_ref(T, img, O, g);
        O.flip[g] = (a == -1 || a == -3) ? 2 : 1;
        return;
    }
    if (kind == FDM_BC_INFLOW) {
        O.kind[g] = GH_STATE;
        O.a[g] = a == -4 ? 0 : a == -2 ? 1 : a == -1 ? 2 : 3;
        O.b[g] = 0;
        return;
    }
    if (kind == FDM_BC_DMR_TOP) {
        O.kind[g] = GH_DMR_TOP; O.a[g] = 0; O.b[g] = 0;
        return;
    }
    O.kind[g] = GH_NONE; O.a[g] = 0; O.b[g] = 0;
}

// --------------------------------------------------------------- faces
// The right (top) face of every interior leaf is face i.  Its left (bottom)
// face is the right face of the left neighbour j when j is an interior
// same-level leaf whose 4-point face stencil is slot-for-slot the same;
// otherwise the leaf owns a separate left face.
__global__ void k_face_flags(Tables T, int32_t *ux, int32_t *uy) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int32_t *s = T.ist + i * 8;
    int shared = 0;
    const int32_t j = s[1];
    if (j >= 0 && j < T.NI) {
        const int32_t *t = T.ist + (int64_t)j * 8;
        shared = (t[1] == s[5]) && (t[0] == (int32_t)i) && (t[4] == s[0]);
    }
    ux[i] = !shared;
    int shy = 0;
    const int32_t jy = s[3];
    if (jy >= 0 && jy < T.NI) {
        const int32_t *t = T.ist + (int64_t)jy * 8;
        shy = (t[3] == s[7]) && (t[2] == (int32_t)i) && (t[6] == s[2]);
    }
    uy[i] = !shy;
}
__global__ void k_face_assign(Tables T, const int32_t *ux, const int32_t *uy, const int32_t *sx,
                              const int32_t *sy, int32_t *ifxl, int32_t *ifyl, int32_t *uxl, int32_t *uyl) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= T.NI) return;
    const int32_t *s = T.ist + i * 8;
    if (ux[i]) { ifxl[i] = (int32_t)(T.NI + sx[i]); uxl[sx[i]] = (int32_t)i; }
    else ifxl[i] = s[1];
    if (uy[i]) { ifyl[i] = (int32_t)(T.NI + sy[i]); uyl[sy[i]] = (int32_t)i; }
    else ifyl[i] = s[3];
}

__global__ void k_lmax(int64_t NI, const uint8_t *ilvl, int32_t *out) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int v = i < NI ? (int)ilvl[i] : 0;
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, v);
}

// Every index a stage kernel will dereference is checked once here, so that
// no stage kernel can read or write outside its buffers.
// face_counts: the unshared left faces (nux, nuy) as the device counted them
__global__ void k_validate(Tables T, const int64_t *__restrict__ face_counts, int32_t *err) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    T.nux = face_counts[0];
    T.nuy = face_counts[1];
    const int64_t NLEAF = T.NI + T.NG + T.NC;
    bool bad = false;
    if (t < T.NI * 8) {
        const int32_t s = T.ist[t];
        bad |= s < 0 || s >= T.NS;
    }
    if (t < T.NI) {
        bad |= T.ifxl[t] < 0 || T.ifxl[t] >= T.NI + T.nux;
        bad |= T.ifyl[t] < 0 || T.ifyl[t] >= T.NI + T.nuy;
    }
    if (t < T.nux) bad |= T.uxl[t] < 0 || T.uxl[t] >= T.NI;
    if (t < T.nuy) bad |= T.uyl[t] < 0 || T.uyl[t] >= T.NI;
    if (t < T.NR) {
        const int k = T.rq_kind[t];
        const int32_t a = T.rq_m[2 * t], b = T.rq_m[2 * t + 1];
        const int32_t *mem = T.rq_mem + t * WLS_MAXM;
        if (k == RQ_WLS) {
            bad |= a < 0 || b < 0 || a + b > WLS_MAXM;
            if (!bad)
                for (int i = 0; i < a + b; ++i) bad |= mem[i] < 0 || mem[i] >= NLEAF;
        } else if (k == RQ_RESTRICT) {
            bad |= a < 0 || b <= a || b > T.NL;
        } else if (k == RQ_COPY) {
            bad |= mem[0] < 0 || mem[0] >= NLEAF;
        } else {
            bad = true;
        }
    }
    if (t < T.NG) {
        const int k = T.gh_kind[t];
        const int32_t a = T.gh_a[t], b = T.gh_b[t];
        if (k == GH_COPY) bad |= a < 0 || a >= NLEAF;
        else if (k == GH_RESTRICT) bad |= a < 0 || b <= a || b > T.NL;
        else if (k == GH_STATE) bad |= a < 0 || a >= 6;
        else if (k != GH_DMR_TOP && k != GH_NONE) bad = true;
    }
    if (bad) atomicExch(err + BE_INDEX, 1);
}

// ------------------------------------------------------------ host side
static int scan_i32(fdm_handle *h, const int32_t *in, int32_t *out, int64_t n) {
    size_t bytes = 0;
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, h->s));
    FDM_CK(h, h->cub_tmp.ensure(bytes));
    FDM_CK(h, cub::DeviceScan::ExclusiveSum(h->cub_tmp.p, bytes, in, out, (int)n, h->s));
    return FDM_OK;
}
// totals of exclusive scans, written on the device (read back later in one copy)
static __global__ void k_scan_total(const int32_t *__restrict__ flags, const int32_t *__restrict__ scan, int64_t n,
                             int64_t *out) {
    if (threadIdx.x == 0) *out = n > 0 ? (int64_t)flags[n - 1] + scan[n - 1] : 0;
}
static __global__ void k_iota_b(int64_t n, int32_t *a) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) a[i] = (int32_t)i;
}
// rf[r] = first sorted leaf of background cell r, rf[nroots] = n; cells
// without leaves (rejected later by the partition check) get the next
// cell's start; roots beyond the grid (rejected as well) are clamped
__global__ void k_root_first(int64_t n, const uint64_t *__restrict__ lkey, int64_t nroots, int32_t *rf) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > n) return;
    auto root = [&](int64_t k) -> int64_t {
        const int64_t r = (int64_t)(lkey[k] >> 34);
        return r < nroots ? r : nroots;
    };
    const int64_t prev = i == 0 ? -1 : root(i - 1);
    const int64_t cur = i == n ? nroots : root(i);
    for (int64_t x = prev + 1; x <= cur; ++x) rf[x] = (int32_t)i;
}
static __global__ void k_set_lmax(const int32_t *lmax, DevScalars *sc) {
    if (threadIdx.x == 0) sc->l_max = *lmax;
}
// the error flags and up to 6 totals in one read-back
static int read_back(fdm_handle *h, int32_t he[8], int64_t *tot, int nt) {
    FDM_CK(h, cudaMemcpyAsync(he, h->flag.p, 8 * sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
    if (nt > 0) FDM_CK(h, cudaMemcpyAsync(tot, h->tmp[7].p, nt * sizeof(int64_t), cudaMemcpyDeviceToHost, h->s));
    FDM_CK(h, cudaStreamSynchronize(h->s));
    return FDM_OK;
}

#define FDM_RC(x)                 \
    do {                          \
        int rc_ = (x);            \
        if (rc_) return rc_;      \
    } while (0)

__global__ void k_restrict_list(int64_t NR, const int32_t *__restrict__ kind, int32_t *list,
                                unsigned long long *count) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r < NR && kind[r] == RQ_RESTRICT) list[atomicAdd(count, 1ull)] = (int32_t)r;
}

int build_tables(fdm_handle *h, int64_t n, const uint64_t *keys_in, const double *prim_in, int key_bits) {
    Nvtx range("fdm tables");
    const int TB = 256;
    cudaStream_t s = h->s;
    if (n <= 0 || n >= (1ll << 31) - 1) return arg_fail(h, "leaf count out of range");
    h->NL = n;
    int32_t *err = h->flag.as<int32_t>();
    FDM_CK(h, cudaMemsetAsync(err, 0, 8 * sizeof(int32_t), s));
    // 1. sort keys, carrying the input index
    FDM_CK(h, h->lkey.ensure(n * 8));
    FDM_CK(h, h->tmp[0].ensure(n * 4));   // iota
    FDM_CK(h, h->tmp[1].ensure(n * 4));   // perm
    FDM_CK(h, h->tmp[7].ensure(6 * sizeof(int64_t)));
    int64_t *dtot = h->tmp[7].as<int64_t>();
    {
        int32_t *iota = h->tmp[0].as<int32_t>();
        if (key_bits <= 0) {
            k_iota_b<<<nblk(n, TB), TB, 0, s>>>(n, h->tmp[1].as<int32_t>());
            FDM_CK(h, cudaMemcpyAsync(h->lkey.as<uint64_t>(), keys_in, n * 8, cudaMemcpyDeviceToDevice, s));
        } else {
            k_iota_b<<<nblk(n, TB), TB, 0, s>>>(n, iota);
            size_t bytes = 0;
            FDM_CK(h, cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys_in, h->lkey.as<uint64_t>(), iota,
                                                      h->tmp[1].as<int32_t>(), (int)n, 0, key_bits, s));
            FDM_CK(h, h->cub_tmp.ensure(bytes));
            FDM_CK(h, cub::DeviceRadixSort::SortPairs(h->cub_tmp.p, bytes, keys_in, h->lkey.as<uint64_t>(), iota,
                                                      h->tmp[1].as<int32_t>(), (int)n, 0, key_bits, s));
        }
    }
    const uint64_t *lkey = h->lkey.as<uint64_t>();
    const int32_t *perm = h->tmp[1].as<int32_t>();
    {
        const int64_t nroots = (int64_t)h->G.m * h->G.n;
        FDM_CK(h, h->rfirst.ensure((nroots + 1) * 4));
        k_root_first<<<nblk(n + 1, TB), TB, 0, s>>>(n, lkey, nroots, h->rfirst.as<int32_t>());
    }
    // 2. classify + partition check
    Carve c2;
    for (int q = 0; q < 6; ++q) c2.add(n * 4);
    FDM_CK(h, h->tmp[2].ensure(c2.total));
    int32_t *fI = c2.at<int32_t>(h->tmp[2], 0), *fG = c2.at<int32_t>(h->tmp[2], 1), *fC = c2.at<int32_t>(h->tmp[2], 2);
    int32_t *sI = c2.at<int32_t>(h->tmp[2], 3), *sG = c2.at<int32_t>(h->tmp[2], 4), *sC = c2.at<int32_t>(h->tmp[2], 5);
    FDM_CK(h, h->lcross.ensure(n));
    k_classify<<<nblk(n, TB), TB, 0, s>>>(lkey, n, h->G, fI, fG, fC, h->lcross.as<int8_t>(), err);
    FDM_RC(scan_i32(h, fI, sI, n));
    FDM_RC(scan_i32(h, fG, sG, n));
    FDM_RC(scan_i32(h, fC, sC, n));
    int64_t NI, NG, NC;
    {
        k_scan_total<<<1, 32, 0, s>>>(fI, sI, n, dtot);
        k_scan_total<<<1, 32, 0, s>>>(fG, sG, n, dtot + 1);
        k_scan_total<<<1, 32, 0, s>>>(fC, sC, n, dtot + 2);
        int32_t he[8];
        int64_t tot[3];
        FDM_RC(read_back(h, he, tot, 3));
        NI = tot[0]; NG = tot[1]; NC = tot[2];
        if (he[BE_ROOT]) return arg_fail(h, "leaf key names a background cell outside the m x n grid");
        if (he[BE_PARTITION]) return arg_fail(h, "leaf set does not partition the background grid (gap, overlap or duplicate)");
        if (he[BE_LEVEL]) return arg_fail(h, "leaf level above the supported maximum (14)");
    }
    if (NI == 0) return arg_fail(h, "no interior leaves");
    h->NI = NI; h->NG = NG; h->NC = NC;
    // 3. slots, values, centres
    FDM_CK(h, h->lslot.ensure(n * 4));
    FDM_CK(h, h->slot_leaf.ensure(n * 4));
    k_slots<<<nblk(n, TB), TB, 0, s>>>(n, NI, NG, fI, fG, sI, sG, sC, h->lslot.as<int32_t>(), h->slot_leaf.as<int32_t>());
    FDM_CK(h, h->lcx.ensure(n * 8));
    FDM_CK(h, h->lcy.ensure(n * 8));
    k_centers<<<nblk(n, TB), TB, 0, s>>>(n, lkey, h->G, h->lcx.as<double>(), h->lcy.as<double>());
    // 4. stencil resolution
    const int64_t ne = NI * 8;
    FDM_CK(h, h->ist.ensure(ne * 4));
    FDM_CK(h, h->ilvl.ensure(NI));
    Carve c3;
    c3.add(ne * 4); c3.add(ne * 4); c3.add(ne * 8); c3.add(ne * 8); c3.add(ne * 8); c3.add(ne * 4); c3.add(ne * 4);
    FDM_CK(h, h->tmp[3].ensure(c3.total));
    ResolveOut RO;
    RO.slot = c3.at<int32_t>(h->tmp[3], 0);
    RO.kind = c3.at<int32_t>(h->tmp[3], 1);
    RO.ref = c3.at<int64_t>(h->tmp[3], 2);
    RO.tx = c3.at<double>(h->tmp[3], 3);
    RO.ty = c3.at<double>(h->tmp[3], 4);
    int32_t *rflag = c3.at<int32_t>(h->tmp[3], 5);
    int32_t *ridx = c3.at<int32_t>(h->tmp[3], 6);
    {
        Tables T = h->tables();
        k_resolve<<<nblk(NI, 128), 128, 0, s>>>(T, h->G, RO, h->ilvl.as<uint8_t>(), err);
    }
    k_req_flags<<<nblk(ne, TB), TB, 0, s>>>(ne, RO.slot, rflag);
    FDM_RC(scan_i32(h, rflag, ridx, ne));
    int64_t NR;
    {
        k_scan_total<<<1, 32, 0, s>>>(rflag, ridx, ne, dtot);
        int32_t he[8];
        FDM_RC(read_back(h, he, &NR, 1));
        if (he[BE_NULLNB]) return arg_fail(h, "an interior leaf has a null stencil neighbour (fewer than 3 ghost layers?)");
    }
    h->NR = NR;
    h->NS = NI + NG + NC + NR;
    const int64_t VS0 = NI + NG + NC;
    const int64_t nrq = NR > 0 ? NR : 1;
    Carve c4;
    c4.add(nrq * 4); c4.add(nrq * 8); c4.add(nrq * 8); c4.add(nrq * 8);
    FDM_CK(h, h->tmp[4].ensure(c4.total));
    ReqDesc RD;
    RD.kind = c4.at<int32_t>(h->tmp[4], 0);
    RD.ref = c4.at<int64_t>(h->tmp[4], 1);
    RD.tx = c4.at<double>(h->tmp[4], 2);
    RD.ty = c4.at<double>(h->tmp[4], 3);
    k_emit<<<nblk(ne, TB), TB, 0, s>>>(ne, VS0, RO, ridx, h->ist.as<int32_t>(), RD);
    // 5. requests: gather + WLS geometry
    FDM_CK(h, h->rq_kind.ensure(nrq * 4));
    FDM_CK(h, h->rq_m.ensure(nrq * 8));
    FDM_CK(h, h->rq_mem.ensure(nrq * WLS_MAXM * 4));
    FDM_CK(h, h->rq_geo.ensure(nrq * RQ_GEO * 8));
    FDM_CK(h, h->rq_node.ensure(nrq * 8));
    FDM_CK(h, h->tmp[5].ensure(64));
    unsigned long long *counts = h->tmp[5].as<unsigned long long>();
    FDM_CK(h, cudaMemsetAsync(counts, 0, 64, s));
    if (NR > 0) {
        Tables T = h->tables();
        ReqOut O{h->rq_kind.as<int32_t>(), h->rq_m.as<int32_t>(), h->rq_mem.as<int32_t>(),
                 h->rq_geo.as<double>(), h->rq_node.as<uint64_t>(), counts};
        k_gather<<<nblk(NR, 64), 64, 0, s>>>(T, h->G, RD, O, err);
    }
    // the interpA fallbacks among the requests, listed (in no particular
    // order: each writes only its own value), so that their warps are
    // launched for them alone
    FDM_CK(h, h->rq_rlist.ensure((NR > 0 ? NR : 1) * 4));
    if (NR > 0)
        k_restrict_list<<<nblk(NR, TB), TB, 0, s>>>(NR, h->rq_kind.as<int32_t>(), h->rq_rlist.as<int32_t>(),
                                                    counts + 6);
    // 6. ghosts
    const int64_t ngh = NG > 0 ? NG : 1;
    FDM_CK(h, h->gh_kind.ensure(ngh * 4));
    FDM_CK(h, h->gh_a.ensure(ngh * 4));
    FDM_CK(h, h->gh_b.ensure(ngh * 4));
    FDM_CK(h, h->gh_flip.ensure(ngh * 4));
    FDM_CK(h, h->gh_x.ensure(ngh * 8));
    FDM_CK(h, h->gh_y.ensure(ngh * 8));
    if (NG > 0) {
        Tables T = h->tables();
        GhostOut O{h->gh_kind.as<int32_t>(), h->gh_a.as<int32_t>(), h->gh_b.as<int32_t>(),
                   h->gh_flip.as<int32_t>(), h->gh_x.as<double>(),  h->gh_y.as<double>(),
                   h->tmp[5].as<unsigned long long>() + 4};
        k_ghosts<<<nblk(NG, 128), 128, 0, s>>>(T, h->G, h->p, O);
    }
    // 7. faces
    Carve c6;
    for (int q = 0; q < 4; ++q) c6.add(NI * 4);
    FDM_CK(h, h->tmp[6].ensure(c6.total));
    int32_t *ux = c6.at<int32_t>(h->tmp[6], 0), *uy = c6.at<int32_t>(h->tmp[6], 1);
    int32_t *sx = c6.at<int32_t>(h->tmp[6], 2), *sy = c6.at<int32_t>(h->tmp[6], 3);
    {
        Tables T = h->tables();
        k_face_flags<<<nblk(NI, TB), TB, 0, s>>>(T, ux, uy);
    }
    FDM_RC(scan_i32(h, ux, sx, NI));
    FDM_RC(scan_i32(h, uy, sy, NI));
    // the face counts come back with the final checks; until then the
    // buffers take their bound (at most one unshared left face per leaf)
    k_scan_total<<<1, 32, 0, s>>>(ux, sx, NI, dtot + 4);
    k_scan_total<<<1, 32, 0, s>>>(uy, sy, NI, dtot + 5);
    const int64_t nux_max = NI, nuy_max = NI;
    FDM_CK(h, h->ifxl.ensure(NI * 4));
    FDM_CK(h, h->ifyl.ensure(NI * 4));
    FDM_CK(h, h->uxl.ensure(nux_max * 4));
    FDM_CK(h, h->uyl.ensure(nuy_max * 4));
    {
        Tables T = h->tables();
        k_face_assign<<<nblk(NI, TB), TB, 0, s>>>(T, ux, uy, sx, sy, h->ifxl.as<int32_t>(), h->ifyl.as<int32_t>(),
                                                  h->uxl.as<int32_t>(), h->uyl.as<int32_t>());
    }
    // 8. state buffers (corner values copied into all three)
    const int64_t NS = h->NS;
    for (int b = 0; b < 3; ++b) FDM_CK(h, h->B[b].ensure(NS * 32));
    FDM_CK(h, h->Fx.ensure((NI + nux_max) * 32));
    FDM_CK(h, h->Fy.ensure((NI + nuy_max) * 32));
    FDM_CK(h, h->Ut.ensure(NI * 32));
    k_scatter<<<nblk(n, TB), TB, 0, s>>>(n, perm, h->lslot.as<int32_t>(), prim_in, h->B[0].as<double4>());
    if (NC > 0)
        for (int b = 1; b < 3; ++b)
            FDM_CK(h, cudaMemcpyAsync(h->B[b].as<double4>() + NI + NG, h->B[0].as<double4>() + NI + NG, NC * 32,
                                      cudaMemcpyDeviceToDevice, s));
    // 9. index validation of every table the stage kernels use
    {
        Tables T = h->tables();
        int64_t nv = NI * 8;
        const int64_t others[5] = {nux_max, nuy_max, NR, NG, NI};
        for (int q = 0; q < 5; ++q) nv = nv > others[q] ? nv : others[q];
        k_validate<<<nblk(nv, TB), TB, 0, s>>>(T, dtot + 4, err);
    }
    // 10. l_max
    int32_t *dl = err + 7;
    FDM_CK(h, cudaMemsetAsync(dl, 0, 4, s));
    k_lmax<<<nblk(NI, TB), TB, 0, s>>>(NI, h->ilvl.as<uint8_t>(), dl);
    k_set_lmax<<<1, 32, 0, s>>>(dl, h->scal.as<DevScalars>());
    int32_t he[8];
    unsigned long long hc[7];
    FDM_CK(h, cudaMemcpyAsync(he, err, sizeof(he), cudaMemcpyDeviceToHost, s));
    FDM_CK(h, cudaMemcpyAsync(hc, counts, sizeof(hc), cudaMemcpyDeviceToHost, s));
    int64_t fc[2] = {0, 0};
    FDM_CK(h, cudaMemcpyAsync(fc, dtot + 4, sizeof(fc), cudaMemcpyDeviceToHost, s));
    FDM_CK(h, cudaStreamSynchronize(s));
    FDM_CK(h, cudaGetLastError());
    h->nux = fc[0];
    h->nuy = fc[1];
    if (hc[2] != hc[6]) return arg_fail(h, "internal table check failed: restrict list");
    if (he[BE_OVERFLOW]) return arg_fail(h, "hanging-node stencil larger than supported");
    if (he[BE_INDEX]) return arg_fail(h, "internal table check failed: an index is out of range");
    h->l_max = he[7];
    h->n_singular += (int64_t)hc[0];
    h->n_restrict = (int64_t)hc[2];
    h->n_ghost_restrict = (int64_t)hc[4];
    h->table_version++;
    h->gate_stage1_valid = false;
    h->lam_fresh = false;
    h->cur_buf = 0;
    h->loaded = true;
    return FDM_OK;
}

}  // namespace fdm
