// fdm_common.cuh — shared types of libfdm (device tables, request kinds,
// key/Morton helpers).  Everything here is plain data; the numerics live in
// numerics.cuh and the neighbour walks in topo.cuh.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/fdm.h"

#define FDM_HD __host__ __device__ __forceinline__

namespace fdm {

constexpr int LMAX = FDM_LMAX;
constexpr int MAXLVL_TAB = 16;   // per-level tables
constexpr int WLS_MAXM = 12;     // members of one WLS stencil (<= 9 in practice)

// Request kinds: values of the "virtual" stencil slots that a leaf cannot
// read directly from a same-level leaf (hanging nodes).
enum ReqKind : int32_t {
    RQ_WLS = 0,       // WLSI_US_WENO (src/XuanGua.F90:179-356)
    RQ_RESTRICT = 1,  // interpA over a subtree (src/XuanGua.F90:359-398)
    RQ_COPY = 2,      // child_value_weno fallback m<7: c%U (src/XuanGua.F90:143-144)
};

// Ghost fill kinds (body_boundary_RK, src/solution.F90:314-356, + extensions)
enum GhostKind : int32_t {
    GH_COPY = 0,      // image is a leaf
    GH_RESTRICT = 1,  // image is an internal node: interpA of its subtree
    GH_STATE = 2,     // fixed inflow state (extension)
    GH_DMR_TOP = 3,   // moving oblique shock (extension)
    GH_NONE = 4,      // corner or unsupported: never written
};

// Per-level constants (dx, dy and the derivative coefficients of
// LXL_X_wcns3 / LXL_Y_wcns3, src/nnd_center_RK.F90:109-110, 230).
struct LevelTab {
    double dx[MAXLVL_TAB], dy[MAXLVL_TAB];
    double cxa[MAXLVL_TAB], cxb[MAXLVL_TAB];   // 4/(3 dx), 1/(6 dx)
    double cya[MAXLVL_TAB], cyb[MAXLVL_TAB];   // (4/3)/dy, (1/6)/dy
    double dxdy[MAXLVL_TAB];                   // unused placeholder (fu*dx*dy is (fu*dx)*dy)
    double p15[MAXLVL_TAB];                    // dy**1.5 computed by the host libm
};

struct Geometry {
    double xmin, ymin, h, xf, gama, cv;
    int32_t m, n;              // root columns / rows held (n = the strip's rows)
    int32_t row0, nglob;       // global row of local row 0; rows of the whole mesh
    int32_t halo_lo, halo_hi;  // the strip's bottom / top three rows are a halo
};

// All device pointers of the current leaf set.  Passed by value to kernels.
struct Tables {
    // sorted leaves (key order), NL entries
    int64_t NL, NI, NG, NC, NR, NS;   // NS = NI+NG+NC+NR slots
    const uint64_t *lkey;
    const int32_t *lslot;             // sorted leaf -> slot
    const int32_t *slot_leaf;         // slot (< NI+NG+NC) -> sorted leaf
    const double *lcx, *lcy;          // leaf centres (sorted order)
    const int32_t *rfirst;            // [nroots + 1] first sorted leaf of each background cell
    int64_t nroots;                   // background cells (m * n)
    // interior leaves (slot order == key order of interior leaves)
    const int32_t *ist;               // [NI][8] stencil slots
    const uint8_t *ilvl;              // [NI]
    const int32_t *ifxl, *ifyl;       // [NI] index of the left/bottom face
    const int32_t *uxl, *uyl;         // unshared left faces -> owning leaf
    int64_t nux, nuy;                 // counts of unshared left faces
    // requests (virtual slots NI+NG+NC+r)
    const int32_t *rq_kind;           // [NR]
    const int32_t *rq_m;              // [NR][2]  (m1, m2) or (lo, hi) range
    const int32_t *rq_mem;            // [NR][WLS_MAXM] member slots
    const double *rq_geo;             // [NR][RQ_GEO] geometry block
    const uint64_t *rq_node;          // [NR] key of the node the value belongs to
    const int32_t *rq_rlist;          // [NRR] the requests of kind RQ_RESTRICT (interpA fallbacks)
    int64_t NRR;
    // ghosts (slots NI .. NI+NG)
    const int32_t *gh_kind;           // [NG]
    const int32_t *gh_a;              // [NG] source slot / range lo
    const int32_t *gh_b;              // [NG] range hi / state index
    const int32_t *gh_flip;           // [NG] 0 none, 1 negate u, 2 negate v
    const double *gh_x;               // [NG] ghost centre x (for DMR top)
    const double *gh_y;
};

// Layout of the per-request geometry block (doubles).
constexpr int G_XX = 0, G_YY = 1, G_BOX = 2;     // box: x_min, x_max, y_min, y_max
constexpr int G_X = 6;                            // x[WLS_MAXM]
constexpr int G_Y = G_X + WLS_MAXM;               // y[WLS_MAXM]
constexpr int G_W = G_Y + WLS_MAXM;               // w[WLS_MAXM]
constexpr int G_L = G_W + WLS_MAXM;               // inverse 6x6
constexpr int G_A = G_L + 36;                     // inverse 3x3 (axis points)
constexpr int G_B = G_A + 9;                      // inverse 3x3 (diagonal points)
constexpr int G_LVL = G_B + 9;                    // level (restrict) as double
constexpr int G_ORIGIN = G_LVL + 1;               // 0 parent_value_weno, 1 child_value_weno
constexpr int RQ_GEO = G_LVL + 2;                 // 96 doubles

// Device-side scalars of the time loop.
struct DevScalars {
    double lambda_x, lambda_y;   // monotone global maxima
    double tstep, tt, t_end;
    double res_max[4];
    double res_rms[4];
    double lam_next_x, lam_next_y;
    int64_t it;
    int32_t l_max;
    int32_t status;              // sticky: FDM_ERR_NAN when a NaN residual appeared
    int32_t done;                // tt >= t_end: further steps are no-ops
    int32_t pad;
};

// ------------------------------------------------------------ key helpers
FDM_HD uint32_t part1by1(uint32_t x) {
    x &= 0x0000ffffu;
    x = (x | (x << 8)) & 0x00ff00ffu;
    x = (x | (x << 4)) & 0x0f0f0f0fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}
FDM_HD uint32_t compact1by1(uint32_t x) {
    x &= 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0f0f0f0fu;
    x = (x | (x >> 4)) & 0x00ff00ffu;
    x = (x | (x >> 8)) & 0x0000ffffu;
    return x;
}
// Global Morton position of a key: root << 30 | path
FDM_HD uint64_t key_pos(uint64_t key) { return key >> 4; }
FDM_HD uint64_t span_of_level(int lvl) { return 1ull << (2 * (LMAX - lvl)); }

// A node of the (implicit) quadtree: background cell `root`, level and the
// local integer coordinates (ix, iy) in [0, 2^lvl).
struct Node {
    int64_t root;
    int32_t lvl;
    uint32_t ix, iy;
};
FDM_HD uint64_t node_pos(const Node &n) {
    const int s = LMAX - n.lvl;
    return ((uint64_t)n.root << 30) |
           (uint64_t)(part1by1(n.ix << s) | (part1by1(n.iy << s) << 1));
}
FDM_HD uint64_t node_key(const Node &n) { return (node_pos(n) << 4) | (uint64_t)n.lvl; }
FDM_HD Node node_of_key(uint64_t key) {
    Node n;
    n.root = (int64_t)(key >> 34);
    n.lvl = (int32_t)(key & 15u);
    const uint32_t path = (uint32_t)((key >> 4) & ((1ull << 30) - 1ull));
    const int s = LMAX - n.lvl;
    n.ix = compact1by1(path) >> s;
    n.iy = compact1by1(path >> 1) >> s;
    return n;
}
// child quadrant of a node inside its father: q = xbit | ybit << 1
FDM_HD int node_quadrant(const Node &n) { return (int)((n.ix & 1u) | ((n.iy & 1u) << 1)); }
// reference sp (src/mesh.F90:204-258): son1 SW, son2 SE, son3 NE, son4 NW
FDM_HD int quadrant_to_sp(int q) { return q == 0 ? 1 : q == 1 ? 2 : q == 3 ? 3 : 4; }

}  // namespace fdm
