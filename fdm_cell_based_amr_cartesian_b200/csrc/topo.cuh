// topo.cuh — the quadtree as a sorted array of leaf keys.
//
// The reference keeps a pointer tree and caches eight neighbour pointers per
// node (idnei, src/neighbor.F90:412-449).  Here a node is named by
// (root, lvl, ix, iy); whether it exists, is a leaf or is internal follows
// from one binary search for the leaf that contains its lower-left corner
// in the Morton-sorted leaf array.  The functions below return exactly what
// the reference's recursive walks return (a same-level node, which may be
// internal, or the coarser leaf that covers it; null across the edge of the
// background grid), and the diagonal walks reproduce the reference's
// sp-dependent rules one for one.
#pragma once
#include "fdm_common.cuh"

namespace fdm {

struct NodeRef {
    Node n;
    int32_t leaf;   // sorted leaf index, or -1 if the node is internal
    int32_t valid;  // 0 = null pointer
};

FDM_HD NodeRef null_ref() {
    NodeRef r;
    r.n.root = 0; r.n.lvl = 0; r.n.ix = 0; r.n.iy = 0;
    r.leaf = -1; r.valid = 0;
    return r;
}

// largest k with key_pos(lkey[k]) <= pos
__device__ __forceinline__ int64_t find_leaf(const uint64_t *__restrict__ lkey, int64_t NL,
                                             uint64_t pos) {
    int64_t lo = 0, hi = NL - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (key_pos(__ldg(lkey + mid)) <= pos) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
// first k with key_pos(lkey[k]) >= pos
__device__ __forceinline__ int64_t lower_bound_pos(const uint64_t *__restrict__ lkey, int64_t NL,
                                                   uint64_t pos) {
    int64_t lo = 0, hi = NL;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (key_pos(__ldg(lkey + mid)) < pos) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// rf[r] = first index of background cell r in a key-sorted array (leaves or
// nodes), rf[nroots] = n (build.cu)
__global__ void k_root_first(int64_t n, const uint64_t *__restrict__ lkey, int64_t nroots, int32_t *rf);

// The same two searches confined to the leaves of the position's background
// cell (pos >> 30), which the per-cell index T.rfirst delimits: the sorted
// leaves of cell r are [rfirst[r], rfirst[r + 1]), and a leaf set that
// partitions the grid gives every cell at least one leaf, the first of which
// starts at the cell's corner.  About 8 dependent loads instead of 17 on a
// 140k-leaf mesh.
__device__ __forceinline__ int64_t find_leaf_t(const Tables &T, uint64_t pos) {
    const int64_t r = (int64_t)(pos >> 30);
    if (!T.rfirst || r >= T.nroots) return find_leaf(T.lkey, T.NL, pos);
    int64_t lo = __ldg(T.rfirst + r), hi = (int64_t)__ldg(T.rfirst + r + 1) - 1;
    if (lo > hi) return find_leaf(T.lkey, T.NL, pos);
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (key_pos(__ldg(T.lkey + mid)) <= pos) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int64_t lower_bound_pos_t(const Tables &T, uint64_t pos) {
    const int64_t r = (int64_t)(pos >> 30);
    if (!T.rfirst) return lower_bound_pos(T.lkey, T.NL, pos);
    if (r >= T.nroots) return T.NL;
    int64_t lo = __ldg(T.rfirst + r), hi = __ldg(T.rfirst + r + 1);
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (key_pos(__ldg(T.lkey + mid)) < pos) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ NodeRef resolve(const Tables &T, const Node &n) {
    const int64_t f = find_leaf_t(T, node_pos(n));
    const uint64_t k = __ldg(T.lkey + f);
    NodeRef r;
    r.valid = 1;
    if ((int)(k & 15u) <= n.lvl) {
        r.n = node_of_key(k);
        r.leaf = (int32_t)f;
    } else {
        r.n = n;
        r.leaf = -1;
    }
    return r;
}

enum Dir { DIR_UP = 0, DIR_DOWN = 1, DIR_RIGHT = 2, DIR_LEFT = 3 };

// up/down/right/left_neighbor (src/neighbor.F90:65-196) in closed form
__device__ __forceinline__ NodeRef face_nb(const Tables &T, const Geometry &G, const NodeRef &x,
                                           int dir) {
    if (!x.valid) return null_ref();
    Node n = x.n;
    int64_t row = n.root / G.m, col = n.root % G.m;
    const uint32_t N = 1u << n.lvl;
    switch (dir) {
        case DIR_UP:
            if (n.iy + 1 == N) { if (row + 1 >= G.n) return null_ref(); ++row; n.iy = 0; }
            else ++n.iy;
            break;
        case DIR_DOWN:
            if (n.iy == 0) { if (row == 0) return null_ref(); --row; n.iy = N - 1; }
            else --n.iy;
            break;
        case DIR_RIGHT:
            if (n.ix + 1 == N) { if (col + 1 >= G.m) return null_ref(); ++col; n.ix = 0; }
            else ++n.ix;
            break;
        default:
            if (n.ix == 0) { if (col == 0) return null_ref(); --col; n.ix = N - 1; }
            else --n.ix;
            break;
    }
    n.root = row * G.m + col;
    return resolve(T, n);
}

// son with quadrant q of an internal node
__device__ __forceinline__ NodeRef child_ref(const Tables &T, const NodeRef &x, int q) {
    Node c;
    c.root = x.n.root;
    c.lvl = x.n.lvl + 1;
    c.ix = 2u * x.n.ix + (uint32_t)(q & 1);
    c.iy = 2u * x.n.iy + (uint32_t)(q >> 1);
    return resolve(T, c);
}
// sibling with quadrant q (father%sonX)
__device__ __forceinline__ NodeRef sibling_ref(const Tables &T, const NodeRef &x, int q) {
    Node c = x.n;
    c.ix = (c.ix & ~1u) | (uint32_t)(q & 1);
    c.iy = (c.iy & ~1u) | (uint32_t)(q >> 1);
    return resolve(T, c);
}

// Diagonal walks, src/neighbor.F90:199-396.  q codes: son1 = 0, son2 = 1,
// son3 = 3, son4 = 2.
__device__ __forceinline__ NodeRef descend_while(const Tables &T, NodeRef r, int lvl, int q) {
    while (r.valid && r.n.lvl < lvl && r.leaf < 0) r = child_ref(T, r, q);
    return r;
}

__device__ inline NodeRef upleft_nb(const Tables &T, const Geometry &G, const NodeRef &c) {
    const NodeRef celln = face_nb(T, G, c, DIR_LEFT), cellfn = face_nb(T, G, c, DIR_UP);
    if (c.n.lvl == 0) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return face_nb(T, G, celln, DIR_UP);
    }
    const int sp = quadrant_to_sp(node_quadrant(c.n));
    if (sp == 2) return sibling_ref(T, c, 2);
    if (sp == 4) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return descend_while(T, face_nb(T, G, celln, DIR_UP), c.n.lvl, 1);
    }
    if (sp == 1) {
        if (!celln.valid || celln.n.lvl < c.n.lvl) return null_ref();
        return face_nb(T, G, celln, DIR_UP);
    }
    if (!cellfn.valid || cellfn.n.lvl < c.n.lvl) return null_ref();
    return face_nb(T, G, cellfn, DIR_LEFT);
}
__device__ inline NodeRef upright_nb(const Tables &T, const Geometry &G, const NodeRef &c) {
    const NodeRef celln = face_nb(T, G, c, DIR_RIGHT), cellfn = face_nb(T, G, c, DIR_UP);
    if (c.n.lvl == 0) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return face_nb(T, G, celln, DIR_UP);
    }
    const int sp = quadrant_to_sp(node_quadrant(c.n));
    if (sp == 1) return sibling_ref(T, c, 3);
    if (sp == 3) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return descend_while(T, face_nb(T, G, celln, DIR_UP), c.n.lvl, 0);
    }
    if (sp == 2) {
        if (!celln.valid || celln.n.lvl < c.n.lvl) return null_ref();
        return face_nb(T, G, celln, DIR_UP);
    }
    if (!cellfn.valid || cellfn.n.lvl < c.n.lvl) return null_ref();
    return face_nb(T, G, cellfn, DIR_RIGHT);
}
__device__ inline NodeRef downright_nb(const Tables &T, const Geometry &G, const NodeRef &c) {
    const NodeRef celln = face_nb(T, G, c, DIR_RIGHT), cellfn = face_nb(T, G, c, DIR_DOWN);
    if (c.n.lvl == 0) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return face_nb(T, G, celln, DIR_DOWN);
    }
    const int sp = quadrant_to_sp(node_quadrant(c.n));
    if (sp == 4) return sibling_ref(T, c, 1);
    if (sp == 2) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return descend_while(T, face_nb(T, G, celln, DIR_DOWN), c.n.lvl, 2);
    }
    if (sp == 3) {
        if (!celln.valid || celln.n.lvl < c.n.lvl) return null_ref();
        return face_nb(T, G, celln, DIR_DOWN);
    }
    if (!cellfn.valid || cellfn.n.lvl < c.n.lvl) return null_ref();
    return face_nb(T, G, cellfn, DIR_RIGHT);
}
__device__ inline NodeRef downleft_nb(const Tables &T, const Geometry &G, const NodeRef &c) {
    const NodeRef celln = face_nb(T, G, c, DIR_LEFT), cellfn = face_nb(T, G, c, DIR_DOWN);
    if (c.n.lvl == 0) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return face_nb(T, G, celln, DIR_DOWN);
    }
    const int sp = quadrant_to_sp(node_quadrant(c.n));
    if (sp == 3) return sibling_ref(T, c, 0);
    if (sp == 1) {
        if (!celln.valid || !cellfn.valid) return null_ref();
        return descend_while(T, face_nb(T, G, celln, DIR_DOWN), c.n.lvl, 3);
    }
    if (sp == 4) {
        if (!celln.valid || celln.n.lvl < c.n.lvl) return null_ref();
        return face_nb(T, G, celln, DIR_DOWN);
    }
    if (!cellfn.valid || cellfn.n.lvl < c.n.lvl) return null_ref();
    return face_nb(T, G, cellfn, DIR_LEFT);
}

// gridcross (src/mesh.F90:89-142) from the background cell of a node
// The class is that of the root in the whole mesh (global row), also for a
// strip of it.
FDM_HD int root_cross(const Geometry &G, int64_t root) {
    const int r = (int)(root / G.m) + 1 + G.row0, q = (int)(root % G.m) + 1;
    const int m = G.m, n = G.nglob;
    if ((r < 4 && q < 4) || (r < 4 && q > m - 3) || (r > n - 3 && q > m - 3) || (r > n - 3 && q < 4))
        return -5;
    if (r < 4) return -1;
    if (r > n - 3) return -3;
    if (q > m - 3) return -2;
    if (q < 4) return -4;
    return 0;
}

// A root in one of the three halo rows of a strip (filled by the caller).
FDM_HD bool root_in_halo(const Geometry &G, int64_t root) {
    const int r = (int)(root / G.m);
    return (G.halo_lo && r < 3) || (G.halo_hi && r >= G.n - 3);
}

FDM_HD double ipow2d(int l) { return (double)(1ll << l); }

// Node centre by the same chain of operations as creat_mesh + Refine_cell
// (src/mesh.F90:25-26, 205-248).
FDM_HD void node_center(const Geometry &G, const Node &n, double &cx, double &cy) {
    const int64_t row = n.root / G.m + G.row0, col = n.root % G.m;
    const double nj = (double)(col + 1), ni = (double)(row + 1);
    cx = 0.5 * (2.0 * nj - 1.0) * G.xf * G.h + G.xmin;
    cy = (ni - 0.5) * G.h + G.ymin;
    for (int k = 1; k <= n.lvl; ++k) {
        const uint32_t xb = (n.ix >> (n.lvl - k)) & 1u, yb = (n.iy >> (n.lvl - k)) & 1u;
        const double qx = G.xf * G.h / ipow2d(k + 1);
        const double qy = G.h / ipow2d(k + 1);
        cx = xb ? cx + qx : cx - qx;
        cy = yb ? cy + qy : cy - qy;
    }
}

}  // namespace fdm
