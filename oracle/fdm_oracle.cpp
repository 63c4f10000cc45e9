/*
 * fdm_oracle.cpp — TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the reference solver Jian-cd/FDM-cell-based-AMR-Cartesian
 * (Fortran 90 sources under src/), written line by line from the reference sources.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it, as the checker and the timed CPU baseline; the product (libfdm) never
 * links or calls it.
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or fixtures,
 * and it is Fortran-only while this image has no Fortran compiler, so its own
 * outputs cannot be produced here.  This restatement is checked instead
 * against analytic known answers (linear reproduction of WCNS_Z3, R*Rinv = I,
 * brinv vs an LU inverse, quadratic reproduction of the WLS fit, uniform-flow
 * preservation, the exact isentropic vortex) and against an independent
 * Python transliteration of the numerics (tests/test_oracle_*.py).
 *
 * Semantics fixed here (the original build flags are unknown):
 *  - source evaluation order, left to right; no FMA contraction
 *    (-ffp-contract=off); every sum of an intrinsic MATMUL/SUM starts at 0.0
 *    and runs over the inner index ascending;
 *  - default-REAL(4) literals are promoted as the Fortran does
 *    (1.e-40 -> 9.99994610111476e-41, 1./11., 10./11., 1e-10 in
 *    get_direction, gama = 1.4 passed in promoted by the caller);
 *  - the racy OpenMP max of lambda_x/lambda_y (src/solution.F90:186-193) is
 *    taken race-free; Res_rms is summed in leaf-list order;
 *  - search_cell_5's `do i=1,4` repetition (src/XuanGua.F90:170-175) is
 *    walked once: after the first pass every sector of every leaf in the
 *    subtree is marked used, so the repeats can add nothing;
 *  - var(4) (T) of a WLS result is left undefined by the reference
 *    (src/XuanGua.F90:257-307); here it is set to NaN, which proves that
 *    the residual never reads it.
 * Extensions with no reference counterpart (marked EXT below): transmissive,
 * reflecting-wall, inflow and double-Mach boundary kinds; four-quadrant and
 * double-Mach initial states.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/fdm.h"

namespace orc {

constexpr int NVAR = 9;
constexpr int BCcorner = -5;
constexpr double Pi = 3.1415926535897932;
// REAL(4) literals promoted to REAL(8)
static const double EPS_WCNS = (double)1.e-40f;          // src/nnd_center_RK.F90:319
static const double D1_WCNS = (double)(1.f / 11.f);      // src/nnd_center_RK.F90:331
static const double D2_WCNS = (double)(10.f / 11.f);
static const double ATAN_BIAS = (double)1e-10f;          // src/XuanGua.F90:40
static const double QNAN = std::numeric_limits<double>::quiet_NaN();

struct Grid {
    int num[2];
    int lvl, sort, cross;
    double cx, cy;
    Grid *father, *son1, *son2, *son3, *son4;
    Grid *upnei, *downnei, *leftnei, *rightnei;
    Grid *upleftnei, *downrightnei, *downleftnei, *uprightnei;
    int sp;
    double U[7], Ut[7], Un[7];
    double rot, div;
    uint64_t key;
};

struct Counters {
    int64_t singular = 0;       // brinv flag=0
    int64_t wls_calls = 0;
    int64_t parent_interp = 0;  // parent_value_weno fell back to interpA (m<7)
    int64_t child_copy = 0;     // child_value_weno fell back to c%U (m<7)
    int64_t gm4_nonleaf = 0;    // gridmodify4 Refine_cell of a non-leaf nnbor
    int64_t regrids = 0;
};

struct Solver {
    fdm_params p{};
    double Xmin, Xmax, Ymin, Ymax, h, xf, gama, cv, Ma;
    int m = 0, n = 0, total = 0;
    // strip of a mesh (no reference counterpart): local row 1 is global row
    // row0 + 1 of nglob rows; halo_lo / halo_hi: the three outer rows on that
    // side are a halo (neither advanced nor filled here)
    int row0 = 0, nglob = 0;
    bool halo_lo = false, halo_hi = false;
    std::vector<Grid> cell;  // cell(i) == cell[i-1]
    std::vector<Grid *> cell_NS, cell_BC;
    std::vector<double> fu_buf;  // per-leaf fu*dx*dy of the last stage (4 each)
    double lambda_x = 0, lambda_y = 0, tstep = 0, tt = 0;
    int64_t it = 0;
    int l_max = 0;
    double Res_max[6] = {0}, Res_rms[6] = {0};
    double Srot = 0, Sdiv = 0;
    int64_t Ne = 0;
    int Neq = 4;
    Counters cnt;
    int ic_kind = 0;
    double icp[32] = {0};
    int nthreads = 1;
    Grid *C(int i) { return &cell[(size_t)(i - 1)]; }
};

static inline double ipow2(int l) { return (double)(1LL << l); }  // 2**l as REAL

// ====================================================== src/neighbor.F90
static Grid *initial_up_neighbor(Solver &S, Grid *c) {          // :6-18
    if (c->num[0] == S.n) return nullptr;
    return S.C(c->num[0] * S.m + c->num[1]);
}
static Grid *initial_down_neighbor(Solver &S, Grid *c) {        // :21-33
    if (c->num[0] == 1) return nullptr;
    return S.C(c->num[0] * S.m - 2 * S.m + c->num[1]);
}
static Grid *initial_left_neighbor(Solver &S, Grid *c) {        // :36-48
    if (c->num[1] == 1) return nullptr;
    return S.C(c->num[0] * S.m - S.m + c->num[1] - 1);
}
static Grid *initial_right_neighbor(Solver &S, Grid *c) {       // :51-63
    if (c->num[1] == S.m) return nullptr;
    return S.C(c->num[0] * S.m - S.m + c->num[1] + 1);
}

static Grid *up_neighbor(Solver &S, Grid *cell) {               // :65-96
    Grid *celln = initial_up_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cell->father) return celln;
    if (cell->sp == 1) return cellf->son4;
    if (cell->sp == 2) return cellf->son3;
    Grid *cellfn = up_neighbor(S, cellf);
    if (cellfn) {
        if (!cellfn->son1) return cellfn;
        if (cell->sp == 4) return cellfn->son1;
        if (cell->sp == 3) return cellfn->son2;
    }
    return nullptr;
}
static Grid *down_neighbor(Solver &S, Grid *cell) {             // :98-129
    Grid *celln = initial_down_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cell->father) return celln;
    if (cell->sp == 4) return cellf->son1;
    if (cell->sp == 3) return cellf->son2;
    Grid *cellfn = down_neighbor(S, cellf);
    if (cellfn) {
        if (!cellfn->son1) return cellfn;
        if (cell->sp == 1) return cellfn->son4;
        if (cell->sp == 2) return cellfn->son3;
    }
    return nullptr;
}
static Grid *left_neighbor(Solver &S, Grid *cell) {             // :131-162
    Grid *celln = initial_left_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cell->father) return celln;
    if (cell->sp == 2) return cellf->son1;
    if (cell->sp == 3) return cellf->son4;
    Grid *cellfn = left_neighbor(S, cellf);
    if (cellfn) {
        if (!cellfn->son1) return cellfn;
        if (cell->sp == 4) return cellfn->son3;
        if (cell->sp == 1) return cellfn->son2;
    }
    return nullptr;
}
static Grid *right_neighbor(Solver &S, Grid *c) {               // :164-196
    Grid *celln = initial_right_neighbor(S, c);
    Grid *cellf = c->father;
    if (!c->father) return celln;
    if (c->sp == 1) return cellf->son2;
    if (c->sp == 4) return cellf->son3;
    Grid *cellfn = right_neighbor(S, cellf);
    if (cellfn) {
        if (!cellfn->son1) return cellfn;
        if (c->sp == 2) return cellfn->son1;
        if (c->sp == 3) return cellfn->son4;
    }
    return nullptr;
}

static Grid *upleft_neighbor(Solver &S, Grid *cell) {           // :199-246
    Grid *celln = left_neighbor(S, cell);
    Grid *cellfn = up_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cellf) {
        if (!celln || !cellfn) return nullptr;
        return up_neighbor(S, celln);
    } else if (cell->sp == 2) {
        return cellf->son4;
    } else if (cell->sp == 4) {
        if (!celln || !cellfn) return nullptr;
        Grid *r = up_neighbor(S, celln);
        while (r->lvl < cell->lvl && r->son2) r = r->son2;
        return r;
    } else if (cell->sp == 1) {
        if (!celln || celln->lvl < cell->lvl) return nullptr;
        return up_neighbor(S, celln);
    } else if (cell->sp == 3) {
        if (!cellfn || cellfn->lvl < cell->lvl) return nullptr;
        return left_neighbor(S, cellfn);
    }
    return nullptr;
}
static Grid *upright_neighbor(Solver &S, Grid *cell) {          // :249-296
    Grid *celln = right_neighbor(S, cell);
    Grid *cellfn = up_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cellf) {
        if (!celln || !cellfn) return nullptr;
        return up_neighbor(S, celln);
    } else if (cell->sp == 1) {
        return cellf->son3;
    } else if (cell->sp == 3) {
        if (!celln || !cellfn) return nullptr;
        Grid *r = up_neighbor(S, celln);
        while (r->lvl < cell->lvl && r->son1) r = r->son1;
        return r;
    } else if (cell->sp == 2) {
        if (!celln || celln->lvl < cell->lvl) return nullptr;
        return up_neighbor(S, celln);
    } else if (cell->sp == 4) {
        if (!cellfn || cellfn->lvl < cell->lvl) return nullptr;
        return right_neighbor(S, cellfn);
    }
    return nullptr;
}
static Grid *downright_neighbor(Solver &S, Grid *cell) {        // :299-346
    Grid *celln = right_neighbor(S, cell);
    Grid *cellfn = down_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cellf) {
        if (!celln || !cellfn) return nullptr;
        return down_neighbor(S, celln);
    } else if (cell->sp == 4) {
        return cellf->son2;
    } else if (cell->sp == 2) {
        if (!celln || !cellfn) return nullptr;
        Grid *r = down_neighbor(S, celln);
        while (r->lvl < cell->lvl && r->son4) r = r->son4;
        return r;
    } else if (cell->sp == 3) {
        if (!celln || celln->lvl < cell->lvl) return nullptr;
        return down_neighbor(S, celln);
    } else if (cell->sp == 1) {
        if (!cellfn || cellfn->lvl < cell->lvl) return nullptr;
        return right_neighbor(S, cellfn);
    }
    return nullptr;
}
static Grid *downleft_neighbor(Solver &S, Grid *cell) {         // :349-396
    Grid *celln = left_neighbor(S, cell);
    Grid *cellfn = down_neighbor(S, cell);
    Grid *cellf = cell->father;
    if (!cellf) {
        if (!celln || !cellfn) return nullptr;
        return down_neighbor(S, celln);
    } else if (cell->sp == 3) {
        return cellf->son1;
    } else if (cell->sp == 1) {
        if (!celln || !cellfn) return nullptr;
        Grid *r = down_neighbor(S, celln);
        while (r->lvl < cell->lvl && r->son3) r = r->son3;
        return r;
    } else if (cell->sp == 4) {
        if (!celln || celln->lvl < cell->lvl) return nullptr;
        return down_neighbor(S, celln);
    } else if (cell->sp == 2) {
        if (!cellfn || cellfn->lvl < cell->lvl) return nullptr;
        return left_neighbor(S, cellfn);
    }
    return nullptr;
}

static void idnei(Solver &S, Grid *c) {                         // :412-449
    Grid *ct1 = up_neighbor(S, c), *ct2 = down_neighbor(S, c);
    Grid *ct3 = right_neighbor(S, c), *ct4 = left_neighbor(S, c);
    Grid *ct5 = nullptr, *ct6 = nullptr, *ct7 = nullptr, *ct8 = nullptr;
    if (c->cross >= 0) {
        ct5 = upleft_neighbor(S, c);
        ct6 = upright_neighbor(S, c);
        ct7 = downleft_neighbor(S, c);
        ct8 = downright_neighbor(S, c);
    }
    c->upnei = ct1; c->downnei = ct2; c->rightnei = ct3; c->leftnei = ct4;
    c->upleftnei = ct5; c->uprightnei = ct6; c->downleftnei = ct7; c->downrightnei = ct8;
    if (c->son1) {
        idnei(S, c->son1); idnei(S, c->son2); idnei(S, c->son3); idnei(S, c->son4);
    }
}
static void idneighbor(Solver &S) {                             // :399-409
    for (int i = 1; i <= S.total; ++i) idnei(S, S.C(i));
}

// ====================================================== src/XuanGua.F90
struct NList {  // type(p_array), allocatable :: neighbors(:)
    Grid *a[16];
    int n = 0;
};
static void add_to_neighbor_list(Grid *nw, NList &L) {          // :11-30
    for (int k = 0; k < L.n; ++k) if (L.a[k] == nw) return;
    L.a[L.n++] = nw;
}

static int get_direction(double xx, double yy, double x, double y) {  // :33-43
    double dx = xx - x;
    double dy = yy - y;
    double angle = (std::atan2(dy, dx) + ATAN_BIAS) * 180.0 / Pi;
    int f = (int)std::floor((angle + 22.5) / 45.0 + 8);
    return ((f % 8) + 8) % 8 + 1;
}

static void search_cell_5(Grid *c, double x, double y, NList &n1, NList &n2,
                          bool dir_used[8]) {                   // :152-177
    if (!c->son1) {
        int dir = get_direction(c->cx, c->cy, x, y);
        if (!dir_used[dir - 1]) {
            if (dir == 1 || dir == 5 || dir == 3 || dir == 7) add_to_neighbor_list(c, n1);
            else add_to_neighbor_list(c, n2);
            dir_used[dir - 1] = true;
        }
    } else {
        // the reference repeats this group 4 times; repeats are no-ops
        search_cell_5(c->son1, x, y, n1, n2, dir_used);
        search_cell_5(c->son2, x, y, n1, n2, dir_used);
        search_cell_5(c->son3, x, y, n1, n2, dir_used);
        search_cell_5(c->son4, x, y, n1, n2, dir_used);
    }
}

// brinv: full-pivot Gauss-Jordan inverse, in place on r (n x n, r[i][j]
// = row i, column j, 0-based).  Returns false on the singular test.
template <int N>
static bool brinv(double r[N][N], Counters *cnt) {              // :593-660
    int is[N], js[N];
    for (int k = 0; k < N; ++k) { is[k] = 0; js[k] = 0; }
    for (int k = 0; k < N; ++k) {
        double d = 0.0;
        for (int i = k; i < N; ++i)
            for (int j = k; j < N; ++j)
                if (std::fabs(r[i][j]) > d) { d = std::fabs(r[i][j]); is[k] = i; js[k] = j; }
        if (d + 1.0 == 1.0) {
            if (cnt) {
#pragma omp atomic
                cnt->singular++;
            }
            return false;
        }
        for (int j = 0; j < N; ++j) { double t = r[k][j]; r[k][j] = r[is[k]][j]; r[is[k]][j] = t; }
        for (int i = 0; i < N; ++i) { double t = r[i][k]; r[i][k] = r[i][js[k]]; r[i][js[k]] = t; }
        r[k][k] = 1.0 / r[k][k];
        for (int j = 0; j < N; ++j) if (j != k) r[k][j] = r[k][j] * r[k][k];
        for (int i = 0; i < N; ++i)
            if (i != k)
                for (int j = 0; j < N; ++j)
                    if (j != k) r[i][j] = r[i][j] - r[i][k] * r[k][j];
        for (int i = 0; i < N; ++i) if (i != k) r[i][k] = -r[i][k] * r[k][k];
    }
    for (int k = N - 1; k >= 0; --k) {
        for (int j = 0; j < N; ++j) { double t = r[k][j]; r[k][j] = r[js[k]][j]; r[js[k]][j] = t; }
        for (int i = 0; i < N; ++i) { double t = r[i][k]; r[i][k] = r[i][is[k]]; r[i][is[k]] = t; }
    }
    return true;
}

static double integrate_square_poly(const double k[3], double x_min, double x_max,
                                    double y_min, double y_max) {    // :342-355
    double term1 = k[0] * k[0] * (x_max - x_min) * (y_max - y_min);
    double term2 = 2 * k[0] * k[1] * (x_max * x_max - x_min * x_min) / 2 * (y_max - y_min) +
                   2 * k[0] * k[2] * (x_max - x_min) * (y_max * y_max - y_min * y_min) / 2;
    double term3 = k[1] * k[1] * (x_max * x_max * x_max - x_min * x_min * x_min) / 3 * (y_max - y_min) +
                   2 * k[1] * k[2] * (x_max * x_max - x_min * x_min) / 2 * (y_max * y_max - y_min * y_min) / 2 +
                   k[2] * k[2] * (x_max - x_min) * (y_max * y_max * y_max - y_min * y_min * y_min) / 3;
    return term1 + term2 + term3;
}

static double compute_smoothness(const Solver &S, const Grid *c, const double *coeff,
                                  int order) {                   // :309-340
    double hx = S.xf * S.h / ipow2(c->lvl + 1);
    double hy = S.h / ipow2(c->lvl + 1);
    double x_min = c->cx - hx, x_max = c->cx + hx;
    double y_min = c->cy - hy, y_max = c->cy + hy;
    double beta = 0.0;
    if (order == 2) {
        double a1 = coeff[1], a2 = coeff[2], a3 = coeff[3], a4 = coeff[4], a5 = coeff[5];
        double k1[3] = {a1, 2 * a3, a4};
        double k2[3] = {a2, a4, 2 * a5};
        beta = 0.0;
        beta = beta + integrate_square_poly(k1, x_min, x_max, y_min, y_max);
        beta = beta + integrate_square_poly(k2, x_min, x_max, y_min, y_max);
        beta = beta + (2 * a3) * (2 * a3) * (x_max - x_min) * (y_max - y_min);
        beta = beta + a4 * a4 * (x_max - x_min) * (y_max - y_min);
        beta = beta + (2 * a5) * (2 * a5) * (x_max - x_min) * (y_max - y_min);
    } else {
        double b1 = coeff[1], b2 = coeff[2];
        beta = (b1 * b1 + b2 * b2) * (x_max - x_min) * (y_max - y_min);
    }
    return beta;
}

static void WLSI_US_WENO(Solver &S, const Grid *c, double xx, double yy, const NList &n1,
                         const NList &n2, double var[NVAR]) {  // :179-356
    const int m1 = n1.n, m2 = n2.n, m = m1 + m2;
    const double eps = 1.e-6;
    double cvar[16][7], x[16], y[16], d[16], w[16];
    for (int i = 0; i < m1; ++i) {
        for (int k = 0; k < 7; ++k) cvar[i][k] = n1.a[i]->U[k];
        x[i] = n1.a[i]->cx; y[i] = n1.a[i]->cy;
        d[i] = std::sqrt((x[i] - xx) * (x[i] - xx) + (y[i] - yy) * (y[i] - yy));
        w[i] = 1.0 / (d[i] + eps);
    }
    for (int i = 0; i < m2; ++i) {
        for (int k = 0; k < 7; ++k) cvar[m1 + i][k] = n2.a[i]->U[k];
        x[m1 + i] = n2.a[i]->cx; y[m1 + i] = n2.a[i]->cy;
        d[m1 + i] = std::sqrt((x[m1 + i] - xx) * (x[m1 + i] - xx) + (y[m1 + i] - yy) * (y[m1 + i] - yy));
        w[m1 + i] = 1.0 / (d[m1 + i] + eps);
    }
    double P[16][6];
    for (int i = 0; i < m; ++i) {
        P[i][0] = 1.0; P[i][1] = x[i]; P[i][2] = y[i];
        P[i][3] = x[i] * y[i]; P[i][4] = x[i] * x[i]; P[i][5] = y[i] * y[i];
    }
    // WP = W*P with W diagonal: every off-diagonal product is 0*P (+-0),
    // so WP(i,j) = w(i)*P(i,j) exactly.
    double L[6][6];
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b) {
            double s = 0.0;
            for (int i = 0; i < m; ++i) s = s + P[i][a] * (w[i] * P[i][b]);
            L[a][b] = s;
        }
    brinv<6>(L, &S.cnt);
    double A[3][3], B[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
            for (int i = 0; i < m1; ++i) s = s + P[i][a] * (w[i] * P[i][b]);
            A[a][b] = s;
            double t = 0.0;
            for (int i = 0; i < m2; ++i) t = t + P[m1 + i][a] * (w[m1 + i] * P[m1 + i][b]);
            B[a][b] = t;
        }
    brinv<3>(A, &S.cnt);
    brinv<3>(B, &S.cnt);
    const double lw[3] = {0.98, 0.01, 0.01};
    static const int ks[4] = {0, 1, 2, 4};
    for (int kk = 0; kk < 4; ++kk) {
        const int k = ks[kk];
        double wphi[16];
        for (int i = 0; i < m; ++i) wphi[i] = w[i] * cvar[i][k];
        double ptwphi[6], arr[6];
        for (int a = 0; a < 6; ++a) {
            double s = 0.0;
            for (int i = 0; i < m; ++i) s = s + P[i][a] * wphi[i];
            ptwphi[a] = s;
        }
        for (int a = 0; a < 6; ++a) {
            double s = 0.0;
            for (int b = 0; b < 6; ++b) s = s + L[a][b] * ptwphi[b];
            arr[a] = s;
        }
        double var_large = arr[0] + xx * arr[1] + yy * arr[2] + xx * yy * arr[3] +
                           xx * xx * arr[4] + yy * yy * arr[5];
        double sm_large = compute_smoothness(S, c, arr, 2);
        double p1[3], a1[3], p2[3], a2[3];
        for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int i = 0; i < m1; ++i) s = s + P[i][a] * wphi[i];
            p1[a] = s;
        }
        for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int b = 0; b < 3; ++b) s = s + A[a][b] * p1[b];
            a1[a] = s;
        }
        for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int i = 0; i < m2; ++i) s = s + P[m1 + i][a] * wphi[m1 + i];
            p2[a] = s;
        }
        for (int a = 0; a < 3; ++a) {
            double s = 0.0;
            for (int b = 0; b < 3; ++b) s = s + B[a][b] * p2[b];
            a2[a] = s;
        }
        double vs1 = a1[0] + xx * a1[1] + yy * a1[2];
        double vs2 = a2[0] + xx * a2[1] + yy * a2[2];
        double sm1 = compute_smoothness(S, c, a1, 1);
        double sm2 = compute_smoothness(S, c, a2, 1);
        double beta[3] = {sm_large, sm1, sm2};
        double sa = 0.0;
        sa = sa + std::fabs(beta[0] - beta[1]);
        sa = sa + std::fabs(beta[0] - beta[2]);
        double tau = sa / 2.0;
        tau = tau * tau;
        double alpha[3], omega[3];
        for (int q = 0; q < 3; ++q) alpha[q] = lw[q] * (1.0 + tau / (eps + beta[q]));
        double salpha = 0.0;
        salpha = salpha + alpha[0];
        salpha = salpha + alpha[1];
        salpha = salpha + alpha[2];
        for (int q = 0; q < 3; ++q) omega[q] = alpha[q] / salpha;
        var[k] = omega[0] * (1.0 / lw[0] * var_large -
                             (lw[1] / lw[0] * vs1 + lw[2] / lw[0] * vs2)) +
                 (omega[1] * vs1 + omega[2] * vs2);
    }
    var[3] = QNAN;  // undefined in the reference
#pragma omp atomic
    S.cnt.wls_calls++;
}

static void interpA(Grid *c, double var[NVAR]) {               // :359-398
    if (!c->son1) {
        for (int k = 0; k < 7; ++k) var[k] = c->U[k];
        return;
    }
    double s1[NVAR], s2[NVAR], s3[NVAR], s4[NVAR];
    if (c->son1->son1) interpA(c->son1, s1); else for (int k = 0; k < 7; ++k) s1[k] = c->son1->U[k];
    if (c->son2->son1) interpA(c->son2, s2); else for (int k = 0; k < 7; ++k) s2[k] = c->son2->U[k];
    if (c->son3->son1) interpA(c->son3, s3); else for (int k = 0; k < 7; ++k) s3[k] = c->son3->U[k];
    if (c->son4->son1) interpA(c->son4, s4); else for (int k = 0; k < 7; ++k) s4[k] = c->son4->U[k];
    for (int k = 0; k < 7; ++k) var[k] = 0.25 * (s1[k] + s2[k] + s3[k] + s4[k]);
}

// Optional record of the stencil gathered by the next parent/child call
// (test hook: lets the tests compare the hanging-node stencils themselves).
struct GatherRec {
    int kind;           // 0 leaf copy, 1 parent WLS, 2 parent interpA, 3 child WLS, 4 child copy
    uint64_t node;      // key of the node the value is taken from
    double xx, yy;
    int m1, m2;
    uint64_t mem[16];
};
static thread_local GatherRec *tl_rec = nullptr;
static void rec_lists(const NList &n1, const NList &n2) {
    if (!tl_rec) return;
    tl_rec->m1 = n1.n;
    tl_rec->m2 = n2.n;
    for (int i = 0; i < n1.n; ++i) tl_rec->mem[i] = n1.a[i]->key;
    for (int i = 0; i < n2.n; ++i) tl_rec->mem[n1.n + i] = n2.a[i]->key;
}

static void parent_value_weno(Solver &S, Grid *c, double var[NVAR]) {  // :45-94
    NList n1, n2;
    bool used[8] = {false, false, false, false, false, false, false, false};
    double x = c->cx, y = c->cy;
    search_cell_5(c->son1, x, y, n1, n2, used);
    search_cell_5(c->son2, x, y, n1, n2, used);
    search_cell_5(c->son3, x, y, n1, n2, used);
    search_cell_5(c->son4, x, y, n1, n2, used);
    int m = n1.n + n2.n;
    if (m < 8) {
        Grid *nb[4] = {c->leftnei, c->rightnei, c->downnei, c->upnei};
        for (int q = 0; q < 4; ++q)
            if (nb[q]) search_cell_5(nb[q], x, y, n1, n2, used);
    }
    m = n1.n + n2.n;
    if (tl_rec) { rec_lists(n1, n2); tl_rec->node = c->key; tl_rec->xx = x; tl_rec->yy = y; tl_rec->kind = m < 7 ? 2 : 1; }
    if (m < 7) {
        interpA(c, var);
#pragma omp atomic
        S.cnt.parent_interp++;
    } else {
        WLSI_US_WENO(S, c, x, y, n1, n2, var);
    }
}

static void child_value_weno(Solver &S, double xx, double yy, Grid *c,
                             double var[NVAR]) {               // :96-150
    NList n1, n2;
    bool used[8] = {false, false, false, false, false, false, false, false};
    double x = c->cx, y = c->cy;
    add_to_neighbor_list(c, n1);
    Grid *nb[8] = {c->downleftnei, c->leftnei, c->upleftnei, c->downnei,
                   c->upnei, c->downrightnei, c->rightnei, c->uprightnei};
    for (int q = 0; q < 8; ++q)
        if (nb[q]) search_cell_5(nb[q], x, y, n1, n2, used);
    int m = n1.n + n2.n;
    if (tl_rec) { rec_lists(n1, n2); tl_rec->node = c->key; tl_rec->xx = xx; tl_rec->yy = yy; tl_rec->kind = m < 7 ? 4 : 3; }
    if (m < 7) {
        for (int k = 0; k < 7; ++k) var[k] = c->U[k];
#pragma omp atomic
        S.cnt.child_copy++;
    } else {
        WLSI_US_WENO(S, c, xx, yy, n1, n2, var);
    }
}

static inline void copyU(const Grid *c, double var[NVAR]) {
    for (int k = 0; k < 7; ++k) var[k] = c->U[k];
    if (tl_rec) { tl_rec->kind = 0; tl_rec->node = c->key; tl_rec->m1 = 0; tl_rec->m2 = 0; }
}

// Tip/Tim/Tjp/Tjm (src/XuanGua.F90:401-419, 449-467, 497-515, 545-563)
enum Dir { D_RIGHT = 0, D_LEFT = 1, D_UP = 2, D_DOWN = 3 };
static Grid *nei(Grid *c, int d) {
    switch (d) {
        case D_RIGHT: return c->rightnei;
        case D_LEFT: return c->leftnei;
        case D_UP: return c->upnei;
        default: return c->downnei;
    }
}
static void target1(const Solver &S, const Grid *c, int d, double &xx, double &yy) {
    switch (d) {
        case D_RIGHT: xx = c->cx + S.xf * S.h / ipow2(c->lvl); yy = c->cy; break;
        case D_LEFT: xx = c->cx - S.xf * S.h / ipow2(c->lvl); yy = c->cy; break;
        case D_UP: xx = c->cx; yy = c->cy + S.h / ipow2(c->lvl); break;
        default: xx = c->cx; yy = c->cy - S.h / ipow2(c->lvl); break;
    }
}
static void target2(const Solver &S, const Grid *c, int d, double &xx, double &yy) {
    switch (d) {
        case D_RIGHT: xx = c->cx + 2.0 * S.xf * S.h / ipow2(c->lvl); yy = c->cy; break;
        case D_LEFT: xx = c->cx - 2.0 * S.xf * S.h / ipow2(c->lvl); yy = c->cy; break;
        case D_UP: xx = c->cx; yy = c->cy + 2.0 * S.h / ipow2(c->lvl); break;
        default: xx = c->cx; yy = c->cy - 2.0 * S.h / ipow2(c->lvl); break;
    }
}
static void T1(Solver &S, Grid *c, int d, double var[NVAR]) {
    Grid *cn = nei(c, d);
    if (cn->lvl == c->lvl) {
        if (!cn->son1) copyU(cn, var);
        else parent_value_weno(S, cn, var);
    } else {
        double xx, yy;
        target1(S, c, d, xx, yy);
        child_value_weno(S, xx, yy, cn, var);
    }
}
// Tipp/Timm/Tjpp/Tjmm (src/XuanGua.F90:422-446, 470-494, 518-542, 566-590)
static void T2(Solver &S, Grid *c, int d, double var[NVAR]) {
    Grid *cn = nei(c, d);
    double xx, yy;
    if (cn->lvl == c->lvl) {
        Grid *cnn = nei(cn, d);
        if (cnn->lvl == cn->lvl) {
            if (!cnn->son1) copyU(cnn, var);
            else parent_value_weno(S, cnn, var);
        } else {
            target2(S, c, d, xx, yy);
            child_value_weno(S, xx, yy, cnn, var);
        }
    } else {
        target2(S, c, d, xx, yy);
        child_value_weno(S, xx, yy, cn, var);
    }
}

// ================================================== src/nnd_center_RK.F90
static void WCNS_Z3(const double u1[4], const double u2[4], const double u3[4],
                    const double R[4][4], double hp[4]) {       // :310-353
    double uL[4];
    for (int i = 0; i < 4; ++i) {
        const double d1 = D1_WCNS, d2 = D2_WCNS;
        double t;
        t = -u1[i] + u2[i];
        double IS1 = t * t;
        t = -u2[i] + u3[i];
        double IS2 = t * t;
        t = u1[i] - 2. * u2[i] + u3[i];
        double IS3 = t * t;
        double p1 = u2[i];
        double p2 = ((-u1[i] + 6.0 * u2[i] + 3.0 * u3[i]) / 8.0 - d1 * p1) / d2;
        IS1 = std::fmin(IS1, IS2);
        IS2 = IS3 + u1[i] * u1[i] + u2[i] * u2[i] + u3[i] * u3[i] - u1[i] * u2[i] -
              u2[i] * u3[i] - u1[i] * u3[i];
        t = 10. * std::fabs(IS2 - 3. * IS1);
        double tau3 = t * t;
        double a1 = d1 * (1.0 + tau3 / (EPS_WCNS + IS1));
        double a2 = d2 * (1.0 + tau3 / (EPS_WCNS + IS2));
        double w1 = a1 / (a1 + a2);
        double w2 = a2 / (a1 + a2);
        uL[i] = w1 * p1 + w2 * p2;
    }
    for (int r = 0; r < 4; ++r)
        hp[r] = R[r][0] * uL[0] + R[r][1] * uL[1] + R[r][2] * uL[2] + R[r][3] * uL[3];
}

// REcalc (dir 0) / RFcalc (dir 1): src/nnd_center_RK.F90:114-169, 236-291
static void eigen(const Solver &S, int dir, const double U[4], double R[4][4], double Ri[4][4]) {
    const double g = S.gama;
    double r0 = U[0];
    double u = U[1] / U[0];
    double v = U[2] / U[0];
    double p = (g - 1.0) * r0 * (U[3] / r0 - 0.5 * (u * u + v * v));
    double a = std::sqrt(g * p / r0);
    double q2 = 0.5 * (u * u + v * v);
    const double aa = a * a, a2 = 2.0 * a * a;
    if (dir == 0) {
        R[0][0] = 1.0; R[1][0] = u - a; R[2][0] = v; R[3][0] = a * a / (g - 1) + q2 - u * a;
        R[0][1] = 1.0; R[1][1] = u; R[2][1] = v; R[3][1] = q2;
        R[0][2] = 1.0; R[1][2] = u + a; R[2][2] = v; R[3][2] = a * a / (g - 1) + q2 + u * a;
        R[0][3] = 0.0; R[1][3] = 0.0; R[2][3] = -1.0; R[3][3] = -v;
        Ri[0][0] = ((g - 1.0) * q2 + a * u) / a2;
        Ri[1][0] = (aa - (g - 1.0) * q2) / aa;
        Ri[2][0] = ((g - 1.0) * q2 - a * u) / a2;
        Ri[3][0] = v;
        Ri[0][1] = ((1.0 - g) * u - a) / a2;
        Ri[1][1] = ((g - 1.0) * u) / aa;
        Ri[2][1] = ((1.0 - g) * u + a) / a2;
        Ri[3][1] = 0.0;
        Ri[0][2] = ((1.0 - g) * v) / a2;
        Ri[1][2] = ((g - 1.0) * v) / aa;
        Ri[2][2] = ((1.0 - g) * v) / a2;
        Ri[3][2] = -1.0;
    } else {
        R[0][0] = 1.0; R[1][0] = u; R[2][0] = v - a; R[3][0] = a * a / (g - 1) + q2 - v * a;
        R[0][1] = 1.0; R[1][1] = u; R[2][1] = v; R[3][1] = q2;
        R[0][2] = 1.0; R[1][2] = u; R[2][2] = v + a; R[3][2] = a * a / (g - 1) + q2 + v * a;
        R[0][3] = 0.0; R[1][3] = 1.0; R[2][3] = 0.0; R[3][3] = u;
        Ri[0][0] = ((g - 1.0) * q2 + a * v) / a2;
        Ri[1][0] = (aa - (g - 1.0) * q2) / aa;
        Ri[2][0] = ((g - 1.0) * q2 - a * v) / a2;
        Ri[3][0] = -u;
        Ri[0][1] = ((1.0 - g) * u) / a2;
        Ri[1][1] = ((g - 1.0) * u) / aa;
        Ri[2][1] = ((1.0 - g) * u) / a2;
        Ri[3][1] = 1.0;
        Ri[0][2] = ((1.0 - g) * v - a) / a2;
        Ri[1][2] = ((g - 1.0) * v) / aa;
        Ri[2][2] = ((1.0 - g) * v + a) / a2;
        Ri[3][2] = 0.0;
    }
    Ri[0][3] = (g - 1.0) / a2;
    Ri[1][3] = (1.0 - g) / aa;
    Ri[2][3] = (g - 1.0) / a2;
    Ri[3][3] = 0.0;
}

// compute_E (dir 0) / compute_F (dir 1): src/nnd_center_RK.F90:171-185, 293-307
// U0[col][var] primitive (rho,u,v,T,p); Uc[r][col], Fl[r][col]
static void compute_flux(const Solver &S, int dir, const double U0[5][NVAR], double Fl[4][5],
                         double Uc[4][5]) {
    const double g = S.gama;
    for (int c = 0; c < 5; ++c) {
        double r = U0[c][0], u = U0[c][1], v = U0[c][2], p = U0[c][4];
        Uc[0][c] = r;
        Uc[1][c] = r * u;
        Uc[2][c] = r * v;
        Uc[3][c] = p / (g - 1.0) + 0.5 * r * (u * u + v * v);
        if (dir == 0) {
            Fl[0][c] = r * u;
            Fl[1][c] = r * u * u + p;
            Fl[2][c] = r * u * v;
            Fl[3][c] = u * (p / (g - 1.0) + 0.5 * r * (u * u + v * v) + p);
        } else {
            Fl[0][c] = r * v;
            Fl[1][c] = r * u * v;
            Fl[2][c] = r * v * v + p;
            Fl[3][c] = v * (p / (g - 1.0) + 0.5 * r * (u * u + v * v) + p);
        }
    }
}

static void matcols(const double Ri[4][4], const double X[4][5], double Y[4][5]) {
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 5; ++c) {
            double s = 0.0;
            for (int k = 0; k < 4; ++k) s = s + Ri[r][k] * X[k][c];
            Y[r][c] = s;
        }
}

// LXL_X_wcns3 (dir 0, src/nnd_center_RK.F90:66-112) and LXL_Y_wcns3
// (dir 1, :187-234).  st[0..4] = minus2, minus1, cell, plus1, plus2.
static void lxl_dir(const Solver &S, int dir, double dxy, const double *st[5], double dE[4]) {
    double U0[5][NVAR];
    for (int c = 0; c < 5; ++c)
        for (int k = 0; k < 5; ++k) U0[c][k] = st[c][k];
    double Fl[4][5], Uc[4][5], w[4][5], gg[4][5], R[4][4], Ri[4][4];
    compute_flux(S, dir, U0, Fl, Uc);
    const double lam = dir == 0 ? S.lambda_x : S.lambda_y;
    double flux_L[4], flux_R[4];
    for (int face = 0; face < 2; ++face) {
        const int o = face;  // columns o..o+3
        double Um[4];
        for (int r = 0; r < 4; ++r) Um[r] = (Uc[r][1 + o] + Uc[r][2 + o]) / 2.0;
        eigen(S, dir, Um, R, Ri);
        matcols(Ri, Uc, w);
        matcols(Ri, Fl, gg);
        double c0[4], c1[4], c2[4], c3[4];
        double wL[4], wR[4], gL[4], gR[4];
        for (int r = 0; r < 4; ++r) { c0[r] = w[r][o]; c1[r] = w[r][o + 1]; c2[r] = w[r][o + 2]; c3[r] = w[r][o + 3]; }
        WCNS_Z3(c0, c1, c2, R, wL);
        WCNS_Z3(c3, c2, c1, R, wR);
        for (int r = 0; r < 4; ++r) { c0[r] = gg[r][o]; c1[r] = gg[r][o + 1]; c2[r] = gg[r][o + 2]; c3[r] = gg[r][o + 3]; }
        WCNS_Z3(c0, c1, c2, R, gL);
        WCNS_Z3(c3, c2, c1, R, gR);
        double *fl = face == 0 ? flux_L : flux_R;
        for (int r = 0; r < 4; ++r) fl[r] = 0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r]));
    }
    for (int r = 0; r < 4; ++r) {
        if (dir == 0)
            dE[r] = 4.0 / (3.0 * dxy) * (flux_R[r] - flux_L[r]) - 1.0 / (6.0 * dxy) * (Fl[r][3] - Fl[r][1]);
        else
            dE[r] = 4.0 / 3.0 / dxy * (flux_R[r] - flux_L[r]) - 1.0 / 6.0 / dxy * (Fl[r][3] - Fl[r][1]);
    }
}

// The 8 stencil values of a leaf: Tip, Tim, Tjp, Tjm, Tipp, Timm, Tjpp, Tjmm
struct Stencil { double v[8][NVAR]; };
static void fetch_stencil(Solver &S, Grid *c, Stencil &st) {
    T1(S, c, D_RIGHT, st.v[0]); T1(S, c, D_LEFT, st.v[1]);
    T1(S, c, D_UP, st.v[2]); T1(S, c, D_DOWN, st.v[3]);
    T2(S, c, D_RIGHT, st.v[4]); T2(S, c, D_LEFT, st.v[5]);
    T2(S, c, D_UP, st.v[6]); T2(S, c, D_DOWN, st.v[7]);
}

// solution_cell + LXL + Res_LXL (src/solution.F90:302-312,
// src/nnd_center_RK.F90:15-64); fu_out receives fu*dx*dy.
static void solution_cell(Solver &S, Grid *c, double fu_out[4]) {
    Stencil st;
    fetch_stencil(S, c, st);
    const double dy = S.h / ipow2(c->lvl);
    const double dx = S.xf * dy;
    const double g = S.gama;
    double U[4];
    U[0] = c->U[0];
    U[1] = c->U[0] * c->U[1];
    U[2] = c->U[0] * c->U[2];
    U[3] = c->U[4] / (g - 1.0) + 0.5 * c->U[0] * (c->U[1] * c->U[1] + c->U[2] * c->U[2]);
    const double *sx[5] = {st.v[5], st.v[1], c->U, st.v[0], st.v[4]};
    const double *sy[5] = {st.v[7], st.v[3], c->U, st.v[2], st.v[6]};
    double dE[4], dF[4], fu[4], Ut[4];
    lxl_dir(S, 0, dx, sx, dE);
    lxl_dir(S, 1, dy, sy, dF);
    for (int i = 0; i < 4; ++i) fu[i] = -dE[i] - dF[i];
    for (int i = 0; i < 4; ++i) {
        Ut[i] = U[i] + fu[i] * S.tstep;
        fu_out[i] = fu[i] * dx * dy;
    }
    c->Ut[0] = Ut[0];
    c->Ut[1] = Ut[1] / Ut[0];
    c->Ut[2] = Ut[2] / Ut[0];
    c->Ut[3] = (Ut[3] - 0.5 * Ut[0] * (c->Ut[1] * c->Ut[1] + c->Ut[2] * c->Ut[2])) / (S.cv * Ut[0]);
    c->Ut[4] = (g - 1.0) * c->Ut[0] * (Ut[3] / c->Ut[0] - 0.5 * (c->Ut[1] * c->Ut[1] + c->Ut[2] * c->Ut[2]));
}

// ====================================================== src/mesh.F90
static int gridcross(const Solver &S, const Grid *c) {          // :89-142
    // the class in the whole mesh (global row), also for a strip of it
    const int r = c->num[0] + S.row0, q = c->num[1], m = S.m, n = S.nglob;
    if (r < 4 && q < 4) return BCcorner;
    if (r < 4 && q > m - 3) return BCcorner;
    if (r > n - 3 && q > m - 3) return BCcorner;
    if (r > n - 3 && q < 4) return BCcorner;
    if (r < 4) return -1;
    if (r > n - 3) return -3;
    if (q > m - 3) return -2;
    if (q < 4) return -4;
    return 0;  // gridsort is identically 0 (src/mesh.F90:81-87)
}

// a node in the halo rows of a strip
static bool in_halo(const Solver &S, const Grid *c) {
    return (S.halo_lo && c->num[0] <= 3) || (S.halo_hi && c->num[0] > S.n - 3);
}

static const int SP_TO_Q[5] = {0, 0, 1, 3, 2};  // sp -> Morton quadrant

static Grid *new_child(Solver &S, Grid *c, int sp, double sx, double sy) {
    Grid *s = new Grid();
    *s = Grid{};
    s->father = c;
    s->num[0] = c->num[0]; s->num[1] = c->num[1];
    s->lvl = c->lvl + 1;
    s->sp = sp;
    s->cx = sx; s->cy = sy;
    s->sort = 0;
    s->cross = gridcross(S, s);
    for (int k = 0; k < 7; ++k) { s->U[k] = c->U[k]; s->Ut[k] = c->U[k]; s->Un[k] = c->U[k]; }
    s->rot = c->rot; s->div = c->div;
    uint64_t path = FDM_KEY_PATH(c->key) | ((uint64_t)SP_TO_Q[sp] << (2 * (FDM_LMAX - s->lvl)));
    s->key = FDM_KEY(FDM_KEY_ROOT(c->key), s->lvl, path);
    return s;
}

static void free_subtree(Grid *c) {
    if (!c) return;
    free_subtree(c->son1); free_subtree(c->son2); free_subtree(c->son3); free_subtree(c->son4);
    delete c;
}

static void Refine_cell(Solver &S, Grid *c) {                   // :199-260
    // A Refine_cell of a node that already has sons (gridmodify4, :389-392)
    // replaces the old subtree; the old one is unreachable afterwards.
    Grid *old[4] = {c->son1, c->son2, c->son3, c->son4};
    const double qx = S.xf * S.h / ipow2(c->lvl + 2);
    const double qy = S.h / ipow2(c->lvl + 2);
    c->son1 = new_child(S, c, 1, c->cx - qx, c->cy - qy);
    c->son2 = new_child(S, c, 2, c->cx + qx, c->cy - qy);
    c->son3 = new_child(S, c, 3, c->cx + qx, c->cy + qy);
    c->son4 = new_child(S, c, 4, c->cx - qx, c->cy + qy);
    for (auto *o : old) free_subtree(o);
}

static void Coarse_cell(Solver &, Grid *c) {                    // :397-408
    double var[NVAR];
    interpA(c, var);
    for (int k = 0; k < 7; ++k) c->U[k] = var[k];
    for (int k = 0; k < 7; ++k) c->Un[k] = c->U[k];
    free_subtree(c->son1); free_subtree(c->son2); free_subtree(c->son3); free_subtree(c->son4);
    c->son1 = c->son2 = c->son3 = c->son4 = nullptr;
}

// ---- static block refinement, run by creat_mesh when lvlBlock > 0
// (src/mesh.F90:41-44, 49-197, 262-303, 421-461).  box = Block_size(1:4)
// as set_parameter leaves it (+1e-10 on the upper bounds, src/MAIN.F90:57);
// refinesize(i) = BufferLayerLVL*h/2**(i-1) (src/MAIN.F90:63-66); sort is
// identically 0 (gridsort, src/mesh.F90:81-87).
struct BlockSpec {
    int lvlblock = 0;
    double box[4] = {0, 0, 0, 0};
    double refinesize[FDM_LMAX + 2] = {0};
};
static double miblock(const BlockSpec &B, const Grid *c) {      // :421-461
    const double xo = c->cx, yo = c->cy;
    const double *bs = B.box;
    if (xo > bs[1]) {
        if (yo > bs[3]) return std::sqrt((xo - bs[1]) * (xo - bs[1]) + (yo - bs[3]) * (yo - bs[3]));
        if (yo < bs[2]) return std::sqrt((xo - bs[1]) * (xo - bs[1]) + (yo - bs[2]) * (yo - bs[2]));
        return xo - bs[1];
    }
    if (xo < bs[0]) {
        if (yo > bs[3]) return std::sqrt((xo - bs[0]) * (xo - bs[0]) + (yo - bs[3]) * (yo - bs[3]));
        if (yo < bs[2]) return std::sqrt((xo - bs[0]) * (xo - bs[0]) + (yo - bs[2]) * (yo - bs[2]));
        return bs[0] - xo;
    }
    if (yo > bs[3]) return yo - bs[3];
    if (yo < bs[2]) return bs[2] - yo;
    return 0.0;
}
static void Block_refi(Solver &S, const BlockSpec &B, Grid *c) {   // :176-197
    if (c->lvl >= B.lvlblock) return;
    if (c->son1) {
        Block_refi(S, B, c->son1); Block_refi(S, B, c->son2);
        Block_refi(S, B, c->son3); Block_refi(S, B, c->son4);
        return;
    }
    if (c->sort == 1) return;
    if (c->cx < B.box[0] || c->cx > B.box[1] || c->cy < B.box[2] || c->cy > B.box[3]) return;
    Refine_cell(S, c);
    Block_refi(S, B, c->son1); Block_refi(S, B, c->son2);
    Block_refi(S, B, c->son3); Block_refi(S, B, c->son4);
}
static void BlockDis_refi(Solver &S, const BlockSpec &B, Grid *c) {  // :144-174
    if (c->lvl >= B.lvlblock) return;
    if (c->son1) {
        BlockDis_refi(S, B, c->son1); BlockDis_refi(S, B, c->son2);
        BlockDis_refi(S, B, c->son3); BlockDis_refi(S, B, c->son4);
        return;
    }
    if (c->sort == 1) return;
    const double dis = miblock(B, c);
    for (int i = 1; i <= B.lvlblock; ++i) {
        if (dis <= B.refinesize[i] && c->sort == 0 && c->lvl < i) {
            Refine_cell(S, c);
            BlockDis_refi(S, B, c->son1); BlockDis_refi(S, B, c->son2);
            BlockDis_refi(S, B, c->son3); BlockDis_refi(S, B, c->son4);
            break;
        }
    }
}
static void gridmodify0(Solver &S, Grid *c) {                   // gridmodify, :262-303
    if (c->son1) {
        gridmodify0(S, c->son1); gridmodify0(S, c->son2);
        gridmodify0(S, c->son3); gridmodify0(S, c->son4);
        return;
    }
    Grid *cjp = up_neighbor(S, c), *cjm = down_neighbor(S, c);
    Grid *cim = left_neighbor(S, c), *cip = right_neighbor(S, c);
    if (cjp && c->lvl - cjp->lvl > 1) Refine_cell(S, cjp);
    if (cjm && c->lvl - cjm->lvl > 1) Refine_cell(S, cjm);
    if (cim && c->lvl - cim->lvl > 1) Refine_cell(S, cim);
    if (cip && c->lvl - cip->lvl > 1) Refine_cell(S, cip);
}
static void Block_refine(Solver &S, const BlockSpec &B) {        // :49-79
    for (int i = 1; i <= S.total; ++i) Block_refi(S, B, S.C(i));
    for (int i = 1; i <= S.total; ++i) BlockDis_refi(S, B, S.C(i));
    for (int j = 1; j <= B.lvlblock - 1; ++j)
        for (int i = 1; i <= S.total; ++i)
            if (S.C(i)->son1) gridmodify0(S, S.C(i));
}

static void gridmodify1(Solver &S, Grid *c) {                   // :305-353
    if (c->son1) {
        gridmodify1(S, c->son1); gridmodify1(S, c->son2);
        gridmodify1(S, c->son3); gridmodify1(S, c->son4);
    }
    if (c->cross != 0) return;
    Grid *cjp = up_neighbor(S, c), *cjm = down_neighbor(S, c);
    Grid *cim = left_neighbor(S, c), *cip = right_neighbor(S, c);
    bool up = cjp && cjp->son1, down = cjm && cjm->son1;
    bool left = cim && cim->son1, right = cip && cip->son1;
    if (!c->son1) {
        if ((left && right) || (up && down)) Refine_cell(S, c);
    } else if (!c->son1->son1 && !c->son2->son1 && !c->son3->son1 && !c->son4->son1) {
        if ((!left && !right) || (!up && !down)) Coarse_cell(S, c);
    }
}

static void gridmodify4(Solver &S, Grid *c) {                   // :355-395
    if (c->son1) {
        gridmodify4(S, c->son1); gridmodify4(S, c->son2);
        gridmodify4(S, c->son3); gridmodify4(S, c->son4);
        return;
    }
    for (int dir = 1; dir <= 4; ++dir) {
        Grid *nb = dir == 1 ? right_neighbor(S, c) : dir == 2 ? left_neighbor(S, c)
                 : dir == 3 ? up_neighbor(S, c) : down_neighbor(S, c);
        if (!nb) continue;
        if (nb->lvl <= c->lvl - 2) Refine_cell(S, nb);
        Grid *nn = dir == 1 ? right_neighbor(S, nb) : dir == 2 ? left_neighbor(S, nb)
                 : dir == 3 ? up_neighbor(S, nb) : down_neighbor(S, nb);
        if (nn && nn->lvl <= c->lvl - 2) {
            if (nn->son1) S.cnt.gm4_nonleaf++;
            Refine_cell(S, nn);
        }
    }
}

// ====================================================== src/solution.F90
static void IDNS(Solver &S, Grid *c) {                          // :655-670
    if (c->son1) {
        IDNS(S, c->son1); IDNS(S, c->son2); IDNS(S, c->son4); IDNS(S, c->son3);
    } else if (c->sort == 0) {
        if (c->cross < 0 || in_halo(S, c)) return;
        S.cell_NS.push_back(c);
    }
}
static void IDBC(Solver &S, Grid *c) {                          // :672-693
    if (c->son1) {
        IDBC(S, c->son1); IDBC(S, c->son2); IDBC(S, c->son3); IDBC(S, c->son4);
    } else if (c->sort == 0) {
        if (c->cross == BCcorner || in_halo(S, c)) return;
        if (c->cross < 0) S.cell_BC.push_back(c);
    }
}
static void IDgrid(Solver &S) {                                 // :593-615
    S.cell_NS.clear(); S.cell_BC.clear();
    for (int i = 1; i <= S.total; ++i) { IDNS(S, S.C(i)); IDBC(S, S.C(i)); }
}

// ---- boundary conditions
// BC_cyc (src/solution.F90:109-168): periodic image root by index arithmetic,
// then descent along the ghost's sp list taken deepest-first, then interpA.
static Grid *bc_cyc_image(Solver &S, Grid *c, int a) {
    int i = 0;
    const int m = S.m, n = S.n;
    if (a == -4) i = c->num[0] * m + c->num[1] - 6;
    else if (a == -2) i = c->num[0] * m + c->num[1] - 2 * m + 6;
    else if (a == -3) i = c->num[0] * m + c->num[1] - (n - 5) * m;
    else if (a == -1) i = c->num[0] * m + c->num[1] - (7 - n) * m;
    Grid *cn = S.C(i);
    if (c->lvl != 0) {
        int sp[FDM_LMAX + 1];
        Grid *cf = c;
        for (int j = 0; j < c->lvl; ++j) { sp[j] = cf->sp; cf = cf->father; }
        for (int j = 0; j < c->lvl; ++j) {
            if (!cn->son1) break;
            cn = sp[j] == 1 ? cn->son1 : sp[j] == 2 ? cn->son2 : sp[j] == 3 ? cn->son3 : cn->son4;
        }
    }
    return cn;
}

// EXT: image node for the extension kinds: a root given by (row, col) and a
// descent along the ghost's own path (root to leaf), with the quadrant bits
// transformed: mode 0 keeps them, mode 1 forces x to xbit, mode 2 forces y
// to ybit, mode 3 mirrors y, mode 4 mirrors x.
static Grid *ext_image(Solver &S, Grid *c, int row, int col, int mode, int bit) {
    Grid *cn = S.C((row - 1) * S.m + col);
    int path[FDM_LMAX + 1];
    Grid *cf = c;
    for (int j = c->lvl - 1; j >= 0; --j) { path[j] = SP_TO_Q[cf->sp]; cf = cf->father; }
    for (int j = 0; j < c->lvl; ++j) {
        if (!cn->son1) break;
        int q = path[j];
        if (mode == 1) q = (q & 2) | bit;
        else if (mode == 2) q = (q & 1) | (bit << 1);
        else if (mode == 3) q = q ^ 2;
        else if (mode == 4) q = q ^ 1;
        cn = q == 0 ? cn->son1 : q == 1 ? cn->son2 : q == 3 ? cn->son3 : cn->son4;
    }
    return cn;
}

static void set_state(Solver &S, Grid *c, const double st[4]) {
    c->U[0] = st[0]; c->U[1] = st[1]; c->U[2] = st[2]; c->U[4] = st[3];
    c->U[3] = (c->U[4] * S.gama * S.Ma * S.Ma) / c->U[0];
    c->U[5] = 0.0; c->U[6] = 0.0;
}

// One ghost leaf (body_boundary_RK / initial_boundary, src/solution.F90:71-107,
// 314-356) at boundary time t.
static void fill_ghost(Solver &S, Grid *c, double t) {
    if (c->sort != 0 || in_halo(S, c)) return;
    int a = c->cross;
    int kind;
    if (a == -4) kind = S.p.kind_xmbc;
    else if (a == -2) kind = S.p.kind_xpbc;
    else if (a == -3) kind = S.p.kind_ypbc;
    else if (a == -1) kind = S.p.kind_ymbc;
    else return;
    double var[NVAR];
    const int m = S.m, n = S.n;
    const int row = c->num[0], col = c->num[1];
    switch (kind) {
        case FDM_BC_PERIODIC: {
            interpA(bc_cyc_image(S, c, a), var);
            for (int k = 0; k < 7; ++k) c->U[k] = var[k];
            return;
        }
        case FDM_BC_TRANSMISSIVE: {  // EXT
            Grid *cn;
            if (a == -4) cn = ext_image(S, c, row, 4, 1, 0);
            else if (a == -2) cn = ext_image(S, c, row, m - 3, 1, 1);
            else if (a == -1) cn = ext_image(S, c, 4, col, 2, 0);
            else cn = ext_image(S, c, n - 3, col, 2, 1);
            interpA(cn, var);
            for (int k = 0; k < 7; ++k) c->U[k] = var[k];
            return;
        }
        case FDM_BC_WALL:
        case FDM_BC_DMR_BOTTOM: {  // EXT
            if (kind == FDM_BC_DMR_BOTTOM && c->cx <= S.p.dmr_x0) { set_state(S, c, S.p.dmr_post); return; }
            Grid *cn;
            if (a == -1) cn = ext_image(S, c, 7 - row, col, 3, 0);
            else if (a == -3) cn = ext_image(S, c, 2 * n - 5 - row, col, 3, 0);
            else if (a == -4) cn = ext_image(S, c, row, 7 - col, 4, 0);
            else cn = ext_image(S, c, row, 2 * m - 5 - col, 4, 0);
            interpA(cn, var);
            for (int k = 0; k < 7; ++k) c->U[k] = var[k];
            if (a == -1 || a == -3) c->U[2] = -c->U[2]; else c->U[1] = -c->U[1];
            return;
        }
        case FDM_BC_INFLOW: {  // EXT
            int side = a == -4 ? 0 : a == -2 ? 1 : a == -1 ? 2 : 3;
            set_state(S, c, S.p.bc_state[side]);
            return;
        }
        case FDM_BC_DMR_TOP: {  // EXT: exact oblique shock position on the top boundary
            double xs = S.p.dmr_x0 + c->cy * S.p.dmr_angle_cot + S.p.dmr_shock_speed * t;
            set_state(S, c, c->cx < xs ? S.p.dmr_post : S.p.dmr_pre);
            return;
        }
        default:
            return;
    }
}

static void initial_boundary(Solver &S, Grid *c, double t) {
    if (c->son1) {
        initial_boundary(S, c->son1, t); initial_boundary(S, c->son2, t);
        initial_boundary(S, c->son3, t); initial_boundary(S, c->son4, t);
    } else {
        fill_ghost(S, c, t);
    }
}

static void body_boundary(Solver &S, int j) {                   // :288-293, 314-356
    double t = S.tt;
    if (j == 2) t = S.tt + S.tstep;
    else if (j == 3) t = S.tt + 0.5 * S.tstep;
    const int64_t nb = (int64_t)S.cell_BC.size();
#pragma omp parallel for schedule(dynamic, 64) num_threads(S.nthreads)
    for (int64_t i = 0; i < nb; ++i) fill_ghost(S, S.cell_BC[(size_t)i], t);
}

// ---- initial conditions
static void ic_leaf(Solver &S, Grid *c) {
    const double g = S.gama;
    if (S.ic_kind == 0) {  // vortex, src/solution.F90:31-69
        const double cc = 5.0;
        for (int k = 0; k < 7; ++k) c->U[k] = 0.0;
        double rr = (c->cx - 5.0) * (c->cx - 5.0) + (c->cy - 5.0) * (c->cy - 5.0);
        double dT = -(g - 1.0) * (cc * cc) * std::exp(1.0 - rr) / (8.0 * g * Pi * Pi);
        c->U[0] = 1.0 + std::pow(1.0 + dT, 1.0 / (g - 1.0)) - 1.0;
        c->U[1] = 1.0 - (c->cy - 5.0) * cc / (2.0 * Pi) * std::exp(0.5 * (1.0 - rr));
        c->U[2] = 1.0 + (c->cx - 5.0) * cc / (2.0 * Pi) * std::exp(0.5 * (1.0 - rr));
        c->U[4] = 1.0 + std::pow(1.0 + dT, g / (g - 1.0)) - 1.0;
        c->U[3] = (c->U[4] * g * S.Ma * S.Ma) / c->U[0];
    } else if (S.ic_kind == 1) {  // EXT: four quadrants split at (icp[0], icp[1])
        // icp[2..17] = NE, NW, SW, SE states (rho,u,v,p)
        const bool east = c->cx > S.icp[0], north = c->cy > S.icp[1];
        const int q = north ? (east ? 0 : 1) : (east ? 3 : 2);
        set_state(S, c, &S.icp[2 + 4 * q]);
    } else {  // EXT: oblique shock through (icp[0], 0) at cot = icp[1]
        const double xs = S.icp[0] + c->cy * S.icp[1];
        set_state(S, c, c->cx < xs ? S.p.dmr_post : S.p.dmr_pre);
    }
    for (int k = 0; k < 7; ++k) { c->Ut[k] = c->U[k]; c->Un[k] = c->U[k]; }
    c->rot = 0.0; c->div = 0.0;
}
static void ic_tree(Solver &S, Grid *c) {
    if (c->son1) {
        ic_tree(S, c->son1); ic_tree(S, c->son2); ic_tree(S, c->son3); ic_tree(S, c->son4);
    } else {
        ic_leaf(S, c);
    }
}

static void creat_mesh(Solver &S) {                             // src/mesh.F90:9-47
    S.m = (int)((S.Xmax - S.Xmin) / (S.xf * S.h));
    S.n = (int)((S.Ymax - S.Ymin) / S.h);
    S.nglob = S.n;
    if (S.p.window_rows > 0) {
        S.row0 = S.p.window_row0;
        S.n = S.p.window_rows;
        S.halo_lo = S.p.kind_ymbc == FDM_BC_EXCHANGE;
        S.halo_hi = S.p.kind_ypbc == FDM_BC_EXCHANGE;
    }
    S.total = S.m * S.n;
    S.cell.assign((size_t)S.total, Grid{});
    for (int i = 1; i <= S.total; ++i) {
        Grid *c = S.C(i);
        int ni = (i - 1) / S.m + 1;
        int nj = i - S.m * (ni - 1);
        c->num[0] = ni; c->num[1] = nj;
        c->lvl = 0;
        c->cx = 0.5 * (2.0 * nj - 1.0) * S.xf * S.h + S.Xmin;
        c->cy = ((ni + S.row0) - 0.5) * S.h + S.Ymin;
        c->sp = 0;
        c->sort = 0;
        c->father = nullptr;
        c->cross = gridcross(S, c);
        c->son1 = c->son2 = c->son3 = c->son4 = nullptr;
        c->key = FDM_KEY((uint64_t)(i - 1), 0, 0);
    }
}

// ---- time loop pieces
static void getRKn(Solver &S) {                                 // :372-384
    const int64_t nn = (int64_t)S.cell_NS.size();
#pragma omp parallel for schedule(static) num_threads(S.nthreads)
    for (int64_t i = 0; i < nn; ++i) {
        Grid *c = S.cell_NS[(size_t)i];
        for (int k = 0; k < 7; ++k) c->Un[k] = c->U[k];
    }
}
static void updateRK(Solver &S, int krk) {                      // :386-404
    const double Ra[3] = {0.0, 3.0 / 4.0, 1.0 / 3.0};
    const double Rb[3] = {1.0, 1.0 / 4.0, 2.0 / 3.0};
    const int64_t nn = (int64_t)S.cell_NS.size();
#pragma omp parallel for schedule(static) num_threads(S.nthreads)
    for (int64_t i = 0; i < nn; ++i) {
        Grid *c = S.cell_NS[(size_t)i];
        for (int j = 0; j < S.Neq + 1; ++j) c->U[j] = Ra[krk - 1] * c->Un[j] + Rb[krk - 1] * c->Ut[j];
    }
}
static void solution_cells(Solver &S) {                         // :276-284
    const int64_t nn = (int64_t)S.cell_NS.size();
    S.fu_buf.resize((size_t)nn * 4);
#pragma omp parallel for schedule(dynamic, 16) num_threads(S.nthreads)
    for (int64_t i = 0; i < nn; ++i) solution_cell(S, S.cell_NS[(size_t)i], &S.fu_buf[(size_t)i * 4]);
    for (int i = 0; i < 6; ++i) { S.Res_max[i] = 0.0; S.Res_rms[i] = 0.0; }
    for (int64_t i = 0; i < nn; ++i)
        for (int k = 0; k < 4; ++k) {
            double f = S.fu_buf[(size_t)i * 4 + k];
            if (std::fabs(f) > S.Res_max[k]) S.Res_max[k] = std::fabs(f);
            S.Res_rms[k] = S.Res_rms[k] + f * f;
        }
}
static void time_advance_rk(Solver &S) {                        // :267-298
    getRKn(S);
    for (int krk = 1; krk <= 3; ++krk) {
        solution_cells(S);
        updateRK(S, krk);
        body_boundary(S, 3);
    }
}
static void step_control(Solver &S) {                           // :185-201
    S.l_max = 0;
    for (Grid *c : S.cell_NS) {
        S.lambda_x = std::fmax(S.lambda_x, std::fabs(c->U[1]) + std::sqrt(S.gama * c->U[4] / c->U[0]));
        S.lambda_y = std::fmax(S.lambda_y, std::fabs(c->U[2]) + std::sqrt(S.gama * c->U[4] / c->U[0]));
        S.l_max = std::max(S.l_max, c->lvl);
    }
    if (S.p.iflag_localdt)
        S.tstep = S.p.cfl / (S.lambda_x / (S.xf * S.h / ipow2(S.l_max)) + S.lambda_y / (S.h / ipow2(S.l_max)));
    if (S.tt + S.tstep > S.p.t_end) S.tstep = S.p.t_end - S.tt;
}

// ---- AMR (src/solution.F90:408-589)
static void solute_div_rot(Solver &S, Grid *c) {                // :442-466
    if (!c->son1 && (c->cross == 0 || c->cross == 1)) {
        const double dy = S.h / ipow2(c->lvl);
        const double dx = S.xf * dy;
        double Uip[NVAR], Uim[NVAR], Ujp[NVAR], Ujm[NVAR];
        T1(S, c, D_RIGHT, Uip); T1(S, c, D_LEFT, Uim); T1(S, c, D_UP, Ujp); T1(S, c, D_DOWN, Ujm);
        const double p15 = std::pow(dy, 1.5);
        double vx = (Uip[2] - Uim[2]) / (2.0 * dx), uy = (Ujp[1] - Ujm[1]) / (2.0 * dy);
        c->rot = std::fabs(vx - uy) * p15;
        double ux = (Uip[0] - Uim[0]) / (2.0 * dx), vy = (Ujp[0] - Ujm[0]) / (2.0 * dy);
        c->div = (std::fabs(ux) + std::fabs(vy)) * p15;
        S.Srot = S.Srot + c->rot * c->rot;
        S.Sdiv = S.Sdiv + c->div * c->div;
        S.Ne = S.Ne + 1;
    } else if (c->son1) {
        solute_div_rot(S, c->son1); solute_div_rot(S, c->son2);
        solute_div_rot(S, c->son3); solute_div_rot(S, c->son4);
    }
}
static void rot_div(Solver &S) {                                // :424-440
    S.Srot = 0; S.Sdiv = 0; S.Ne = 0;
    for (int i = 1; i <= S.total; ++i) {
        Grid *c = S.C(i);
        if (c->cross == 0 || c->cross == 1 || c->cross == 2) solute_div_rot(S, c);
    }
}
static void solute_coarse_sub(Solver &S, Grid *c, double arot, double adiv) {  // :490-517
    if (c->son1 && c->lvl < S.p.lvl_amr && !c->son1->son1 && !c->son2->son1 && !c->son3->son1 &&
        !c->son4->son1) {
        if ((c->son1->rot + c->son2->rot + c->son3->rot + c->son4->rot) / 4 < S.p.coarse_goal_rot * arot &&
            (c->son1->div + c->son2->div + c->son3->div + c->son4->div) / 4 < S.p.coarse_goal_div * adiv)
            Coarse_cell(S, c);
    } else if (c->son1) {
        if (c->son1->son1) solute_coarse_sub(S, c->son1, arot, adiv);
        if (c->son2->son1) solute_coarse_sub(S, c->son2, arot, adiv);
        if (c->son3->son1) solute_coarse_sub(S, c->son3, arot, adiv);
        if (c->son4->son1) solute_coarse_sub(S, c->son4, arot, adiv);
    }
}
static void solute_ref_sub(Solver &S, Grid *c, double arot, double adiv) {  // :519-535
    if (!c->son1 && c->lvl < S.p.lvl_amr) {
        if (c->rot > S.p.refine_goal_rot * arot || c->div > S.p.refine_goal_div * adiv) Refine_cell(S, c);
    } else if (c->son1 && c->lvl < S.p.lvl_amr) {
        solute_ref_sub(S, c->son1, arot, adiv); solute_ref_sub(S, c->son2, arot, adiv);
        solute_ref_sub(S, c->son3, arot, adiv); solute_ref_sub(S, c->son4, arot, adiv);
    }
}
static void solute_ref(Solver &S) {                             // :468-488
    double arot = std::sqrt(S.Srot / (double)S.Ne);
    double adiv = std::sqrt(S.Sdiv / (double)S.Ne);
    for (int i = 1; i <= S.total; ++i) {
        Grid *c = S.C(i);
        if (c->cross == 0 || c->cross == 1) solute_ref_sub(S, c, arot, adiv);
        if (c->son1) solute_coarse_sub(S, c, arot, adiv);
    }
}
static void solute_gridmodify(Solver &S) {                      // :537-556
    for (int k = 1; k <= S.p.lvl_amr; ++k) {
        for (int i = 1; i <= S.total; ++i) gridmodify1(S, S.C(i));
        idneighbor(S);
        for (int i = 1; i <= S.total; ++i) gridmodify4(S, S.C(i));
        idneighbor(S);
    }
}
static void amr_core(Solver &S) {                               // :413-419 (body)
    rot_div(S);
    solute_ref(S);
    solute_gridmodify(S);
    idneighbor(S);
    IDgrid(S);
    S.cnt.regrids++;
}
static bool amr_due(const Solver &S) {
    return S.it >= S.p.nstep_adapt && S.p.pstep_adapt != 0 && (S.it % S.p.pstep_adapt) == 1;
}

// one iteration of the solute loop without file output; returns FDM_ERR_NAN
static int solute_step(Solver &S) {                             // :182-236
    S.it = S.it + 1;
    step_control(S);
    time_advance_rk(S);
    S.tt = S.tt + S.tstep;
    const double nres = (double)S.cell_NS.size();
    bool bad = false;
    for (int i = 0; i < S.Neq; ++i) {
        S.Res_rms[i] = std::sqrt(S.Res_rms[i] / (1.0 * nres));
        if (std::isnan(S.Res_rms[i])) bad = true;
    }
    if (bad) return FDM_ERR_NAN;
    if (S.p.iflag_amr) {
        if (amr_due(S)) amr_core(S);
        body_boundary(S, 1);
    }
    return FDM_OK;
}

// ---- snapshot import / export
static void collect_leaves(Grid *c, std::vector<Grid *> &out) {  // key order
    if (c->son1) {
        collect_leaves(c->son1, out); collect_leaves(c->son2, out);
        collect_leaves(c->son4, out); collect_leaves(c->son3, out);
    } else {
        out.push_back(c);
    }
}
static void all_leaves(Solver &S, std::vector<Grid *> &out) {
    out.clear();
    for (int i = 1; i <= S.total; ++i) collect_leaves(S.C(i), out);
}
static void set_internal_means(Grid *c) {
    if (!c->son1) return;
    set_internal_means(c->son1); set_internal_means(c->son2);
    set_internal_means(c->son3); set_internal_means(c->son4);
    double var[NVAR];
    interpA(c, var);
    for (int k = 0; k < 7; ++k) { c->U[k] = var[k]; c->Un[k] = var[k]; c->Ut[k] = var[k]; }
}

static void setup(Solver &S, const fdm_params *p) {
    S.p = *p;
    S.Xmin = p->xmin; S.Xmax = p->xmax; S.Ymin = p->ymin; S.Ymax = p->ymax;
    S.h = p->h; S.xf = p->x_factor; S.gama = p->gama; S.cv = p->cv; S.Ma = p->ma;
    S.tstep = p->tstep;
#ifdef _OPENMP
    S.nthreads = omp_get_max_threads();
#endif
}

}  // namespace orc

// ===================================================================== C API
using namespace orc;
extern "C" {

void *orc_create(const fdm_params *p) {
    Solver *S = new Solver();
    setup(*S, p);
    creat_mesh(*S);
    idneighbor(*S);
    return S;
}
void orc_destroy(void *h) {
    Solver *S = (Solver *)h;
    for (auto &c : S->cell) {
        free_subtree(c.son1); free_subtree(c.son2); free_subtree(c.son3); free_subtree(c.son4);
    }
    delete S;
}
void orc_set_threads(void *h, int n) { ((Solver *)h)->nthreads = n > 0 ? n : 1; }
int orc_mesh_dims(void *h, int *m, int *n) {
    Solver *S = (Solver *)h;
    *m = S->m; *n = S->n;
    return 0;
}
// creat_mesh's Block_refine (src/mesh.F90:41-44), before initial
int orc_block_refine(void *h, int lvlblock, const double *box, int buffer_layer_lvl) {
    Solver *S = (Solver *)h;
    if (lvlblock < 0 || lvlblock > FDM_LMAX) return FDM_ERR_ARG;
    BlockSpec B;
    B.lvlblock = lvlblock;
    for (int k = 0; k < 4; ++k) B.box[k] = box[k];
    for (int i = 1; i <= lvlblock; ++i) B.refinesize[i] = (double)buffer_layer_lvl * S->h / (double)(1LL << (i - 1));
    Block_refine(*S, B);
    idneighbor(*S);
    return 0;
}
// initial (src/solution.F90:9-29) + IDgrid; kind 0 vortex, 1 quadrants, 2
// oblique shock.  Internal nodes of a
// block-refined mesh are left unset by the reference (allocated, never
// assigned); here they take the interpA mean, as after an upload.
int orc_initial(void *h, int kind, const double *icp, int nicp) {
    Solver *S = (Solver *)h;
    S->ic_kind = kind;
    for (int i = 0; i < nicp && i < 32; ++i) S->icp[i] = icp[i];
    for (int i = 1; i <= S->total; ++i) ic_tree(*S, S->C(i));
    for (int i = 1; i <= S->total; ++i) set_internal_means(S->C(i));
    for (int i = 1; i <= S->total; ++i) initial_boundary(*S, S->C(i), S->tt);
    IDgrid(*S);
    return 0;
}
int64_t orc_num_leaves(void *h) {
    std::vector<Grid *> v;
    all_leaves(*(Solver *)h, v);
    return (int64_t)v.size();
}
int64_t orc_num_interior(void *h) { return (int64_t)((Solver *)h)->cell_NS.size(); }
// keys, prim (rho,u,v,p) and T of every leaf in key order
int orc_export_leaves(void *h, int64_t cap, uint64_t *keys, double *prim, double *T) {
    Solver *S = (Solver *)h;
    std::vector<Grid *> v;
    all_leaves(*S, v);
    if ((int64_t)v.size() > cap) return FDM_ERR_ARG;
    for (size_t i = 0; i < v.size(); ++i) {
        Grid *c = v[i];
        if (keys) keys[i] = c->key;
        if (prim) { prim[4 * i] = c->U[0]; prim[4 * i + 1] = c->U[1]; prim[4 * i + 2] = c->U[2]; prim[4 * i + 3] = c->U[4]; }
        if (T) T[i] = c->U[3];
    }
    return 0;
}
// rebuild the tree from a leaf set; internal nodes get interpA means
int orc_import_leaves(void *h, int64_t n, const uint64_t *keys, const double *prim) {
    Solver *S = (Solver *)h;
    for (auto &c : S->cell) {
        free_subtree(c.son1); free_subtree(c.son2); free_subtree(c.son3); free_subtree(c.son4);
        c.son1 = c.son2 = c.son3 = c.son4 = nullptr;
    }
    for (int64_t i = 0; i < n; ++i) {
        uint64_t k = keys[i];
        uint64_t r = FDM_KEY_ROOT(k);
        uint32_t l = FDM_KEY_LVL(k);
        uint64_t path = FDM_KEY_PATH(k);
        if ((int64_t)r >= S->total || l > FDM_LMAX) return FDM_ERR_ARG;
        Grid *c = S->C((int)r + 1);
        for (uint32_t j = 1; j <= l; ++j) {
            if (!c->son1) Refine_cell(*S, c);
            int q = (int)((path >> (2 * (FDM_LMAX - j))) & 3u);
            c = q == 0 ? c->son1 : q == 1 ? c->son2 : q == 3 ? c->son3 : c->son4;
        }
        if (c->son1) return FDM_ERR_ARG;  // overlapping leaves
        const double st[4] = {prim[4 * i], prim[4 * i + 1], prim[4 * i + 2], prim[4 * i + 3]};
        set_state(*S, c, st);
        for (int q = 0; q < 7; ++q) { c->Ut[q] = c->U[q]; c->Un[q] = c->U[q]; }
        c->rot = 0.0; c->div = 0.0;
    }
    for (int i = 1; i <= S->total; ++i) set_internal_means(S->C(i));
    idneighbor(*S);
    IDgrid(*S);
    return 0;
}
// overwrite T (slot 4) of every leaf in key order (T is dead state)
int orc_set_T(void *h, int64_t n, const double *T) {
    Solver *S = (Solver *)h;
    std::vector<Grid *> v;
    all_leaves(*S, v);
    if ((int64_t)v.size() != n) return FDM_ERR_ARG;
    for (size_t i = 0; i < v.size(); ++i) v[i]->U[3] = T[i];
    return 0;
}
// scalars: lambda_x, lambda_y, tstep, tt, it, l_max, Res_max[4], Res_rms[4]
int orc_get_scalars(void *h, double *out) {
    Solver *S = (Solver *)h;
    out[0] = S->lambda_x; out[1] = S->lambda_y; out[2] = S->tstep; out[3] = S->tt;
    out[4] = (double)S->it; out[5] = S->l_max;
    for (int i = 0; i < 4; ++i) { out[6 + i] = S->Res_max[i]; out[10 + i] = S->Res_rms[i]; }
    out[14] = S->Srot; out[15] = S->Sdiv; out[16] = (double)S->Ne;
    return 0;
}
int orc_set_scalars(void *h, double lx, double ly, double tstep, double tt, int64_t it) {
    Solver *S = (Solver *)h;
    S->lambda_x = lx; S->lambda_y = ly; S->tstep = tstep; S->tt = tt; S->it = it;
    return 0;
}
int orc_step_control(void *h) { step_control(*(Solver *)h); return 0; }
// the step of src/solution.F90:195-201 from maxima taken over all strips
int orc_step_control_global(void *h, double lx, double ly, int l_max) {
    Solver &S = *(Solver *)h;
    S.lambda_x = lx; S.lambda_y = ly; S.l_max = l_max;
    if (S.p.iflag_localdt)
        S.tstep = S.p.cfl / (S.lambda_x / (S.xf * S.h / ipow2(S.l_max)) + S.lambda_y / (S.h / ipow2(S.l_max)));
    if (S.tt + S.tstep > S.p.t_end) S.tstep = S.p.t_end - S.tt;
    return 0;
}
// U(1:7) of the leaves idx[] (key order) out / in: the halo exchange of strips
int orc_get_U(void *h, int64_t n, const int64_t *idx, double *out) {
    Solver &S = *(Solver *)h;
    std::vector<Grid *> v;
    all_leaves(S, v);
    for (int64_t i = 0; i < n; ++i) {
        if (idx[i] < 0 || idx[i] >= (int64_t)v.size()) return FDM_ERR_ARG;
        for (int k = 0; k < 7; ++k) out[7 * i + k] = v[(size_t)idx[i]]->U[k];
    }
    return 0;
}
int orc_set_U(void *h, int64_t n, const int64_t *idx, const double *in) {
    Solver &S = *(Solver *)h;
    std::vector<Grid *> v;
    all_leaves(S, v);
    for (int64_t i = 0; i < n; ++i) {
        if (idx[i] < 0 || idx[i] >= (int64_t)v.size()) return FDM_ERR_ARG;
        for (int k = 0; k < 7; ++k) v[(size_t)idx[i]]->U[k] = in[7 * i + k];
    }
    return 0;
}
int orc_time_advance_rk(void *h) { time_advance_rk(*(Solver *)h); return 0; }
int orc_stage(void *h, int krk) {
    Solver *S = (Solver *)h;
    if (krk == 1) getRKn(*S);
    solution_cells(*S);
    updateRK(*S, krk);
    body_boundary(*S, 3);
    return 0;
}
int orc_solute_step(void *h) { return solute_step(*(Solver *)h); }
int orc_body_boundary(void *h, int j) { body_boundary(*(Solver *)h, j); return 0; }
int orc_solute(void *h, int64_t nsteps, int64_t *done) {
    Solver *S = (Solver *)h;
    int64_t k = 0;
    int rc = 0;
    while (S->tt < S->p.t_end && k < nsteps) {
        rc = solute_step(*S);
        ++k;
        if (rc) break;
    }
    if (done) *done = k;
    return rc;
}
int orc_amr(void *h) {
    Solver *S = (Solver *)h;
    if (S->p.window_rows > 0) return FDM_ERR_UNSUPPORTED;
    amr_core(*S);
    body_boundary(*S, 1);
    return 0;
}
int orc_rot_div(void *h) { rot_div(*(Solver *)h); return 0; }
// rot/div of the interior leaves in key order
int orc_export_rot_div(void *h, int64_t cap, double *rot, double *div) {
    Solver *S = (Solver *)h;
    if ((int64_t)S->cell_NS.size() > cap) return FDM_ERR_ARG;
    for (size_t i = 0; i < S->cell_NS.size(); ++i) { rot[i] = S->cell_NS[i]->rot; div[i] = S->cell_NS[i]->div; }
    return 0;
}
// 8 stencil values x (rho,u,v,p) per interior leaf, current U
int orc_export_stencil(void *h, int64_t cap, double *out) {
    Solver *S = (Solver *)h;
    const int64_t nn = (int64_t)S->cell_NS.size();
    if (nn > cap) return FDM_ERR_ARG;
#pragma omp parallel for schedule(dynamic, 16) num_threads(S->nthreads)
    for (int64_t i = 0; i < nn; ++i) {
        Stencil st;
        fetch_stencil(*S, S->cell_NS[(size_t)i], st);
        for (int s = 0; s < 8; ++s) {
            out[(i * 8 + s) * 4 + 0] = st.v[s][0];
            out[(i * 8 + s) * 4 + 1] = st.v[s][1];
            out[(i * 8 + s) * 4 + 2] = st.v[s][2];
            out[(i * 8 + s) * 4 + 3] = st.v[s][4];
        }
    }
    return 0;
}
// hanging-node stencils of every interior leaf and entry (Tip, Tim, Tjp, Tjm,
// Tipp, Timm, Tjpp, Tjmm): kind (GatherRec), node key, target, m1/m2 and
// up to 16 member keys
int orc_export_gather(void *h, int64_t cap, int32_t *kind, uint64_t *node, double *xy, int32_t *m12,
                      uint64_t *mem) {
    Solver *S = (Solver *)h;
    const int64_t nn = (int64_t)S->cell_NS.size();
    if (nn > cap) return FDM_ERR_ARG;
    for (int64_t i = 0; i < nn; ++i) {
        Grid *c = S->cell_NS[(size_t)i];
        for (int e = 0; e < 8; ++e) {
            GatherRec r{};
            tl_rec = &r;
            double var[NVAR];
            const int d = e % 4 == 0 ? D_RIGHT : e % 4 == 1 ? D_LEFT : e % 4 == 2 ? D_UP : D_DOWN;
            if (e < 4) T1(*S, c, d, var); else T2(*S, c, d, var);
            tl_rec = nullptr;
            const int64_t o = i * 8 + e;
            kind[o] = r.kind; node[o] = r.node; xy[2 * o] = r.xx; xy[2 * o + 1] = r.yy;
            m12[2 * o] = r.m1; m12[2 * o + 1] = r.m2;
            for (int k = 0; k < 16; ++k) mem[o * 16 + k] = k < r.m1 + r.m2 ? r.mem[k] : ~0ull;
        }
    }
    return 0;
}

// cached neighbour keys per leaf (key order): up, down, right, left,
// upleft, upright, downleft, downright; ~0 for null
int orc_export_neighbors(void *h, int64_t cap, uint64_t *out) {
    Solver *S = (Solver *)h;
    std::vector<Grid *> v;
    all_leaves(*S, v);
    if ((int64_t)v.size() > cap) return FDM_ERR_ARG;
    for (size_t i = 0; i < v.size(); ++i) {
        Grid *c = v[i];
        Grid *nb[8] = {c->upnei, c->downnei, c->rightnei, c->leftnei,
                       c->upleftnei, c->uprightnei, c->downleftnei, c->downrightnei};
        for (int d = 0; d < 8; ++d) out[i * 8 + d] = nb[d] ? nb[d]->key : ~0ull;
    }
    return 0;
}
// counters: singular, wls_calls, parent_interp, child_copy, gm4_nonleaf, regrids
int orc_counters(void *h, int64_t *out) {
    Solver *S = (Solver *)h;
    out[0] = S->cnt.singular; out[1] = S->cnt.wls_calls; out[2] = S->cnt.parent_interp;
    out[3] = S->cnt.child_copy; out[4] = S->cnt.gm4_nonleaf; out[5] = S->cnt.regrids;
    return 0;
}
// residual of the last stage (after orc_solute_step the rms is the sqrt form)
int orc_residual(void *h, double *rmax, double *rrms) {
    Solver *S = (Solver *)h;
    for (int i = 0; i < 4; ++i) { rmax[i] = S->Res_max[i]; rrms[i] = S->Res_rms[i]; }
    return 0;
}

// ---- numerics entry points for known-answer tests
void orc_wcns_z3(const double *u1, const double *u2, const double *u3, const double *R16,
                 double *hp) {
    double R[4][4];
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) R[r][c] = R16[r * 4 + c];
    WCNS_Z3(u1, u2, u3, R, hp);
}
void orc_eigen(double gama, int dir, const double *U4, double *R16, double *Ri16) {
    Solver S;
    S.gama = gama;
    double R[4][4], Ri[4][4];
    eigen(S, dir, U4, R, Ri);
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) { R16[r * 4 + c] = R[r][c]; Ri16[r * 4 + c] = Ri[r][c]; }
}
int orc_brinv(int n, double *a) {
    if (n == 3) {
        double r[3][3];
        for (int i = 0; i < 9; ++i) r[i / 3][i % 3] = a[i];
        bool ok = brinv<3>(r, nullptr);
        for (int i = 0; i < 9; ++i) a[i] = r[i / 3][i % 3];
        return ok ? 0 : 1;
    }
    if (n == 6) {
        double r[6][6];
        for (int i = 0; i < 36; ++i) r[i / 6][i % 6] = a[i];
        bool ok = brinv<6>(r, nullptr);
        for (int i = 0; i < 36; ++i) a[i] = r[i / 6][i % 6];
        return ok ? 0 : 1;
    }
    return -1;
}
int orc_get_direction(double xx, double yy, double x, double y) { return get_direction(xx, yy, x, y); }
// flux difference of one direction for a 5-point primitive stencil
// st[5][4] (rho,u,v,p), lambda; dir 0 = x, 1 = y
void orc_lxl_dir(double gama, int dir, double lam, double dxy, const double *st20, double *out4) {
    Solver S;
    S.gama = gama;
    S.lambda_x = lam; S.lambda_y = lam;
    double v[5][NVAR];
    const double *p[5];
    for (int c = 0; c < 5; ++c) {
        v[c][0] = st20[c * 4]; v[c][1] = st20[c * 4 + 1]; v[c][2] = st20[c * 4 + 2];
        v[c][3] = QNAN; v[c][4] = st20[c * 4 + 3];
        p[c] = v[c];
    }
    lxl_dir(S, dir, dxy, p, out4);
}
// WLS-WENO with explicit stencil: xs, ys, vals[m][4] (rho,u,v,p), m1 axis
// points first; node level/centre for the smoothness box.
int orc_wls(double h, double xf, int lvl, double cx, double cy, double xx, double yy, int m1, int m2,
            const double *xs, const double *ys, const double *vals, double *out4) {
    Solver S;
    S.h = h; S.xf = xf;
    std::vector<Grid> g((size_t)(m1 + m2));
    NList n1, n2;
    for (int i = 0; i < m1 + m2; ++i) {
        g[(size_t)i] = Grid{};
        g[(size_t)i].cx = xs[i]; g[(size_t)i].cy = ys[i];
        g[(size_t)i].U[0] = vals[4 * i]; g[(size_t)i].U[1] = vals[4 * i + 1];
        g[(size_t)i].U[2] = vals[4 * i + 2]; g[(size_t)i].U[4] = vals[4 * i + 3];
        if (i < m1) n1.a[n1.n++] = &g[(size_t)i]; else n2.a[n2.n++] = &g[(size_t)i];
    }
    Grid node{};
    node.lvl = lvl; node.cx = cx; node.cy = cy;
    double var[NVAR];
    WLSI_US_WENO(S, &node, xx, yy, n1, n2, var);
    out4[0] = var[0]; out4[1] = var[1]; out4[2] = var[2]; out4[3] = var[4];
    return (int)S.cnt.singular;
}

}  // extern "C"
