"""Pure-Python transliteration of the reference numerics, written directly
from the Fortran (src/nnd_center_RK.F90, src/XuanGua.F90) and independently
of the C++ oracle, used to cross-check it bit for bit.  Python floats are
IEEE binary64 without FMA contraction; every expression below keeps the
Fortran's left-to-right order, and MATMUL/SUM accumulate from 0.0.
Arrays are 1-based as in the Fortran (index 0 unused)."""
import math

import numpy as np

EPS40 = float(np.float32(1e-40))
D1 = float(np.float32(1.0) / np.float32(11.0))
D2 = float(np.float32(10.0) / np.float32(11.0))
BIAS = float(np.float32(1e-10))
PI = 3.1415926535897932


def wcns_z3(u1, u2, u3, R):
    """WCNS_Z3 (src/nnd_center_RK.F90:310-353); u* and R 1-based."""
    uL = [0.0] * 5
    for i in range(1, 5):
        IS1 = (-u1[i] + u2[i]) ** 2
        IS2 = (-u2[i] + u3[i]) ** 2
        IS3 = (u1[i] - 2. * u2[i] + u3[i]) ** 2
        d1, d2 = D1, D2
        p1 = u2[i]
        p2 = ((-u1[i] + 6.0 * u2[i] + 3.0 * u3[i]) / 8.0 - d1 * p1) / d2
        IS1 = min(IS1, IS2)
        IS2 = IS3 + u1[i] ** 2 + u2[i] ** 2 + u3[i] ** 2 - u1[i] * u2[i] - u2[i] * u3[i] - u1[i] * u3[i]
        tau3 = (10. * abs(IS2 - 3. * IS1)) ** 2
        a1 = d1 * (1.0 + tau3 / (EPS40 + IS1))
        a2 = d2 * (1.0 + tau3 / (EPS40 + IS2))
        w1 = a1 / (a1 + a2)
        w2 = a2 / (a1 + a2)
        uL[i] = w1 * p1 + w2 * p2
    hp = [0.0] * 5
    for r in range(1, 5):
        hp[r] = R[r][1] * uL[1] + R[r][2] * uL[2] + R[r][3] * uL[3] + R[r][4] * uL[4]
    return hp


def _mat(n):
    return [[0.0] * (n + 1) for _ in range(n + 1)]


def eigen(gama, direction, U):
    """REcalc (direction 0) / RFcalc (direction 1), U 1-based conserved."""
    U0 = [0.0] * 6
    U0[1] = U[1]
    U0[2] = U[2] / U[1]
    U0[3] = U[3] / U[1]
    U0[5] = (gama - 1.0) * U0[1] * (U[4] / U0[1] - 0.5 * (U0[2] * U0[2] + U0[3] * U0[3]))
    a = math.sqrt(gama * U0[5] / U0[1])
    q2 = 0.5 * (U0[2] * U0[2] + U0[3] * U0[3])
    R, Ri = _mat(4), _mat(4)
    u, v = U0[2], U0[3]
    if direction == 0:
        R[1][1] = 1.0; R[2][1] = u - a; R[3][1] = v; R[4][1] = a * a / (gama - 1) + q2 - u * a
        R[1][2] = 1.0; R[2][2] = u; R[3][2] = v; R[4][2] = q2
        R[1][3] = 1.0; R[2][3] = u + a; R[3][3] = v; R[4][3] = a * a / (gama - 1) + q2 + u * a
        R[1][4] = 0.0; R[2][4] = 0.0; R[3][4] = -1.0; R[4][4] = -v
        Ri[1][1] = ((gama - 1.0) * q2 + a * u) / (2.0 * a * a)
        Ri[2][1] = (a * a - (gama - 1.0) * q2) / (a * a)
        Ri[3][1] = ((gama - 1.0) * q2 - a * u) / (2.0 * a * a)
        Ri[4][1] = v
        Ri[1][2] = ((1.0 - gama) * u - a) / (2.0 * a * a)
        Ri[2][2] = ((gama - 1.0) * u) / (a * a)
        Ri[3][2] = ((1.0 - gama) * u + a) / (2.0 * a * a)
        Ri[4][2] = 0.0
        Ri[1][3] = ((1.0 - gama) * v) / (2.0 * a * a)
        Ri[2][3] = ((gama - 1.0) * v) / (a * a)
        Ri[3][3] = ((1.0 - gama) * v) / (2.0 * a * a)
        Ri[4][3] = -1.0
    else:
        R[1][1] = 1.0; R[2][1] = u; R[3][1] = v - a; R[4][1] = a * a / (gama - 1) + q2 - v * a
        R[1][2] = 1.0; R[2][2] = u; R[3][2] = v; R[4][2] = q2
        R[1][3] = 1.0; R[2][3] = u; R[3][3] = v + a; R[4][3] = a * a / (gama - 1) + q2 + v * a
        R[1][4] = 0.0; R[2][4] = 1.0; R[3][4] = 0.0; R[4][4] = u
        Ri[1][1] = ((gama - 1.0) * q2 + a * v) / (2.0 * a * a)
        Ri[2][1] = (a * a - (gama - 1.0) * q2) / (a * a)
        Ri[3][1] = ((gama - 1.0) * q2 - a * v) / (2.0 * a * a)
        Ri[4][1] = -u
        Ri[1][2] = ((1.0 - gama) * u) / (2.0 * a * a)
        Ri[2][2] = ((gama - 1.0) * u) / (a * a)
        Ri[3][2] = ((1.0 - gama) * u) / (2.0 * a * a)
        Ri[4][2] = 1.0
        Ri[1][3] = ((1.0 - gama) * v - a) / (2.0 * a * a)
        Ri[2][3] = ((gama - 1.0) * v) / (a * a)
        Ri[3][3] = ((1.0 - gama) * v + a) / (2.0 * a * a)
        Ri[4][3] = 0.0
    Ri[1][4] = (gama - 1.0) / (2.0 * a * a)
    Ri[2][4] = (1.0 - gama) / (a * a)
    Ri[3][4] = (gama - 1.0) / (2.0 * a * a)
    Ri[4][4] = 0.0
    return R, Ri


def lxl_dir(gama, direction, lam, dxy, st):
    """LXL_X_wcns3 / LXL_Y_wcns3 for a 5-point primitive stencil st[k] =
    (rho,u,v,p), k = 0..4 (Uimm, Uim, c, Uip, Uipp)."""
    Uc = [[0.0] * 6 for _ in range(5)]  # Uc[var][col]
    Fn = [[0.0] * 6 for _ in range(5)]
    for c in range(1, 6):
        r, u, v, p = st[c - 1]
        Uc[1][c] = r
        Uc[2][c] = r * u
        Uc[3][c] = r * v
        Uc[4][c] = p / (gama - 1.0) + 0.5 * r * (u * u + v * v)
        if direction == 0:
            Fn[1][c] = r * u
            Fn[2][c] = r * u * u + p
            Fn[3][c] = r * u * v
            Fn[4][c] = u * (p / (gama - 1.0) + 0.5 * r * (u * u + v * v) + p)
        else:
            Fn[1][c] = r * v
            Fn[2][c] = r * u * v
            Fn[3][c] = r * v * v + p
            Fn[4][c] = v * (p / (gama - 1.0) + 0.5 * r * (u * u + v * v) + p)

    def matmul(Ri, X):
        W = [[0.0] * 6 for _ in range(5)]
        for r in range(1, 5):
            for c in range(1, 6):
                s = 0.0
                for k in range(1, 5):
                    s = s + Ri[r][k] * X[k][c]
                W[r][c] = s
        return W

    def col(W, c):
        return [0.0] + [W[r][c] for r in range(1, 5)]

    fl = {}
    for face, (a, b) in ((0, (2, 3)), (1, (3, 4))):
        Um = [0.0] + [(Uc[r][a] + Uc[r][b]) / 2.0 for r in range(1, 5)]
        R, Ri = eigen(gama, direction, Um)
        w = matmul(Ri, Uc)
        g = matmul(Ri, Fn)
        o = face
        wL = wcns_z3(col(w, 1 + o), col(w, 2 + o), col(w, 3 + o), R)
        wR = wcns_z3(col(w, 4 + o), col(w, 3 + o), col(w, 2 + o), R)
        gL = wcns_z3(col(g, 1 + o), col(g, 2 + o), col(g, 3 + o), R)
        gR = wcns_z3(col(g, 4 + o), col(g, 3 + o), col(g, 2 + o), R)
        fl[face] = [0.0] + [0.5 * (gL[r] + gR[r] - lam * (wR[r] - wL[r])) for r in range(1, 5)]
    out = []
    for n in range(1, 5):
        if direction == 0:
            out.append(4.0 / (3.0 * dxy) * (fl[1][n] - fl[0][n]) - 1.0 / (6.0 * dxy) * (Fn[n][4] - Fn[n][2]))
        else:
            out.append(4.0 / 3.0 / dxy * (fl[1][n] - fl[0][n]) - 1.0 / 6.0 / dxy * (Fn[n][4] - Fn[n][2]))
    return out


def brinv(a):
    """brinv (src/XuanGua.F90:593-660); a is an n x n list (0-based storage,
    loops follow the Fortran's 1-based ones)."""
    n = len(a)
    r = [list(map(float, row)) for row in a]
    is_, js = [0] * n, [0] * n
    for k in range(n):
        d = 0.0
        for i in range(k, n):
            for j in range(k, n):
                if abs(r[i][j]) > d:
                    d = abs(r[i][j]); is_[k] = i; js[k] = j
        if d + 1.0 == 1.0:
            return r, False
        for j in range(n):
            r[k][j], r[is_[k]][j] = r[is_[k]][j], r[k][j]
        for i in range(n):
            r[i][k], r[i][js[k]] = r[i][js[k]], r[i][k]
        r[k][k] = 1 / r[k][k]
        for j in range(n):
            if j != k:
                r[k][j] = r[k][j] * r[k][k]
        for i in range(n):
            if i != k:
                for j in range(n):
                    if j != k:
                        r[i][j] = r[i][j] - r[i][k] * r[k][j]
        for i in range(n):
            if i != k:
                r[i][k] = -r[i][k] * r[k][k]
    for k in range(n - 1, -1, -1):
        for j in range(n):
            r[k][j], r[js[k]][j] = r[js[k]][j], r[k][j]
        for i in range(n):
            r[i][k], r[i][is_[k]] = r[i][is_[k]], r[i][k]
    return r, True


def get_direction(xx, yy, x, y):
    dx = xx - x
    dy = yy - y
    angle = (math.atan2(dy, dx) + BIAS) * 180.0 / PI
    return int(math.floor((angle + 22.5) / 45.0 + 8)) % 8 + 1


def wlsi(h, xf, lvl, cx, cy, xx, yy, m1, m2, xs, ys, vals):
    """WLSI_US_WENO (src/XuanGua.F90:179-356) for variables rho,u,v,p."""
    m = m1 + m2
    eps = 1.e-6
    d = [math.sqrt((xs[i] - xx) ** 2 + (ys[i] - yy) ** 2) for i in range(m)]
    w = [1.0 / (d[i] + eps) for i in range(m)]
    P = [[1.0, xs[i], ys[i], xs[i] * ys[i], xs[i] * xs[i], ys[i] * ys[i]] for i in range(m)]

    def ptwp(rows, ncol):
        M = [[0.0] * ncol for _ in range(ncol)]
        for a in range(ncol):
            for b in range(ncol):
                s = 0.0
                for i in rows:
                    wp = 0.0
                    for k in range(m):  # W_Matrix(i,k) * P(k,b)
                        wp = wp + (w[i] if k == i else 0.0) * P[k][b]
                    s = s + P[i][a] * wp
                M[a][b] = s
        return M

    L, _ = brinv(ptwp(range(m), 6))
    A, _ = brinv(ptwp(range(m1), 3))
    B, _ = brinv(ptwp(range(m1, m), 3))
    hx = xf * h / 2.0 ** (lvl + 1)
    hy = h / 2.0 ** (lvl + 1)
    x_min, x_max, y_min, y_max = cx - hx, cx + hx, cy - hy, cy + hy

    def isp(k):
        term1 = k[0] ** 2 * (x_max - x_min) * (y_max - y_min)
        term2 = 2 * k[0] * k[1] * (x_max ** 2 - x_min ** 2) / 2 * (y_max - y_min) + \
            2 * k[0] * k[2] * (x_max - x_min) * (y_max ** 2 - y_min ** 2) / 2
        term3 = k[1] ** 2 * (x_max * x_max * x_max - x_min * x_min * x_min) / 3 * (y_max - y_min) + \
            2 * k[1] * k[2] * (x_max ** 2 - x_min ** 2) / 2 * (y_max ** 2 - y_min ** 2) / 2 + \
            k[2] ** 2 * (x_max - x_min) * (y_max * y_max * y_max - y_min * y_min * y_min) / 3
        return term1 + term2 + term3

    def smooth(c, order):
        if order == 2:
            a1, a2, a3, a4, a5 = c[1], c[2], c[3], c[4], c[5]
            beta = 0.0
            beta = beta + isp([a1, 2 * a3, a4])
            beta = beta + isp([a2, a4, 2 * a5])
            beta = beta + (2 * a3) ** 2 * (x_max - x_min) * (y_max - y_min)
            beta = beta + a4 ** 2 * (x_max - x_min) * (y_max - y_min)
            beta = beta + (2 * a5) ** 2 * (x_max - x_min) * (y_max - y_min)
            return beta
        return (c[1] ** 2 + c[2] ** 2) * (x_max - x_min) * (y_max - y_min)

    lw = [0.98, 0.01, 0.01]
    out = []
    for k in range(4):
        phi = [vals[i][k] for i in range(m)]
        wphi = [w[i] * phi[i] for i in range(m)]

        def solve(M, rows, ncol):
            pt = []
            for a in range(ncol):
                s = 0.0
                for i in rows:
                    s = s + P[i][a] * wphi[i]
                pt.append(s)
            res = []
            for a in range(ncol):
                s = 0.0
                for b in range(ncol):
                    s = s + M[a][b] * pt[b]
                res.append(s)
            return res

        arr = solve(L, range(m), 6)
        vl = arr[0] + xx * arr[1] + yy * arr[2] + xx * yy * arr[3] + xx * xx * arr[4] + yy * yy * arr[5]
        c1 = solve(A, range(m1), 3)
        c2 = solve(B, range(m1, m), 3)
        vs1 = c1[0] + xx * c1[1] + yy * c1[2]
        vs2 = c2[0] + xx * c2[1] + yy * c2[2]
        beta = [smooth(arr, 2), smooth(c1, 1), smooth(c2, 1)]
        sa = 0.0
        sa = sa + abs(beta[0] - beta[1])
        sa = sa + abs(beta[0] - beta[2])
        tau = (sa / 2.0) ** 2
        alpha = [lw[q] * (1.0 + tau / (eps + beta[q])) for q in range(3)]
        s = 0.0
        for q in range(3):
            s = s + alpha[q]
        om = [alpha[q] / s for q in range(3)]
        out.append(om[0] * (1.0 / lw[0] * vl - (lw[1] / lw[0] * vs1 + lw[2] / lw[0] * vs2)) +
                   (om[1] * vs1 + om[2] * vs2))
    return out
