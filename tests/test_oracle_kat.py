"""Known-answer tests of the oracle (CPU restatement of the reference).

The reference ships no tests or golden vectors, so the oracle is checked
against the mathematics (linear reproduction, eigenvector inverses, LU
inverse, uniform-flow preservation, the exact vortex) and, bit for bit,
against an independent pure-Python transliteration (tests/refnum.py)."""
import math

import numpy as np
import pytest

import refnum
from fdm_cell_based_amr_cartesian_b200 import params as P

G14 = P.f32(1.4)


def test_literal_promotions():
    assert G14 == 1.399999976158142
    assert refnum.EPS40 == 9.99994610111476e-41
    assert refnum.D1 == 0.09090909361839294 and refnum.D2 == 0.9090909361839294
    assert refnum.D1 + refnum.D2 != 1.0


def test_wcns_linear_reproduction(oracle_mod):
    """On linear data the Z-weights are the linear ones; because d1 = 1./11.
    and d2 = 10./11. are REAL(4) literals, d1 + d2 = 1 + 3e-8 and the
    normalised weights give the linear interpolant divided by d1 + d2."""
    rng = np.random.default_rng(0)
    R = np.eye(4)
    for _ in range(50):
        a, b = rng.uniform(-2, 2, 4), rng.uniform(-1, 1, 4)
        u1, u2, u3 = a, a + b, a + 2 * b
        hp = oracle_mod.wcns_z3(u1, u2, u3, R)
        lin = (-u1 + 6 * u2 + 3 * u3) / 8
        np.testing.assert_allclose(hp, lin / (refnum.D1 + refnum.D2), rtol=1e-13, atol=1e-13)
        assert np.max(np.abs(hp - lin) / np.abs(lin)) < 4e-8


@pytest.mark.parametrize("direction", [0, 1])
def test_eigenvectors_inverse(oracle_mod, direction):
    rng = np.random.default_rng(1)
    for _ in range(50):
        rho, u, v, p = rng.uniform(0.2, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.2, 2)
        U = np.array([rho, rho * u, rho * v, p / (G14 - 1) + 0.5 * rho * (u * u + v * v)])
        R, Ri = oracle_mod.eigen(G14, direction, U)
        np.testing.assert_allclose(R @ Ri, np.eye(4), atol=1e-12)


@pytest.mark.parametrize("n", [3, 6])
def test_brinv_matches_lu_inverse(oracle_mod, n):
    rng = np.random.default_rng(2)
    for _ in range(20):
        M = rng.normal(size=(n, n))
        A = M @ M.T + n * np.eye(n)
        inv, ok = oracle_mod.brinv(A)
        assert ok
        np.testing.assert_allclose(inv, np.linalg.inv(A), rtol=1e-10, atol=1e-12)


def test_brinv_singular_flag(oracle_mod):
    A = np.array([[1.0, 2.0, 3.0], [2.0, 4.0, 6.0], [1.0, 0.0, 1.0]])
    _, ok = oracle_mod.brinv(A)
    assert not ok


def test_get_direction_bins(oracle_mod):
    pts = [(1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0), (-1, -1), (0, -1), (1, -1)]
    for k, (dx, dy) in enumerate(pts):
        assert oracle_mod.get_direction(dx, dy, 0.0, 0.0) == k + 1
        assert refnum.get_direction(dx, dy, 0.0, 0.0) == k + 1


def test_wls_reproduces_linear_fields(oracle_mod):
    # 5 axis points (centre + 4) and 4 diagonal points around a coarse cell
    h, lvl, cx, cy = 0.5, 0, 2.25, 3.75
    xs = [cx, cx - h, cx + h, cx, cx] + [cx - h, cx + h, cx - h, cx + h]
    ys = [cy, cy, cy, cy - h, cy + h] + [cy - h, cy - h, cy + h, cy + h]
    f = lambda x, y: np.array([1 + 0.3 * x - 0.2 * y, 0.5 - 0.1 * x, 0.2 * y, 2 + 0.05 * x + 0.07 * y])
    vals = np.array([f(x, y) for x, y in zip(xs, ys)])
    xx, yy = cx + h / 4, cy - h / 4
    out, nsing = oracle_mod.wls(h, 1.0, lvl, cx, cy, xx, yy, 5, 4, xs, ys, vals)
    assert nsing == 0
    np.testing.assert_allclose(out, f(xx, yy), rtol=1e-9, atol=1e-9)


def _rand_state(rng):
    return (rng.uniform(0.2, 2.0), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.2, 2.0))


def test_python_transliteration_bitwise(oracle_mod):
    """C++ oracle == independent Python transliteration, bit for bit."""
    rng = np.random.default_rng(3)
    for _ in range(30):
        st = np.array([_rand_state(rng) for _ in range(5)])
        # occasionally a discontinuity
        if rng.uniform() < 0.5:
            st[3:] *= rng.uniform(2, 5)
        lam = rng.uniform(1, 4)
        for d in (0, 1):
            a = oracle_mod.lxl_dir(G14, d, lam, 0.125, st)
            b = refnum.lxl_dir(G14, d, lam, 0.125, [tuple(r) for r in st])
            assert list(a) == b, (d, a, b)
    for _ in range(20):
        for n in (3, 6):
            M = rng.normal(size=(n, n))
            A = M @ M.T + 0.1 * np.eye(n)
            inv, ok = oracle_mod.brinv(A)
            inv2, ok2 = refnum.brinv(A.tolist())
            assert ok == ok2 and inv.tolist() == inv2


def test_python_transliteration_wls_bitwise(oracle_mod):
    rng = np.random.default_rng(4)
    for trial in range(20):
        h, lvl = 0.3125, int(rng.integers(0, 3))
        cx, cy = 1.0 + 0.3125 * rng.integers(0, 10), 2.0 + 0.3125 * rng.integers(0, 10)
        m1, m2 = int(rng.integers(3, 6)), int(rng.integers(2, 5))
        if m1 + m2 < 7:
            m1 = 7 - m2
        xs = list(cx + h * rng.integers(-2, 3, m1 + m2) / 2.0)
        ys = list(cy + h * rng.integers(-2, 3, m1 + m2) / 2.0)
        vals = np.array([_rand_state(rng) for _ in range(m1 + m2)])
        xx, yy = cx + h / 4, cy
        out, _ = oracle_mod.wls(h, 1.0, lvl, cx, cy, xx, yy, m1, m2, xs, ys, vals)
        ref = refnum.wlsi(h, 1.0, lvl, cx, cy, xx, yy, m1, m2, xs, ys, vals)
        assert list(out) == ref, trial


def _interior_mask(cfg, keys):
    root = (keys >> np.uint64(34)).astype(np.int64)
    row, col = root // cfg.m, root % cfg.m
    return (row >= 3) & (row < cfg.n - 3) & (col >= 3) & (col < cfg.m - 3)


def _uniform_flow_drift(oracle_mod, steps_before):
    cfg = P.vortex()
    o = oracle_mod.Oracle(cfg)
    o.solute(steps_before)
    keys, prim, T = o.leaves()
    prim[:] = (1.3, 0.4, -0.25, 0.9)
    o.set_leaves(keys, prim)
    o.set_scalars(1.5, 1.5, 0.01, 0.0, 1)
    for _ in range(3):
        o.time_advance_rk()
    _, prim2, _ = o.leaves()
    return np.max(np.abs(prim2 - prim))


def test_uniform_flow_preserved_uniform_mesh(oracle_mod):
    assert _uniform_flow_drift(oracle_mod, 0) < 1e-13


def test_uniform_flow_on_amr_mesh_bounded(oracle_mod):
    """At hanging nodes the reference fits a quadratic in absolute (not
    cell-centred) coordinates (src/XuanGua.F90:224-229), so a constant is
    reproduced only to the conditioning of P^T W P: ~1e-8, not round-off."""
    d = _uniform_flow_drift(oracle_mod, 12)
    assert 1e-12 < d < 1e-6


def test_vortex_convergence_order(oracle_mod):
    """Uniform-grid isentropic vortex: third-order scheme, observed order >= 2.5."""
    errs = []
    for base in (32, 64):
        cfg = P.vortex(base=base, lvl_amr=0)
        cfg.params.t_end = 0.5
        cfg.params.cfl = 0.2
        o = oracle_mod.Oracle(cfg)
        o.solute(10 ** 6)
        keys, prim, _ = o.leaves()
        inter = _interior_mask(cfg, keys)
        root = (keys >> np.uint64(34)).astype(np.int64)
        x = cfg.params.xmin + (root % cfg.m + 0.5) * cfg.params.h
        y = cfg.params.ymin + (root // cfg.m + 0.5) * cfg.params.h
        t = o.scalars()["tt"]
        xc, yc = (x - t) % 10.0, (y - t) % 10.0
        rr = (xc - 5) ** 2 + (yc - 5) ** 2
        dT = -(G14 - 1) * 25 * np.exp(1 - rr) / (8 * G14 * math.pi ** 2)
        exact = (1 + dT) ** (1 / (G14 - 1))
        errs.append(np.abs(prim[inter, 0] - exact[inter]).mean())
    assert math.log2(errs[0] / errs[1]) > 2.5


def test_leaf_order_is_reference_order(oracle_mod):
    """Keys exported in ascending order equal IDNSgrid's order."""
    cfg = P.vortex()
    o = oracle_mod.Oracle(cfg)
    o.solute(12)
    keys, _, _ = o.leaves()
    assert np.all(np.diff(keys.astype(np.uint64)) > 0)
    assert o.num_interior() == int(_interior_mask(cfg, keys).sum())


def test_wls_constant_error_grows_with_resolution(oracle_mod):
    """The reference's hanging-node fit (src/XuanGua.F90:224-229: basis 1, x,
    y, xy, x^2, y^2 in absolute coordinates, Gauss-Jordan inverse) loses
    digits as the mesh spacing shrinks: on a band-refined 4-level mesh with a
    constant state, the hanging-node values miss the constant by an amount
    that grows with the background resolution.  The oracle (and the GPU,
    bit for bit) reproduce this."""
    from fdm_cell_based_amr_cartesian_b200.solver import distance_refined_keys
    errs = []
    for base in (16, 32):
        cfg = P.riemann4(base=base, lvl_amr=4)
        keys = distance_refined_keys(cfg, [("y", 0.5)], [0.2, 0.15, 0.1, 0.05])
        prim = np.tile(np.array([1.5, 0.0, 0.0, 1.5]), (len(keys), 1))
        o = oracle_mod.Oracle(cfg, initial=False)
        o.set_leaves(keys, prim)
        errs.append(float(np.abs(o.stencil()[:, :, 0] - 1.5).max()))
        o.close()
    assert 0.0 < errs[0] < errs[1] < 1e-3, errs
