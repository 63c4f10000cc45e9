"""Learned smoothness gate of the face flux: data, training, evaluation.

The plain solver emits per-face samples (8 features, target exp(-dev/tau)
with dev the largest effect of the nonlinear WCNS weights' deviation from
the linear ones on a reconstruction) on randomized four-quadrant problems;
the MLP is trained on the GPU by libfdm's tensor-core forward/backward
kernels (fdm_gate_train_step).  The trained parameters are kept in
gate_params.npy next to this file:

    python -m fdm_cell_based_amr_cartesian_b200.learned --train
"""
from __future__ import annotations

import argparse
import ctypes
import os
import time

import numpy as np

from . import params as P
from .solver import FdmError, Solver, load_library

HERE = os.path.dirname(os.path.abspath(__file__))
PARAMS_PATH = os.path.join(HERE, "gate_params.npy")
N_PARAMS = 1377
TAU = 1e-3          # target = exp(-dev / TAU): above 0.9 for dev < 1.05e-4
THRESHOLD = 0.9     # gate >= 0.9 takes the linear path
NEG_WEIGHT = 4.0    # weight of the non-smooth term of the loss (false "smooth" costs more)


def _lib():
    L = load_library()
    vp, i64, f32p = ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)
    L.fdm_gate_param_count.restype = ctypes.c_int
    L.fdm_gate_set.argtypes = [vp, f32p, ctypes.c_float, ctypes.c_int32]
    L.fdm_gate_samples.argtypes = [vp, i64, i64, ctypes.c_double, vp, vp, i64, i64, ctypes.POINTER(i64)]
    L.fdm_gate_train_step.argtypes = [vp, vp, i64, i64, i64, i64, ctypes.c_float, vp, vp, vp, vp, i64,
                                      ctypes.c_float, vp, vp]
    L.fdm_gate_eval.argtypes = [vp, i64, vp, vp, vp]
    L.fdm_gate_stats.argtypes = [vp, ctypes.POINTER(i64), ctypes.POINTER(i64)]
    return L


def stats(solver: Solver):
    """(faces on the linear path in the last stage, all faces)."""
    L = _lib()
    a, b = ctypes.c_int64(), ctypes.c_int64()
    rc = L.fdm_gate_stats(solver.h, ctypes.byref(a), ctypes.byref(b))
    if rc:
        raise FdmError(rc, "fdm_gate_stats failed")
    return a.value, b.value


def init_params(seed: int = 0) -> np.ndarray:
    """Scaled-normal initialisation of W1[32][8], b1, W2[32][32], b2, w3, b3."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[0:256] = rng.normal(0, 1 / np.sqrt(8), 256)
    p[288:1312] = rng.normal(0, 1 / np.sqrt(32), 1024)
    p[1344:1376] = rng.normal(0, 1 / np.sqrt(32), 32)
    p[1376] = 2.0          # start biased toward "smooth" (most faces are)
    return p


def enable(solver: Solver, params: np.ndarray | None = None, threshold: float = THRESHOLD):
    L = _lib()
    p = np.ascontiguousarray(load_params() if params is None else params, np.float32)
    rc = L.fdm_gate_set(solver.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), threshold, 1)
    if rc:
        raise FdmError(rc, "fdm_gate_set failed")


def disable(solver: Solver):
    L = _lib()
    rc = L.fdm_gate_set(solver.h, None, 0.5, 0)
    if rc:
        raise FdmError(rc, "fdm_gate_set failed")


def jump_rule(solver: Solver, jump_threshold: float):
    """The plain rule in place of the network (the gate must be enabled):
    linear when the largest normalised jump <= jump_threshold; a negative
    threshold restores the network."""
    rc = solver.L.fdm_gate_set_jump_rule(solver.h, float(jump_threshold))
    if rc:
        raise FdmError(rc, "fdm_gate_set_jump_rule failed")


def stage1_fraction(cfg: P.Config, keys, prim, setup) -> float:
    """Gated share of the faces at stage 1 of one step from (keys, prim)
    with the gate as `setup(solver)` leaves it."""
    g = Solver(cfg)
    g.upload(keys, prim)
    g.body_boundary(1)
    g.step_control()
    setup(g)
    g.solution_cells(1)
    a, b = stats(g)
    g.close()
    return a / max(b, 1)


def rule_vs_network(cfg: P.Config, keys, prim, steps: int, params=None, threshold: float = THRESHOLD):
    """What the network buys: the network gate against the plain jump rule
    on the same eight features, the rule's threshold tuned (bisection) so
    that it gates the same share of faces at stage 1 as the network.  Both
    run `steps` steps from (keys, prim) beside a plain run; returns their
    gated shares, ms per step and density errors against the plain run."""
    import torch

    def on_net(g):
        enable(g, params, threshold)

    frac_net = stage1_fraction(cfg, keys, prim, on_net)
    lo, hi = 0.0, 1.0
    while stage1_fraction(cfg, keys, prim, lambda g: (on_net(g), jump_rule(g, hi))) < frac_net and hi < 1e6:
        lo, hi = hi, hi * 4.0
    for _ in range(24):
        mid = 0.5 * (lo + hi)
        if stage1_fraction(cfg, keys, prim, lambda g: (on_net(g), jump_rule(g, mid))) < frac_net:
            lo = mid
        else:
            hi = mid
    thr_rule = hi

    def run(setup):
        g = Solver(cfg)
        g.upload(keys, prim)
        g.body_boundary(1)
        g.step_control()
        setup(g)
        g.advance(2)                     # warm-up (graph capture)
        g.upload(keys, prim)
        g.body_boundary(1)
        g.step_control()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.advance(steps)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1e3 / steps
        a, b = stats(g)
        out = g.leaves()
        g.close()
        return out, ms, a / max(b, 1)

    plain, ms_plain, _ = run(lambda g: None)
    net, ms_net, last_net = run(on_net)
    rule, ms_rule, last_rule = run(lambda g: (on_net(g), jump_rule(g, thr_rule)))
    l1n, lin_n = density_errors(cfg, plain, net)
    l1r, lin_r = density_errors(cfg, plain, rule)
    return {"steps": steps, "plain_ms_per_step": ms_plain,
            "network": {"stage1_gated_fraction": frac_net, "last_stage_gated_fraction": last_net,
                        "ms_per_step": ms_net, "l1_density_vs_plain": l1n, "linf_density_vs_plain": lin_n},
            "jump_rule": {"jump_threshold": thr_rule,
                          "stage1_gated_fraction": stage1_fraction(
                              cfg, keys, prim, lambda g: (on_net(g), jump_rule(g, thr_rule))),
                          "last_stage_gated_fraction": last_rule, "ms_per_step": ms_rule,
                          "l1_density_vs_plain": l1r, "linf_density_vs_plain": lin_r}}


def load_params() -> np.ndarray:
    return np.load(PARAMS_PATH).astype(np.float32)


def collect(seeds, base=64, lvl_amr=3, steps=200, every=10, stride=3, tau=TAU, cap=12_000_000):
    """(features, targets) on the GPU (torch tensors) from plain runs of
    random four-quadrant problems (rho, p ~ U[0.1,2], u, v ~ U[-1,1])."""
    import torch
    L = _lib()
    X = torch.empty((cap, 8), dtype=torch.float32, device="cuda")
    Y = torch.empty((cap,), dtype=torch.float32, device="cuda")
    n = 0
    phase = 0
    for seed in seeds:
        cfg = P.random_riemann4(seed, base=base, lvl_amr=lvl_amr, t_end=1e9)
        g = Solver(cfg)
        g.creat_mesh_and_initial()
        for k in range(steps):
            g.solute_step()
            if k % every == every - 1 and n < cap:
                w = ctypes.c_int64()
                rc = L.fdm_gate_samples(g.h, stride, phase % stride, tau, X.data_ptr(), Y.data_ptr(), n, cap,
                                        ctypes.byref(w))
                if rc:
                    raise FdmError(rc, "fdm_gate_samples failed")
                n += w.value
                phase += 1
        g.close()
        if n >= cap:
            break
    torch.cuda.synchronize()
    return X[:n], Y[:n]


def train(X, Y, steps=3000, batch=65536, lr=3e-3, seed=0, params=None, log_every=0, neg_weight=NEG_WEIGHT,
          cosine=False):
    """Adam on the weighted cross entropy of minibatches (cosine-decayed
    learning rate if asked); returns (params, loss history)."""
    import torch
    L = _lib()
    n = X.shape[0]
    p = torch.tensor(init_params(seed) if params is None else params, device="cuda")
    grad = torch.zeros_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(seed)
    hist = []
    for t in range(1, steps + 1):
        idx0 = int(rng.integers(0, n))
        step = int(rng.choice([1, 3, 7, 11, 13, 17, 19, 23]))   # strided, wrapped minibatch
        lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * (t - 1) / steps)) if cosine else lr
        rc = L.fdm_gate_train_step(X.data_ptr(), Y.data_ptr(), n, idx0, step, min(batch, n), neg_weight,
                                   p.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), t, lr_t,
                                   loss.data_ptr(), ctypes.c_void_p(stream))
        if rc:
            raise FdmError(rc, "fdm_gate_train_step failed")
        if log_every and (t % log_every == 0 or t == 1):
            hist.append((t, float(loss.item()) / min(batch, n)))
    torch.cuda.synchronize()
    return p.cpu().numpy(), hist


def gradients(X, Y, params, batch, idx0=0, step=1, neg_weight=1.0):
    """Mean-loss gradients of one minibatch from the GPU kernels (lr = 0)."""
    import torch
    L = _lib()
    p = torch.tensor(params, device="cuda")
    grad = torch.zeros_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    rc = L.fdm_gate_train_step(X.data_ptr(), Y.data_ptr(), X.shape[0], idx0, step, batch, neg_weight,
                               p.data_ptr(), grad.data_ptr(), m.data_ptr(), v.data_ptr(), 1, 0.0,
                               loss.data_ptr(), None)
    if rc:
        raise FdmError(rc, "fdm_gate_train_step failed")
    torch.cuda.synchronize()
    return grad.cpu().numpy(), float(loss.item())


def probabilities(X, params):
    import torch
    L = _lib()
    p = torch.tensor(params, device="cuda")
    out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
    rc = L.fdm_gate_eval(X.data_ptr(), X.shape[0], p.data_ptr(), out.data_ptr(), None)
    if rc:
        raise FdmError(rc, "fdm_gate_eval failed")
    torch.cuda.synchronize()
    return out


def fine_density(cfg: P.Config, keys, prim, level=None):
    """Leaf densities painted onto the uniform grid of the finest level
    (each leaf covers 4^(L - lvl) fine cells) over all m x n roots."""
    p = cfg.params
    keys = np.asarray(keys, dtype=np.uint64)
    lvl = (keys & np.uint64(15)).astype(np.int64)
    L = int(lvl.max(initial=0)) if level is None else level
    root = (keys >> np.uint64(34)).astype(np.int64)
    path = ((keys >> np.uint64(4)) & np.uint64((1 << 30) - 1)).astype(np.int64)
    ix = (root % p.m) << L
    iy = (root // p.m) << L
    for k in range(1, L + 1):
        act = lvl >= k
        q = (path >> (2 * (15 - k))) & 3
        ix = ix + np.where(act, (q & 1) << (L - k), 0)
        iy = iy + np.where(act, (q >> 1) << (L - k), 0)
    out = np.zeros(((p.n << L), (p.m << L)), np.float64)
    side = 1 << (L - lvl)
    for s in np.unique(side):
        sel = side == s
        for dy in range(s):
            for dx in range(s):
                out[iy[sel] + dy, ix[sel] + dx] = prim[sel, 0]
    return out


def density_errors(cfg: P.Config, plain, gated):
    """(L1, Linf) of the gated density against the plain one, area-weighted
    on the finest uniform grid, relative to the plain density's L1 / Linf."""
    kp, pp = plain
    kg, pg = gated
    L = int(max((np.asarray(kp, np.uint64) & np.uint64(15)).max(), (np.asarray(kg, np.uint64) & np.uint64(15)).max()))
    a = fine_density(cfg, kp, pp, L)
    b = fine_density(cfg, kg, pg, L)
    d = np.abs(b - a)
    return float(d.sum() / np.abs(a).sum()), float(d.max() / np.abs(a).max())


def compare(cfg: P.Config, steps: int, params=None, threshold: float = THRESHOLD):
    """Run the plain and the gated solver side by side for `steps` solute
    iterations; returns the density errors, the gated face fraction of the
    last stage and the leaf counts."""
    plain, gated = Solver(cfg), Solver(cfg)
    plain.creat_mesh_and_initial()
    gated.creat_mesh_and_initial()
    enable(gated, params, threshold)
    plain.solute(steps)
    gated.solute(steps)
    g, n = stats(gated)
    pl, gl = plain.leaves(), gated.leaves()
    l1, linf = density_errors(cfg, pl, gl)
    plain.close()
    gated.close()
    return {"l1": l1, "linf": linf, "gated_fraction": g / max(n, 1), "leaves_plain": len(pl[0]),
            "leaves_gated": len(gl[0])}


def compare_paired(cfg: P.Config, steps: int | None = None, params=None, threshold: float = THRESHOLD,
                   chunk: int = 100, follower: str = "gate"):
    """The plain solver and a follower in lockstep (fdm_solute_paired): the
    follower takes the plain run's time steps and regrid decisions, so both
    keep one leaf set and the density difference at the end comes from the
    follower alone.  follower "gate": the learned gate on; "ulp": the plain
    scheme started from an initial density one ulp higher, which measures how
    far rounding-level differences grow in this problem.  Runs to t_end (or
    `steps` iterations); returns the density errors, the steps and regrids
    taken, the leaf count at the end and the follower's gated face share in
    its last stage."""
    plain, gated = Solver(cfg), Solver(cfg)
    plain.creat_mesh_and_initial()
    gated.creat_mesh_and_initial()
    if follower == "gate":
        enable(gated, params, threshold)
    elif follower == "ulp":
        _, p0 = gated.leaves()
        p0 = p0.copy()
        p0[:, 0] = np.nextafter(p0[:, 0], np.inf)
        gated.set_values(p0)
    else:
        raise ValueError(follower)
    n = 0
    while (steps is None or n < steps) and plain.scalars()["tt"] < cfg.params.t_end:
        k = plain.solute_paired(gated, chunk if steps is None else min(chunk, steps - n))
        n += k
        if k == 0:
            break
    pl, gl = plain.leaves(), gated.leaves()
    assert np.array_equal(pl[0], gl[0]), "paired runs ended on different leaf sets"
    l1, linf = density_errors(cfg, pl, gl)
    out = {"l1": l1, "linf": linf, "steps": n, "tt": plain.scalars()["tt"],
           "regrids": plain.counters()["n_regrids"], "leaves": len(pl[0])}
    if follower == "gate":
        a, b = stats(gated)
        out["gated_fraction_last_stage"] = a / max(b, 1)
    plain.close()
    gated.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--seeds", type=int, default=24)
    ap.add_argument("--steps", type=int, default=3000)
    args = ap.parse_args()
    if args.train:
        import torch
        t0 = time.time()
        X, Y = collect(range(args.seeds))
        print(f"samples {X.shape[0]} collected in {time.time() - t0:.1f}s; smooth fraction "
              f"{float((Y > THRESHOLD).float().mean()):.3f}")
        params, hist = train(X, Y, steps=args.steps, log_every=500, cosine=True)
        for t, l in hist:
            print(f"step {t} loss {l:.5f}")
        Xe, Ye = collect(range(1000, 1004))
        prob = probabilities(Xe, params)
        gate = prob >= THRESHOLD
        smooth = Ye >= THRESHOLD
        dev = -TAU * torch.log(Ye.clamp(min=1e-30))
        print(f"held-out: smooth fraction {float(smooth.float().mean()):.3f}, gated fraction "
              f"{float(gate.float().mean()):.3f}, precision {float((gate & smooth).sum() / gate.sum().clamp(min=1)):.4f}, "
              f"largest dev among gated {float(dev[gate].max()) if bool(gate.any()) else 0.0:.3e}")
        np.save(PARAMS_PATH, params)
        print("saved", PARAMS_PATH, f"{time.time() - t0:.1f}s")


if __name__ == "__main__":
    main()
