#!/usr/bin/env python
"""Benchmark: leaf-cell RK3 updates/s on the four-quadrant Riemann workload.

One step = one solute iteration (step control + 3 SSP-RK3 stages + ghost
fill) over every interior leaf.  Workload: four-quadrant Riemann problem on
[0,1]^2, base grid 128^2 (134^2 with ghosts), 4 refinement levels, the cells
within 0.2/0.15/0.1/0.05 of the quadrant split lines refined to levels
1/2/3/4 (about 1.0M leaves); synthetic state (the config's initial
condition).  The state (~1.1 GB with tables) is far larger than L2, and L2
is also flushed before every timed step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): one independent instance per rank (weak scaling, no
collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from fdm_cell_based_amr_cartesian_b200 import params as P  # noqa: E402

METRIC = "leaf-cell RK3 updates/s"
UNIT = "updates/s"
BAND = [0.2, 0.15, 0.1, 0.05]
FLOPS_PER_FACE = 1233          # IEEE FP64 ops of one face flux (add/mul/div/sqrt/min)
FLOPS_PER_CELL = 150           # residual, conversions and RK blend per leaf and stage
BYTES_PER_UPDATE = 256         # 8 x 32-byte (rho,u,v,p) transfers per leaf per RK3 step


def workload():
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    cfg = P.riemann4(base=128, lvl_amr=4)
    keys = S.distance_refined_keys(cfg, [("x", 0.5), ("y", 0.5)], BAND)
    prim = S.initial_state(cfg, keys)
    return cfg, keys, prim


def workload_desc(n_leaves, n_interior):
    return {"workload": "riemann4 four-quadrant, base 128x128, 4 levels, distance-refined bands "
                        "0.2/0.15/0.1/0.05 around the split lines",
            "leaves": int(n_leaves), "interior_leaves": int(n_interior),
            "l2": "flushed before every timed step (256 MiB write); state > L2"}


# ------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def profile_figure(name):
    """A figure of the committed ncu summary of the face kernel (a line
    'name: value'): DRAM bytes per x+y launch pair, FP64 pipe activity."""
    path = os.path.join(ROOT, "profiles", "face_flux_riemann4.md")
    try:
        for line in open(path):
            if line.startswith(name + ":"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


def profile_traffic():
    return profile_figure("traffic_bytes_per_launch")


def profile_text(name):
    """A text field of the face kernel's ncu summary (a line 'name: value')."""
    path = os.path.join(ROOT, "profiles", "face_flux_riemann4.md")
    try:
        for line in open(path):
            if line.startswith(name + ":"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


# ------------------------------------------------------------ CPU legs
def cpu_sample(cfg, keys, prim, lam, tstep, steps):
    """Time the oracle (the CPU restatement of the reference OpenMP path) on
    the same mesh: `steps` RK3 steps, all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(cfg, initial=False)
    o.set_leaves(keys, prim)
    o.set_scalars(lam[0], lam[1], tstep, 0.0, 1)
    n_int = o.num_interior()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.time_advance_rk()
    dt = time.perf_counter() - t0
    o.close()
    return n_int, dt


FORTRAN_COMPILERS = ("gfortran", "gfortran-14", "gfortran-13", "gfortran-12", "flang", "flang-new", "ifx", "ifort",
                     "nvfortran", "pgfortran", "lfortran", "f95", "f77")


def fortran_probe() -> str:
    """Which Fortran compilers this box has (the reference is Fortran only)."""
    import shutil
    found = [c for c in FORTRAN_COMPILERS if shutil.which(c)]
    if found:
        return "Fortran compilers on the box: " + ", ".join(found) + "; the reference is not built by the bench"
    return "probed on the box: no Fortran compiler (" + ", ".join(FORTRAN_COMPILERS) + " absent)"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg, keys, prim = workload()
    threads = os.cpu_count() or 1
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    # lambda of the initial state (the GPU arm's first step control gives the same)
    r, u, v, p = prim[:, 0], prim[:, 1], prim[:, 2], prim[:, 3]
    c = np.sqrt(cfg.params.gama * p / r)
    lam = (float(np.max(np.abs(u) + c)), float(np.max(np.abs(v) + c)))
    o = oracle.Oracle(cfg, initial=False, threads=threads)
    o.set_leaves(keys, prim)
    o.set_scalars(lam[0], lam[1], 1e-5, 0.0, 1)
    n_int = o.num_interior()
    per = []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        o.time_advance_rk()
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            per.append(dt)
        if sum(per) > 150:
            break
    o.close()
    total = sum(per)
    value = n_int * len(per) / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(per), "warmup": args.warmup, "ms_per_step": 1e3 * total / len(per),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_desc(len(keys), n_int),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{len(per)} RK3 steps of the full mesh, OpenMP restatement of "
                                       f"Time_advance_RK ({fortran_probe()})"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------- GPU arm
def timed_window(g, steps, warmup, flush):
    """Device time (ms) of `steps` solute iterations (step graph replays)
    on the handle's stream, L2 flushed before each, after `warmup` untimed."""
    import torch
    for _ in range(warmup):
        g.advance(1)
    torch.cuda.synchronize()
    stream_ptr, _, _ = g.device_state()
    ext = torch.cuda.ExternalStream(stream_ptr)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(ext):
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(ext)
            g.advance(1)
            ev[k][1].record(ext)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def fast_window(args, keys, prim, NI, flush, world):
    """flux_variant 1 (FMA contraction, shared reciprocals) on the same mesh
    and window: updates/s, and the difference after one step from the same
    state against the exact path (relative to each field's magnitude)."""
    import torch
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks
    cfg_f = P.riemann4(base=128, lvl_amr=4)
    cfg_f.params.flux_variant = 1
    gf = S.Solver(cfg_f)
    gf.upload(keys, prim)
    gf.body_boundary(1)
    gf.step_control()
    tuned, _ = gf.autotune(reps=5)
    ms = max_over_ranks(timed_window(gf, args.steps, args.warmup, flush), device="cuda")
    kt = gf.time_kernels(reps=9)
    gf.close()
    # one step from the initial state on fresh handles (scalars included),
    # fast against exact
    pair = []
    for fv in (1, 0):
        c = P.riemann4(base=128, lvl_amr=4)
        c.params.flux_variant = fv
        g = S.Solver(c)
        g.upload(keys, prim)
        g.body_boundary(1)
        g.advance(1)
        pair.append(g.leaves()[1])
        g.close()
    a, b = pair
    dev = float(np.max(np.max(np.abs(a - b), axis=0) / np.max(np.abs(b), axis=0)))
    return {"value": NI * world * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "face_variant": tuned, "kernel_ms": kt, "one_step_rel_diff_vs_exact": dev,
            "note": "flux_variant 1: FMA contraction, shared reciprocals, one division per Z-weight pair"}


def learned_window(args, cfg, keys, prim, NI, flush, world):
    """The learned-gated solver on the same mesh and window as the plain
    one: updates/s, the gated face share, and the density error against a
    plain run over the same steps."""
    import torch
    from fdm_cell_based_amr_cartesian_b200 import learned as LG
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks
    if not os.path.exists(LG.PARAMS_PATH):
        return {"unavailable": "no trained gate parameters"}
    gl = S.Solver(cfg)
    gl.upload(keys, prim)
    gl.body_boundary(1)
    gl.step_control()
    LG.enable(gl)
    ms = max_over_ranks(timed_window(gl, args.steps, args.warmup, flush), device="cuda")
    gated, total = LG.stats(gl)
    ref = S.Solver(cfg)
    ref.upload(keys, prim)
    ref.body_boundary(1)
    ref.step_control()
    ref.advance(args.warmup + args.steps)
    torch.cuda.synchronize()
    l1, linf = LG.density_errors(cfg, ref.leaves(), gl.leaves())
    kt = gl.time_kernels(reps=5)
    gl.close()
    ref.close()
    # what the network buys: the plain jump rule on the same features at the
    # same gated share of faces (host-timed windows, same mesh)
    try:
        rvn = LG.rule_vs_network(cfg, keys, prim, args.steps)
    except Exception as ex:              # an auxiliary leg never costs the line
        rvn = {"error": f"{type(ex).__name__}: {ex}"}
    return {"value": NI * world * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "gated_face_fraction": gated / max(total, 1), "threshold": LG.THRESHOLD,
            "l1_density_vs_plain": l1, "linf_density_vs_plain": linf,
            "error_window_steps": args.warmup + args.steps, "kernel_ms": kt, "rule_vs_network": rvn}


def ensemble_window(args, world):
    """The ensemble configuration: 64 random four-quadrant problems (maximum
    level drawn from 2..5, band-refined meshes, 66M leaves in all) on one GPU
    with learned gating, advanced by the batched path (one persistent launch
    per RK3 stage over all members).  Timed beside the same members with the
    gate off, and beside the single-mesh path (one step graph per member,
    each on its own stream).  Inputs far exceed L2, so no flush is needed."""
    import torch
    from fdm_cell_based_amr_cartesian_b200 import ensemble as E
    from fdm_cell_based_amr_cartesian_b200 import learned as LG
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks
    if not os.path.exists(LG.PARAMS_PATH):
        return {"unavailable": "no trained gate parameters"}
    from fdm_cell_based_amr_cartesian_b200.ensemble import sum_over_ranks
    t_setup = time.perf_counter()
    cfgs_all = E.ensemble_configs()
    meshes_all = E.ensemble_meshes(cfgs_all)
    # the natural shard: whole members per rank, balanced by leaf count, no
    # collective on the data path (every rank computes the same owner map)
    rank = int(os.environ.get("RANK", "0"))
    owner = E.partition([len(k) for k, _ in meshes_all], world)
    mine = [i for i in range(len(cfgs_all)) if owner[i] == rank]
    cfgs = [cfgs_all[i] for i in mine]
    meshes = [meshes_all[i] for i in mine]
    sols = []
    for cfg, (k, p) in zip(cfgs, meshes):
        g = S.Solver(cfg)
        g.upload(k, p)
        g.body_boundary(1)
        LG.enable(g)
        sols.append(g)
    NI_rank = sum(g.counters()["n_interior"] for g in sols)
    NI = int(sum_over_ranks(NI_rank, device="cuda"))
    batch = S.Batch(sols)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    ext = torch.cuda.ExternalStream(batch.stream())

    def timed_batch():
        batch.advance(args.warmup)
        batch.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            a.record(ext)
            batch.advance(args.steps)
            b.record(ext)
        batch.sync()
        return max_over_ranks(a.elapsed_time(b), device="cuda")

    # the persistent kernel at 1 or 2 resident blocks per SM, or (0) the
    # members' own step graphs on their own streams: the fastest
    tune = {}
    for bps in (0, 1, 2, 3):
        batch.set_blocks_per_sm(bps)
        batch.advance(2)
        batch.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(ext):
            a.record(ext)
            batch.advance(3)
            b.record(ext)
        batch.sync()
        tune[bps] = a.elapsed_time(b) / 3
    best_bps = min(tune, key=tune.get)
    batch.set_blocks_per_sm(best_bps)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        ms_gated = timed_batch()
    gated, total = 0, 0
    for g in sols:
        a, b = LG.stats(g)
        gated += a
        total += b
    info = batch.info()
    for g in sols:
        LG.disable(g)
    ms_plain = timed_batch()
    # the single-mesh path on the same members: one step graph per member,
    # members on their own streams (host-timed: the launches are the cost)
    for g in sols:
        LG.enable(g)
        g.advance(args.warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for g in sols:
        g.advance(args.steps)
    torch.cuda.synchronize()
    ms_single = max_over_ranks((time.perf_counter() - t0) * 1e3, device="cuda")
    finite = all(bool(np.isfinite(g.leaves()[1]).all()) for g in sols[:4])
    batch.close()
    for g in sols:
        g.close()
    # accuracy of the gate: one member per level, gated against plain (on
    # rank 0; no collective inside)
    acc = {}
    for L in ((2, 3, 4, 5) if rank == 0 else ()):
        i = next(j for j, c in enumerate(cfgs_all) if int(c.params.lvl_amr) == L)
        pair = []
        for gate in (False, True):
            g = S.Solver(cfgs_all[i])
            g.upload(*meshes_all[i])
            g.body_boundary(1)
            if gate:
                LG.enable(g)
            g.advance(args.warmup + args.steps)
            pair.append(g.leaves())
            g.close()
        l1, linf = LG.density_errors(cfgs_all[i], pair[0], pair[1])
        acc[f"level{L}_seed{E.ENSEMBLE_SEEDS[i]}"] = {"l1": l1, "linf": linf}
    # NI counts the members of every rank: whole-job updates per second
    per = lambda ms: NI * args.steps / (ms / 1e3)
    return {"workload": f"64 random four-quadrant problems (seeds 1000-1063, rho,p~U[0.1,2], u,v~U[-1,1]), "
                        f"base {E.ENSEMBLE_BASE}^2, max level U{{2..5}}, band-refined meshes, learned gate on",
            "blocks_per_sm_ms_per_step": tune,
            "strategy": {0: "member step graphs on their own streams",
                         3: "phase kernels: one launch per phase over every member"}.get(
                             best_bps, f"persistent kernel, {best_bps} block(s) per SM"),
            "members": len(cfgs_all), "members_on_rank0": len(cfgs) if rank == 0 else None,
            "sharding": f"whole members per rank, balanced by leaf count over {world} rank(s)",
            "interior_leaves": int(NI), "value": per(ms_gated), "unit": UNIT,
            "ms_per_step": ms_gated / args.steps, "gated_face_fraction": gated / max(total, 1),
            "plain_batched": {"value": per(ms_plain), "ms_per_step": ms_plain / args.steps},
            "single_mesh_graphs": {"value": per(ms_single), "ms_per_step": ms_single / args.steps,
                                   "note": "same members, one step graph each, own streams, host-timed"},
            "density_error_vs_plain": acc, "launch": info, "setup_s": t_setup, "clocks": clk.summary(),
            "state_finite": finite,
            "gpu_launches_per_step": 3 if best_bps else None}


def strips_window(keys, prim, nstrips=4, steps=3, asynchronous=False):
    """One mesh as strips of background rows with the halo exchange after
    every stage, all strips on this GPU: time per step and bit-identity with
    the whole mesh after the same steps."""
    import torch
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    from fdm_cell_based_amr_cartesian_b200 import strips as SP
    cfg = P.riemann4(base=128, lvl_amr=4)
    cfg.params.iflag_amr = 0
    t_end = cfg.params.t_end
    plan = SP.StripPlan(cfg, keys, nstrips)
    engines = [SP.GpuStrip(plan, s, prim, asynchronous) for s in range(nstrips)]
    xchg = SP.LocalExchange(engines)
    tt, it, _ = SP.run(engines, xchg, 1, t_end)          # warm-up step
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tt, it, k = SP.run(engines, xchg, steps, t_end, tt, it)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    ks, ps = plan.gather([e.leaves() for e in engines])
    for e in engines:
        e.close()
    whole = S.Solver(cfg)
    whole.upload(keys, prim)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(1 + steps):
        whole.solute_step()
    torch.cuda.synchronize()
    dt_whole = (time.perf_counter() - t1) / (1 + steps)
    kw, pw = whole.leaves()
    ni = whole.counters()["n_interior"]
    whole.close()
    return {"strips": nstrips, "asynchronous": asynchronous, "rows": [list(st.own) for st in plan.strips],
            "steps": k,
            "ms_per_step": dt / k * 1e3, "value": ni * k / dt, "unit": UNIT,
            "whole_mesh_ms_per_step": dt_whole * 1e3,
            "bit_identical_to_whole_mesh": bool(np.array_equal(ks, kw) and np.array_equal(ps, pw)),
            "note": "all strips on one GPU (synchronous: every split-API call waits; asynchronous: each strip "
                    "on its own stream, ordered by events, one host wait per strip at step control and step "
                    "end): the cost of the protocol, not a multi-GPU scaling figure; host-timed"}


def strips_window_dist(keys, prim, rank, world, steps=5):
    """One mesh split over the ranks: strip r of the benchmark mesh on rank r,
    the halo exchange after every stage over NCCL (paired send/recv between
    neighbouring ranks) and one all-reduce(max) of the wave speeds per step.
    Device-timed (CUDA events on each strip's stream, max over ranks); rank 0
    gathers the strips and checks them bit for bit against the whole mesh."""
    import torch
    import torch.distributed as dist
    from fdm_cell_based_amr_cartesian_b200 import solver as S
    from fdm_cell_based_amr_cartesian_b200 import strips as SP
    from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks
    cfg = P.riemann4(base=128, lvl_amr=4)
    cfg.params.iflag_amr = 0
    t_end = cfg.params.t_end
    dev = torch.device("cuda", torch.cuda.current_device())
    plan = SP.StripPlan(cfg, keys, world)
    eng = SP.GpuStrip(plan, rank, prim, asynchronous=True)
    xchg = SP.DistExchange(eng, rank, world, dev)
    tt, it, _ = SP.run([eng], xchg, 1, t_end)          # warm-up step
    torch.cuda.synchronize()
    dist.barrier()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(eng.stream)
    tt, it, k = SP.run([eng], xchg, steps, t_end, tt, it)
    b.record(eng.stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(a.elapsed_time(b), device=dev)
    got = [None] * world if rank == 0 else None
    dist.gather_object(eng.leaves(), got, dst=0)
    eng.close()
    out = {"strips": world, "ranks": world, "rows": [list(st.own) for st in plan.strips], "steps": k,
           "ms_per_step": ms / k, "transport": "NCCL send/recv of the halo rows, all-reduce(max) per step"}
    if rank == 0:
        ks, ps = plan.gather(got)
        whole = S.Solver(cfg)
        whole.upload(keys, prim)
        for _ in range(1 + steps):
            whole.solute_step()
        kw, pw = whole.leaves()
        ni = whole.counters()["n_interior"]
        whole.close()
        out.update({"value": ni * k / (ms / 1e3), "unit": UNIT,
                    "bit_identical_to_whole_mesh": bool(np.array_equal(ks, kw) and np.array_equal(ps, pw))})
    return out


GOLDEN_RUNS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "oracle_runs.json")


def matches_golden(name, keys, prim, steps, regrids):
    """True when the run ends on the oracle's recorded final leaf set and
    states bit for bit (SHA-256 of the uint64 keys and the float64 states in
    key order), False when it does not, None when the run is not recorded."""
    import hashlib
    if not os.path.exists(GOLDEN_RUNS):
        return None
    want = json.load(open(GOLDEN_RUNS)).get(name)
    if want is None:
        return None
    hk = hashlib.sha256(np.ascontiguousarray(keys, dtype=np.uint64).tobytes()).hexdigest()
    hp = hashlib.sha256(np.ascontiguousarray(prim, dtype=np.float64).tobytes()).hexdigest()
    return bool(hk == want["sha256_keys"] and hp == want["sha256_prim"]
                and steps == want["steps"] and regrids == want["regrids"])


FULL_RUNS = {
    # name: (configuration, description, golden record)
    "riemann4": (lambda: P.riemann4(base=128, lvl_amr=4, t_end=0.3),
                 "riemann4 128^2, 4 levels, t = 0 -> 0.3, regrid every 10 steps", "riemann4_128_l4_to_t0.3"),
    "double_mach": (lambda: P.double_mach(base_y=64, lvl_amr=4, t_end=0.2),
                    "double Mach reflection (Mach-10 shock, reflecting wall) 256x64, 4 levels, "
                    "t = 0 -> 0.2, regrid every 5 steps", "double_mach_256x64_l4_to_t0.2"),
}


def full_run(S, gate, ulp=False, case="riemann4"):
    import torch
    make, desc, golden = FULL_RUNS[case]
    cfg = make()
    t_end = cfg.params.t_end
    chunk = cfg.params.pstep_adapt
    gf = S.Solver(cfg)
    gf.creat_mesh_and_initial()
    if ulp:
        _, p0 = gf.leaves()
        p0 = p0.copy()
        p0[:, 0] = np.nextafter(p0[:, 0], np.inf)
        gf.set_values(p0)
    if gate:
        from fdm_cell_based_amr_cartesian_b200 import learned as LG
        LG.enable(gf)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = 0
    upd = 0
    while True:
        before = gf.scalars()["tt"]
        if before >= t_end:
            break
        ni = gf.counters()["n_interior"]
        n = gf.solute(chunk)
        steps += n
        upd += n * ni
        if n == 0:
            break
    t_full = time.perf_counter() - t0
    cf = gf.counters()
    leaves = gf.leaves()
    out = {"workload": desc,
           "seconds": t_full, "steps": steps, "regrids": cf["n_regrids"],
           "mean_updates_per_s": upd / t_full, "leaves_at_end": cf["n_leaves"],
           "regrid_device_ms_total": gf.amr_phase_ms(total=True),
           "gridmodify_counters": {k: v for k, v in cf.items() if "gm" in k}}
    if not gate and not ulp:
        out["bit_identical_to_oracle_run"] = matches_golden(golden, leaves[0], leaves[1], steps, cf["n_regrids"])
    gf.close()
    return out, leaves


def full_run_batched(S, case="double_mach"):
    """The same full run through the batched path: the autotuner picks the
    face launch shape, then a batch of one member advances it with the
    persistent kernel (2 blocks per SM, one launch per RK3 stage, CUDA-graph
    steps) and regrids when due."""
    import torch
    make, desc, golden = FULL_RUNS[case]
    cfg = make()
    gf = S.Solver(cfg)
    gf.creat_mesh_and_initial()
    tuned, _ = gf.autotune(reps=3)
    b = S.Batch([gf])
    b.set_blocks_per_sm(2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    steps = 0
    while gf.scalars()["tt"] < cfg.params.t_end:
        k = b.solute(10 * cfg.params.pstep_adapt)
        steps += k
        if k == 0:
            break
    b.sync()
    t_full = time.perf_counter() - t0
    keys, prim = gf.leaves()
    cf = gf.counters()
    out = {"workload": desc + "; batched persistent kernel, autotuned face launch shape",
           "seconds": t_full, "steps": steps, "regrids": cf["n_regrids"], "face_variant": tuned,
           "batch": b.info(), "leaves_at_end": cf["n_leaves"],
           "bit_identical_to_oracle_run": matches_golden(golden, keys, prim, steps, cf["n_regrids"])}
    b.close()
    gf.close()
    return out


def summary(line):
    """The key figures of the legs in a few short fields (the end of the line)."""
    def get(d, *ks):
        for k in ks:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return d

    def r3(x):
        return None if x is None else float(f"{x:.4g}")
    plain_ms = line["ms_per_step"]
    out = {"plain_ms_per_step": r3(plain_ms), "face_pair_ms": r3(get(line, "roofline", "ms_per_launch")),
           "fp64_frac": r3(get(line, "roofline_fp64", "frac")), "hbm_frac_faces": r3(get(line, "roofline", "frac"))}
    g = line.get("learned") or {}
    if "ms_per_step" in g:
        out["gated_ms_per_step"] = r3(g["ms_per_step"])
        out["gated_speedup"] = r3(plain_ms / g["ms_per_step"])
        out["gated_l1_window"] = r3(g.get("l1_density_vs_plain"))
        rv = g.get("rule_vs_network") or {}
        if "jump_rule" in rv:
            out["net_vs_rule_l1"] = [r3(rv["network"]["l1_density_vs_plain"]),
                                     r3(rv["jump_rule"]["l1_density_vs_plain"])]
            out["net_vs_rule_gated"] = [r3(rv["network"]["stage1_gated_fraction"]),
                                        r3(rv["jump_rule"]["stage1_gated_fraction"])]
    e = line.get("ensemble") or {}
    if "ms_per_step" in e:
        out["ensemble_gated_ms"] = r3(e["ms_per_step"])
        out["ensemble_plain_ms"] = r3(get(e, "plain_batched", "ms_per_step"))
        out["ensemble_gated_per_s"] = r3(e.get("value"))
        out["ensemble_strategy"] = e.get("strategy")
    f = line.get("full_run") or {}
    if "seconds" in f:
        out["cfg2_full_s"] = r3(f["seconds"])
        out["cfg2_gated_full_s"] = r3(get(f, "gated", "seconds"))
        out["cfg2_gated_l1_shared_regrids"] = r3(get(f, "gated_shared_regrids", "l1_density_vs_plain"))
        out["cfg2_one_ulp_l1_shared_regrids"] = r3(get(f, "gated_shared_regrids", "one_ulp_initial_density_l1"))
        out["cfg2_golden"] = f.get("bit_identical_to_oracle_run")
        out["cfg3_full_s"] = r3(get(f, "double_mach", "seconds"))
        out["cfg3_golden"] = get(f, "double_mach", "bit_identical_to_oracle_run")
        out["cfg3_batched_full_s"] = r3(get(f, "double_mach", "batched", "seconds"))
    st = line.get("strips") or {}
    if "ms_per_step" in st:
        out["strips_ms_per_step"] = r3(st["ms_per_step"])
        out["strips_bit_identical"] = st.get("bit_identical_to_whole_mesh")
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist
    from fdm_cell_based_amr_cartesian_b200 import solver as S

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    cfg, keys, prim = workload()
    g = S.Solver(cfg)
    g.upload(keys, prim)
    g.body_boundary(1)
    g.step_control()
    cnt = g.counters()
    NI = cnt["n_interior"]
    stream_ptr, _, _ = g.device_state()
    ext = torch.cuda.ExternalStream(stream_ptr)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # warm-up (also captures the step graph), then the autotuner on the
    # advanced state (the face kernels' speed depends on the data), then one
    # more untimed step that captures the step graph with the chosen shape
    for _ in range(args.warmup):
        g.advance(1)
    tuned, tune_ms = g.autotune(reps=5)
    g.advance(1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        with torch.cuda.stream(ext):
            for k in range(args.steps):
                flush.zero_()
                ev[k][0].record(ext)
                g.advance(1)
                ev[k][1].record(ext)
        torch.cuda.synchronize()
    from fdm_cell_based_amr_cartesian_b200.ensemble import max_over_ranks
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), device="cuda")
    # the timed steps must have advanced a valid flow
    _, after = g.leaves()
    finite = bool(np.isfinite(after).all() and after[:, 0].min() > 0 and after[:, 3].min() > 0)
    if not finite:
        raise RuntimeError("benchmark state is not finite/positive after the timed steps")
    if world > 1:
        dist.barrier()
    value = NI * world * args.steps / (ms / 1e3)
    clocks = clk.summary()

    # per-kernel times (CUDA events on the handle's stream) -> roofline
    kt = g.time_kernels(reps=10)
    nfaces = cnt["n_faces_x"] + cnt["n_faces_y"]
    face_bytes = (cnt["n_leaves"] + cnt["n_wls_requests"] + cnt["n_restrict_requests"]) * 32 + nfaces * 32
    face_gbs = face_bytes / (kt["faces"] * 1e-3) / 1e9
    peaks = measured_peaks()
    hbm_peak = peaks["hbm_gbs"] if peaks else 6650.0
    fp64_peak = S.fp64_peak_tflops()
    face_tflops = nfaces * FLOPS_PER_FACE / (kt["faces"] * 1e-3) / 1e12
    step_bytes = NI * BYTES_PER_UPDATE
    step_gbs = step_bytes / (ms / args.steps * 1e-3) / 1e9
    traffic = profile_traffic()

    # end-to-end through the public API with host buffers: every step uploads
    # its input state from pinned host memory, advances one step and reads the
    # new state back into pinned host memory.  The asynchronous transfer calls
    # overlap the next step's upload and the last step's read-back with the
    # step in between; the clock stops after the last read-back has landed.
    host_in = torch.empty((len(keys), 4), dtype=torch.float64, pin_memory=True)
    host_out = [torch.empty((len(keys), 4), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    hin, hout = host_in.numpy(), [t.numpy() for t in host_out]
    g.download_values(hin)
    g.set_values_async(hin)    # first use of the staging buffers, untimed
    g.advance(1)
    g.download_values_async(hout[0])
    g.io_sync()
    n_e2e = max(3, args.steps)   # as many steps as the device-timed region: the first upload and last read-back are shared by them
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(n_e2e):
        g.set_values_async(hin)
        g.advance(1)
        g.download_values_async(hout[k % 2])
    g.io_sync()
    e2e_s = max_over_ranks(time.perf_counter() - t0, device="cuda")
    e2e = {"value": NI * world * n_e2e / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(hin.nbytes), "d2h_bytes_per_step": int(hout[0].nbytes),
           "transfers": "pinned host buffers; uploads and read-backs on a copy stream, overlapped with the steps"}

    # step control, lambda reset, step end, residual reduction (stage 3) and,
    # per stage: 2 face kernels, the update, hanging nodes (+ interpA
    # fallbacks), ghosts
    per_stage = 2 + 1 + (1 if cnt["n_wls_requests"] + cnt["n_restrict_requests"] else 0) \
        + (1 if cnt["n_restrict_requests"] else 0) + (1 if cnt["n_ghost"] else 0)
    launches_per_step = 4 + 3 * per_stage

    # the fast face flux (flux_variant 1) on the same mesh and window
    fastf = fast_window(args, keys, prim, NI, flush, world)

    # learned-gated path on the same workload and window
    gated = None
    if not args.no_learned:
        gated = learned_window(args, cfg, keys, prim, NI, flush, world)

    # one mesh as 4 strips with the halo exchange (all on this GPU); this leg
    # and the full runs below are single-GPU figures, taken at N = 1 only
    # (every rank would repeat the same work)
    strips = None
    if not args.no_strips and world == 1:
        try:
            strips = strips_window(keys, prim, asynchronous=True)
            strips["synchronous"] = strips_window(keys, prim, asynchronous=False)
        except Exception as ex:          # an auxiliary leg never costs the line
            strips = {"error": f"{type(ex).__name__}: {ex}"}
    elif not args.no_strips:
        # N > 1: one strip of the same mesh per rank (every rank runs it: its
        # collectives are taken by all ranks in the same order)
        strips = strips_window_dist(keys, prim, rank, world)

    # the batched ensemble (configuration 5)
    ens = None
    if not args.no_ensemble:
        ens = ensemble_window(args, world)

    # the full configuration as the reference runs it: t = 0 -> 0.3 with the
    # device regrid every 10 steps (time to solution, all regrids included),
    # plain and learned-gated, and the gated run's density error at t = 0.3
    full = None
    if not args.no_full_run and world == 1:
        from fdm_cell_based_amr_cartesian_b200 import learned as LG
        full, leaves_plain = full_run(S, gate=False)
        cfg_full = P.riemann4(base=128, lvl_amr=4)
        if gated is not None:
            full_g, leaves_gated = full_run(S, gate=True)
            l1, linf = LG.density_errors(cfg_full, leaves_plain, leaves_gated)
            full["gated"] = dict(full_g, l1_density_vs_plain=l1, linf_density_vs_plain=linf)
            # the gate's own error over the whole run: the gated run takes the
            # plain run's time steps and regrid decisions (one leaf set)
            t0 = time.perf_counter()
            pr = LG.compare_paired(P.riemann4(base=128, lvl_amr=4, t_end=0.3))
            pu = LG.compare_paired(P.riemann4(base=128, lvl_amr=4, t_end=0.3), follower="ulp")
            full["gated_shared_regrids"] = {
                "l1_density_vs_plain": pr["l1"], "linf_density_vs_plain": pr["linf"], "steps": pr["steps"],
                "regrids": pr["regrids"], "leaves_at_end": pr["leaves"],
                "gated_fraction_last_stage": pr.get("gated_fraction_last_stage"),
                "one_ulp_initial_density_l1": pu["l1"], "one_ulp_initial_density_linf": pu["linf"],
                "seconds_four_runs": time.perf_counter() - t0,
                "note": "follower in lockstep with the plain run (fdm_solute_paired): same time steps, same regrid "
                        "decisions; the one-ulp follower is the plain scheme from a density one ulp higher"}
        # configuration 3: the Mach-10 reflection to t = 0.2, a regrid every 5 steps
        try:
            full["double_mach"] = full_run(S, gate=False, case="double_mach")[0]
        except Exception as ex:
            full["double_mach"] = {"error": f"{type(ex).__name__}: {ex}"}
        try:
            full["double_mach"]["batched"] = full_run_batched(S, case="double_mach")
        except Exception as ex:
            full["double_mach"]["batched"] = {"error": f"{type(ex).__name__}: {ex}"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        sc = g.scalars()
        n_int, dt = cpu_sample(cfg, keys, prim, (sc["lambda_x"], sc["lambda_y"]), sc["tstep"], args.cpu_steps)
        cpu = {"value": n_int * args.cpu_steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{args.cpu_steps} RK3 step(s) of the same mesh, OpenMP restatement of Time_advance_RK"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_desc(len(keys), NI),
                "roofline": {"bound": "hbm", "achieved": face_gbs, "peak": hbm_peak, "unit": "GB/s",
                             "frac": face_gbs / hbm_peak, "traffic": traffic,
                             "kernel": f"face flux (x+y), autotuned variant {tuned}",
                             "ms_per_launch": kt["faces"],
                             "algorithmic_bytes": face_bytes,
                             "achieved_from_traffic_gbs": (traffic / (kt["faces"] * 1e-3) / 1e9) if traffic else None,
                             "traffic_profile_kernel": profile_text("traffic_kernel"),
                             "note": "achieved/frac use the algorithmic bytes; traffic is the ncu DRAM bytes of "
                                     "one x+y pair of the profiled kernel",
                             "peak_source": "measured" if peaks else "fallback"},
                "roofline_fp64": {"achieved": face_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                                  "frac": face_tflops / fp64_peak, "flops_per_face": FLOPS_PER_FACE,
                                  "peak_source": "measured DFMA probe",
                                  "fp64_pipe_active_pct_ncu": profile_figure("fp64_pipe_active_pct"),
                                  "note": "a correctly rounded division is one flop here but several FP64-pipe "
                                          "instructions; the pipe figure is ncu's, from profiles/"},
                "step_hbm": {"algorithmic_bytes_per_update": BYTES_PER_UPDATE, "achieved_gbs": step_gbs,
                             "frac": step_gbs / hbm_peak},
                "kernel_ms": kt, "autotune": {"face_variant": tuned, "ms_per_variant": list(tune_ms),
                                              "nr_fallback_faces": list(g.nr_fallbacks())},
                "clocks": clocks, "e2e": e2e, "gpu_launches": launches_per_step * args.steps,
                "counters": cnt, "state_finite_after_timed_steps": finite, "cpu_baseline": cpu,
                "fast_flux": fastf, "learned": gated, "ensemble": ens, "full_run": full, "strips": strips}
        line["summary"] = summary(line)      # last key: the end of the line carries the key figures
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    g.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-full-run", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-strips", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
