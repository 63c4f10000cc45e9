"""Command-line run of one configuration, in the place of the reference's
main program (src/MAIN.F90:1-25: set_parameter, creat_mesh, idneighbor,
initial, solute), without its file output.

    python -m fdm_cell_based_amr_cartesian_b200 --case riemann4 --base 128 --lvl-amr 4 --steps 200

runs the four-quadrant problem on a 128^2 background with 4 levels for 200
steps (or to t_end when --steps is 0) with device regrids every nstep_adapt
steps, and prints one JSON line: steps, seconds, the solver's counters and
the device time of each regrid phase, summed over the run.

    --block LVL X1 X2 Y1 Y2 BUF

adds creat_mesh's static block refinement (lvlBlock, Block_size,
BufferLayerLVL of src/MAIN.F90:42-45) to the initial mesh, and

    --output DIR [--dump-every N]

writes the reference's diagnostic files there (Residual.dat every 100 steps
and at t_end, accuracy_error.dat at t_end with the norms formed on the
device; src/solution.F90:217-234) and, with --dump-every, a field dump of
the leaves (field_<it>.npz) every N steps, read back while the run goes on.

    --strips N

runs the configuration as N strips of background rows with the halo
exchange after every stage (all on this GPU); under torchrun (WORLD_SIZE > 1)
one strip per rank over NCCL, rank 0 holding the whole-mesh regrid host:

    python -m torch.distributed.run --nproc-per-node 4 --master-addr 127.0.0.1 \
        -m fdm_cell_based_amr_cartesian_b200 --case riemann4 --base 128 --lvl-amr 4 --strips 4

    --save-config FILE / --config FILE

write the configuration's parameters as JSON / run from such a file
(every fdm_params field, the initial condition, the block refinement).

    --case ensemble --members 64 [--bps 0|1|2] [--plain] [--save-leaves F.npz]

runs the ensemble configuration (random four-quadrant members, seeds from
1000, maximum level drawn from 2..5, learned gate on unless --plain) as one
batch to each member's t_end (or --steps), regrids included, and prints the
per-member steps and leaf counts.  The gate itself is trained
by ``python -m fdm_cell_based_amr_cartesian_b200.learned``.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

from . import params as P
from .solver import Solver


# options that set the configuration itself (refused beside --config FILE)
CONFIG_OPTIONS = ("case", "base", "lvl_amr", "t_end", "block", "members")


def config(args) -> P.Config:
    path = getattr(args, "config", None)
    if path:
        with open(path) as f:
            return P.config_from_dict(json.load(f))
    if args.case == "riemann4":
        cfg = P.riemann4(base=args.base, lvl_amr=args.lvl_amr, t_end=args.t_end or 0.3)
    elif args.case == "vortex":
        cfg = P.vortex(base=args.base, lvl_amr=args.lvl_amr)
        if args.t_end:
            cfg.params.t_end = args.t_end
    elif args.case == "double_mach":
        cfg = P.double_mach(base_y=args.base, lvl_amr=args.lvl_amr, t_end=args.t_end or 0.2)
    elif args.case == "reference":
        cfg = P.reference_default()
    else:
        raise SystemExit(f"unknown case {args.case}")
    block = getattr(args, "block", None)
    if block:
        lvl, x1, x2, y1, y2, buf = block
        P.with_block(cfg, int(lvl), (float(x1), float(x2), float(y1), float(y2)), int(buf))
    return cfg


def run_strips(args, cfg) -> int:
    """The configuration on strips of one mesh (strips.StripRun): all in this
    process, or one per rank of a torchrun world (NCCL)."""
    import datetime

    import torch

    from . import strips as SP
    if P.BC_PERIODIC in (cfg.params.kind_ymbc, cfg.params.kind_ypbc):
        raise SystemExit(f"--strips: {args.case} has periodic y sides, which cannot be cut into strips")
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    nstrips = args.strips if world == 1 else world
    if world > 1:
        import torch.distributed as dist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", torch.cuda.current_device())
    # creat_mesh + initial with the ghost fill of the whole mesh, on rank 0
    box = [None]
    if rank == 0:
        g0 = Solver(cfg)
        g0.creat_mesh_and_initial()
        box = [g0.leaves()]
        g0.close()
    if world > 1:
        torch.distributed.broadcast_object_list(box, src=0)
    keys, prim = box[0]
    run = SP.StripRun(cfg, keys, prim, nstrips,
                      lambda plan, s, v: SP.GpuStrip(plan, s, v, asynchronous=True),
                      lambda k, v: SP.GpuRegridHost(cfg, k, v),
                      rank=None if world == 1 else rank, device=dev)
    t0 = time.perf_counter()
    target = args.steps if args.steps > 0 else None
    n = 0
    while (target is None or n < target) and run.tt < cfg.params.t_end:
        k = run.solute(min(100, target - n) if target is not None else 100)
        n += k
        if k == 0:
            break
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    whole = run.gather()
    if rank == 0:
        print(json.dumps({"case": args.case, "strips": nstrips, "ranks": world, "steps": n,
                          "seconds": seconds, "tt": run.tt, "regrids": run.regrids,
                          "leaves": int(len(whole[0]))}))
    run.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def run_ensemble(args) -> int:
    """The ensemble configuration as one batch (fdm_batch_solute), each
    member to its own t_end; learned gate on unless --plain.  Prints the
    whole run's time and the per-member steps, leaf counts (interior leaves
    at the start and at the end; smallest and largest member) and times."""
    from . import ensemble as E
    from . import learned
    from .solver import Batch
    cfgs = E.ensemble_configs(seeds=tuple(range(1000, 1000 + args.members)))
    sols = []
    for cfg, (k, p) in zip(cfgs, E.ensemble_meshes(cfgs)):
        g = Solver(cfg)
        g.upload(k, p)
        g.body_boundary(1)
        if not args.plain:
            learned.enable(g)
        sols.append(g)
    import numpy as np

    from .solver import FdmError
    lv0 = [g.counters()["n_interior"] for g in sols]
    peak = list(lv0)
    active = list(range(len(sols)))
    nan_members = []
    batch = Batch(sols)
    batch.set_blocks_per_sm(args.bps)
    t0 = time.perf_counter()
    n = 0
    target = args.steps if args.steps > 0 else None
    while target is None or n < target:
        try:
            k = batch.solute(min(100, target - n) if target is not None else 100)
        except FdmError as ex:
            # a member whose residual turned NaN stops (the reference stops
            # there); the others go on in a batch without it
            if ex.code != 3:
                raise
            bad = [i for i in active if np.isnan(np.asarray(sols[i].residual()[1])).any()]
            if not bad:
                raise
            nan_members += [{"seed": 1000 + i, "lvl_amr": int(cfgs[i].params.lvl_amr),
                             "step": sols[i].scalars()["it"], "tt": sols[i].scalars()["tt"]} for i in bad]
            active = [i for i in active if i not in bad]
            batch.close()
            if not active:
                break
            batch = Batch([sols[i] for i in active])
            batch.set_blocks_per_sm(args.bps)
            continue
        n += k
        for i in active:
            peak[i] = max(peak[i], sols[i].counters()["n_interior"])
        if k == 0 or all(sols[i].scalars()["tt"] >= sols[i].cfg.params.t_end for i in active):
            break
    if active:
        batch.sync()
    seconds = time.perf_counter() - t0
    sc = [g.scalars() for g in sols]
    lv1 = [g.counters()["n_interior"] for g in sols]
    tts = [s["tt"] for s in sc]
    out = {"case": "ensemble", "gate": not args.plain, "members": len(sols), "steps": n, "seconds": seconds,
           "interior_leaves_at_start": sum(lv0), "interior_leaves_at_end": sum(lv1),
           "member_interior_leaves_at_start": [min(lv0), max(lv0)],
           "member_interior_leaves_peak": [min(peak), max(peak)],
           "member_interior_leaves_at_end": [min(lv1), max(lv1)],
           "member_steps": [min(s["it"] for s in sc), max(s["it"] for s in sc)],
           "members_stopped_by_nan": nan_members,
           "regrids": sum(g.counters()["n_regrids"] for g in sols),
           "members_at_t_end": sum(1 for g, t in zip(sols, tts) if t >= g.cfg.params.t_end),
           "tt_min": min(tts), "tt_max": max(tts), "batch": batch.info() if active else None,
           "per_member": [{"seed": 1000 + i, "lvl_amr": int(c.params.lvl_amr), "steps": s["it"], "tt": s["tt"],
                           "interior_leaves": [a, p, b]}
                          for i, (c, s, a, p, b) in enumerate(zip(cfgs, sc, lv0, peak, lv1))]}
    if args.save_leaves:
        import numpy as np
        np.savez(args.save_leaves, **{f"m{i}_keys": g.leaves()[0] for i, g in enumerate(sols)},
                 **{f"m{i}_prim": g.leaves()[1] for i, g in enumerate(sols)})
    if active:
        batch.close()
    for g in sols:
        g.close()
    print(json.dumps(out))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m fdm_cell_based_amr_cartesian_b200")
    ap.add_argument("--case", default="riemann4",
                    choices=["riemann4", "vortex", "double_mach", "reference", "ensemble"])
    ap.add_argument("--members", type=int, default=64, help="ensemble members (--case ensemble)")
    ap.add_argument("--config", default=None, help="run the configuration in this JSON file")
    ap.add_argument("--save-config", default=None, help="write the configuration as JSON and exit")
    ap.add_argument("--strips", type=int, default=0,
                    help="run as this many strips with halo exchange (one per rank under torchrun)")
    ap.add_argument("--bps", type=int, default=0,
                    help="ensemble: 1 or 2 blocks per SM of the persistent kernel, 0 the members' own graphs")
    ap.add_argument("--base", type=int, default=128, help="background cells (per side; rows for double_mach)")
    ap.add_argument("--lvl-amr", type=int, default=4)
    ap.add_argument("--t-end", type=float, default=0.0, help="end time (0: the case's own)")
    ap.add_argument("--steps", type=int, default=0, help="steps to run (0: run to t_end)")
    ap.add_argument("--gate", action="store_true", help="learned face gate on")
    ap.add_argument("--plain", action="store_true", help="ensemble: learned gate off")
    ap.add_argument("--save-leaves", default=None, help="ensemble: write every member's final leaves (.npz)")
    ap.add_argument("--output", default=None, help="directory for Residual.dat / accuracy_error.dat")
    ap.add_argument("--dump-every", type=int, default=0,
                    help="field dump (keys, rho, u, v, p as field_<it>.npz in --output) every this many steps")
    ap.add_argument("--block", nargs=6, metavar=("LVL", "X1", "X2", "Y1", "Y2", "BUF"), default=None,
                    help="static block refinement of the initial mesh (lvlBlock, Block_size, BufferLayerLVL)")
    argv = list(sys.argv[1:] if argv is None else argv)
    args = ap.parse_args(argv)
    if args.config:
        # the file fixes the configuration: options that would change it are refused
        given = [o for a in ap._actions if a.dest in CONFIG_OPTIONS for o in a.option_strings
                 if any(t == o or t.startswith(o + "=") for t in argv)]
        if given:
            ap.error(f"--config FILE fixes the configuration; drop {', '.join(given)}")
    if args.case == "ensemble":
        return run_ensemble(args)

    cfg = config(args)
    if args.save_config:
        with open(args.save_config, "w") as f:
            json.dump(P.config_to_dict(cfg), f, indent=1)
        return 0
    if args.strips > 1 or int(os.environ.get("WORLD_SIZE", "1")) > 1:
        return run_strips(args, cfg)
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    if args.gate:
        from . import learned
        learned.enable(g)
    diag = dump = None
    if args.output:
        from .output import PSTEP_RES, Output
        diag = Output(args.output)
    if args.dump_every > 0:
        from .output import FieldDump
        dump = FieldDump(args.output or "Output")
    # chunks end on multiples of Pstep_Res = 100, where output_Res writes,
    # and of the dump interval
    every = 100 if dump is None else min(100, args.dump_every)
    t0 = time.perf_counter()
    n = 0
    target = args.steps if args.steps > 0 else None
    while (target is None or n < target) and g.scalars()["tt"] < cfg.params.t_end:
        it0 = g.scalars()["it"]
        k = g.solute(min(every - it0 % every, target - n) if target is not None else every - it0 % every)
        n += k
        sc = g.scalars()
        if diag is not None and (sc["it"] % PSTEP_RES == 0 or sc["tt"] == cfg.params.t_end):
            print(diag.res(g), file=sys.stderr)
        if dump is not None and sc["it"] % args.dump_every == 0:
            dump.dump(g)
        if k == 0:
            break
    tt = g.scalars()["tt"]   # waits for the device
    seconds = time.perf_counter() - t0
    if diag is not None and tt == cfg.params.t_end:
        diag.error(g)
    if dump is not None:
        dump.close()
    out = {"case": args.case, "steps": n, "seconds": seconds, "tt": tt,
           "counters": g.counters(), "regrid_device_ms_total": g.amr_phase_ms(total=True)}
    g.close()
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
