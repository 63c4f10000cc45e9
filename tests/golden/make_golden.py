"""Golden final states of the oracle (the CPU restatement of the reference's
solver) for whole runs with regrids, stored as digests in oracle_runs.json.

    python tests/golden/make_golden.py            # the short cases (about 2 min on 8 cores)
    python tests/golden/make_golden.py --long     # also the four-quadrant
                                                  # problem at 128^2, 4 levels
                                                  # (about 25 min on 8 cores)
                                                  # and the double Mach
                                                  # reflection at 256x64, 4 levels
    python tests/golden/make_golden.py --long --only NAME   # one case

A case is a configuration run with Oracle.solute from its initial condition
until t_end (or for a number of steps); the record holds the step count,
leaf count, regrid counters, SHA-256 of the leaf keys (uint64) and of the
primitive states (float64, (rho, u, v, p) per leaf) in key order, and a few
plain numbers for reading."""
import argparse
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

from fdm_cell_based_amr_cartesian_b200 import params as P  # noqa: E402

OUT = os.path.join(HERE, "oracle_runs.json")


def cases(long=False):
    c = {
        "vortex_200_steps": (lambda: P.vortex(), 200),
        "riemann4_32_l2_to_t0.3": (lambda: P.riemann4(base=32, lvl_amr=2, t_end=0.3), None),
        # the Mach-10 reflection: time-dependent top boundary, wall, inflow,
        # a regrid every 5 steps (the larger one has non-leaf refinements)
        "double_mach_64x16_l2_to_t0.2": (lambda: P.double_mach(base_y=16, lvl_amr=2, t_end=0.2), None),
        "double_mach_128x32_l3_to_t0.2": (lambda: P.double_mach(base_y=32, lvl_amr=3, t_end=0.2), None),
    }
    if long:
        c["riemann4_128_l4_to_t0.3"] = (lambda: P.riemann4(base=128, lvl_amr=4, t_end=0.3), None)
        c["double_mach_256x64_l4_to_t0.2"] = (lambda: P.double_mach(base_y=64, lvl_amr=4, t_end=0.2), None)
    return c


def digest(keys, prim):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    return {"n_leaves": int(len(keys)),
            "sha256_keys": hashlib.sha256(keys.tobytes()).hexdigest(),
            "sha256_prim": hashlib.sha256(prim.tobytes()).hexdigest(),
            "sum_rho": float(prim[:, 0].sum()), "max_rho": float(prim[:, 0].max()),
            "min_p": float(prim[:, 3].min())}


def run(make, steps, threads=None):
    import oracle
    cfg = make()
    o = oracle.Oracle(cfg, threads=threads or os.cpu_count())
    n = 0
    if steps is not None:
        n = o.solute(steps)
    else:
        while o.scalars()["tt"] < cfg.params.t_end:
            k = o.solute(100)
            n += k
            if k == 0:
                break
    keys, prim, _ = o.leaves()
    rec = digest(keys, prim)
    cnt = o.counters()
    rec.update({"steps": int(n), "tt": float(o.scalars()["tt"]), "regrids": int(cnt["regrids"]),
                "gm4_nonleaf": int(cnt["gm4_nonleaf"])})
    o.close()
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--long", action="store_true")
    ap.add_argument("--only", default=None, help="run this case alone")
    args = ap.parse_args()
    out = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name, (make, steps) in cases(args.long).items():
        if args.only and name != args.only:
            continue
        t0 = time.time()
        out[name] = run(make, steps)
        print(name, out[name], f"{time.time() - t0:.1f}s", flush=True)
        json.dump(out, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
