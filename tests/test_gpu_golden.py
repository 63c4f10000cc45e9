"""The GPU solver (libfdm through the C-ABI) against the oracle's golden final
states of whole runs with regrids: bit-identical leaf sets and states after
the configuration-1 vortex (200 steps, 20 regrids), the four-quadrant
problem at 32^2 / 2 levels, the double Mach reflection at 64x16 / 2 levels
and 128x32 / 3 levels to t = 0.2 (698 steps with 140 regrids, 3011 steps with
603 regrids), and (when recorded) the four-quadrant problem at 128^2 / 4
levels to t = 0.3 (6032 steps, 604 regrids) and the Mach-10 reflection at
256x64 / 4 levels to t = 0.2 (12939 steps, 2588 regrids)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

from fdm_cell_based_amr_cartesian_b200.solver import Solver  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_runs.json")))


@pytest.mark.parametrize("name", sorted(make_golden.cases(long=True)))
def test_gpu_reproduces_golden_run(name):
    if name not in GOLDEN:
        pytest.skip("not recorded")
    make, steps = make_golden.cases(long=True)[name]
    cfg = make()
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    n = 0
    if steps is not None:
        n = g.solute(steps)
    else:
        while g.scalars()["tt"] < cfg.params.t_end:
            k = g.solute(100)
            n += k
            if k == 0:
                break
    keys, prim = g.leaves()
    rec = make_golden.digest(keys, prim)
    want = GOLDEN[name]
    assert n == want["steps"]
    assert g.counters()["n_regrids"] == want["regrids"]
    assert g.counters()["n_gm4_nonleaf"] == want["gm4_nonleaf"]
    for k in ("n_leaves", "sha256_keys", "sha256_prim"):
        assert rec[k] == want[k], (k, rec, want)


@pytest.mark.parametrize("name", ["riemann4_32_l2_to_t0.3", "double_mach_64x16_l2_to_t0.2"])
def test_batched_persistent_kernel_reproduces_golden_run(name):
    """The same whole runs through the batched path (a batch of one member,
    the persistent kernel at 2 blocks per SM, regrids when due), after the
    autotuner has picked the face launch shape."""
    from fdm_cell_based_amr_cartesian_b200.solver import Batch
    make, steps = make_golden.cases(long=True)[name]
    cfg = make()
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    g.autotune(reps=2)
    b = Batch([g])
    b.set_blocks_per_sm(2)
    n = 0
    while g.scalars()["tt"] < cfg.params.t_end:
        k = b.solute(50)
        n += k
        if k == 0:
            break
    b.sync()
    keys, prim = g.leaves()
    rec = make_golden.digest(keys, prim)
    want = GOLDEN[name]
    assert n == want["steps"] and g.counters()["n_regrids"] == want["regrids"]
    for k in ("n_leaves", "sha256_keys", "sha256_prim"):
        assert rec[k] == want[k], (k, rec, want)
    b.close()
    g.close()
