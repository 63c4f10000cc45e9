"""Strips of one mesh on one GPU (libfdm strip handles, halo rows exchanged
by device copies after every stage) against the same mesh advanced whole by
one handle and by the oracle: bit-identical leaf states.  The largest case
is the benchmark's 1.08M-leaf four-quadrant mesh in 4 strips."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200 import strips as SP
from fdm_cell_based_amr_cartesian_b200.solver import FdmError, Solver, distance_refined_keys, initial_state
from test_strips_cpu import dmr_mesh, riemann_mesh, whole_run

pytestmark = pytest.mark.gpu


def whole_gpu(cfg, keys, prim, nsteps):
    g = Solver(cfg)
    g.upload(keys, prim)
    for _ in range(nsteps):
        g.solute_step()
    k, v = g.leaves()
    sc = g.scalars()
    g.close()
    return k, v, sc


def strips_gpu(cfg, keys, prim, nstrips, nsteps, asynchronous=False):
    plan = SP.StripPlan(cfg, keys, nstrips)
    engines = [SP.GpuStrip(plan, s, prim, asynchronous) for s in range(nstrips)]
    tt, it, k = SP.run(engines, SP.LocalExchange(engines), nsteps, cfg.params.t_end)
    parts = [e.leaves() for e in engines]
    for st, (lk, _) in zip(plan.strips, parts):
        assert np.array_equal(lk, st.keys)
    for e in engines:
        e.close()
    kg, vg = plan.gather(parts)
    return kg, vg, tt, k


@pytest.mark.parametrize("asynchronous", [False, True])
@pytest.mark.parametrize("mesh,nstrips", [(riemann_mesh, 3), (dmr_mesh, 2), (dmr_mesh, 4)])
def test_gpu_strips_equal_whole_mesh(oracle_mod, mesh, nstrips, asynchronous):
    cfg, keys, prim = mesh()
    nsteps = 5
    k0, v0, sc0 = whole_gpu(cfg, keys, prim, nsteps)
    ko, vo, _ = whole_run(oracle_mod, cfg, keys, prim, nsteps)
    assert np.array_equal(v0, vo)
    kg, vg, tt, k = strips_gpu(cfg, keys, prim, nstrips, nsteps, asynchronous)
    assert k == nsteps and tt == sc0["tt"]
    assert np.array_equal(kg, k0)
    assert np.array_equal(vg, v0)


@pytest.mark.parametrize("asynchronous", [False, True])
def test_gpu_strips_benchmark_mesh(asynchronous):
    cfg = P.riemann4(base=128, lvl_amr=4)
    cfg.params.iflag_amr = 0
    keys = distance_refined_keys(cfg, [("x", 0.5), ("y", 0.5)], [0.2, 0.15, 0.1, 0.05])
    prim = initial_state(cfg, keys)
    k0, v0, sc0 = whole_gpu(cfg, keys, prim, 3)
    kg, vg, tt, k = strips_gpu(cfg, keys, prim, 4, 3, asynchronous)
    assert len(keys) > 1_000_000
    assert tt == sc0["tt"]
    assert np.array_equal(kg, k0) and np.array_equal(vg, v0)


def test_gpu_strip_errors():
    import torch
    cfg, keys, prim = riemann_mesh()
    plan = SP.StripPlan(cfg, keys, 2)
    e = SP.GpuStrip(plan, 0, prim)
    # a strip takes no regrid
    with pytest.raises(FdmError) as ex:
        e.g.amr()
    assert ex.value.code == 7
    # a slot outside the leaf slots is refused (skipped on the device)
    bad = torch.tensor([0, 1 << 30], dtype=torch.int32, device="cuda")
    buf = torch.zeros((2, 4), dtype=torch.float64, device="cuda")
    with pytest.raises(FdmError) as ex:
        e.g.pack_slots(bad.data_ptr(), 2, buf.data_ptr())
    assert ex.value.code == 1
    with pytest.raises(FdmError):
        e.g.step_control_global(1.0, 1.0, 99)
    e.close()


@pytest.mark.parametrize("make,nstrips,nsteps,asynchronous", [
    (lambda: P.riemann4(base=32, lvl_amr=2), 3, 25, False),
    (lambda: P.double_mach(base_y=16, lvl_amr=2, t_end=0.2), 2, 12, False),
    (lambda: P.riemann4(base=128, lvl_amr=4), 4, 31, False),      # configuration 2, 4 regrids
    (lambda: P.riemann4(base=128, lvl_amr=4), 4, 31, True),
])
def test_gpu_strip_run_with_regrids(make, nstrips, nsteps, asynchronous):
    """The time loop with AMR on, strips on one GPU and the regrid host
    beside them: the same leaf sets and states as the whole handle."""
    cfg = make()
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    keys, prim = g.leaves()
    run = SP.StripRun(cfg, keys, prim, nstrips, lambda plan, s, v: SP.GpuStrip(plan, s, v, asynchronous),
                      lambda k, v: SP.GpuRegridHost(cfg, k, v))
    for _ in range(nsteps):
        g.solute_step()
        run.solute_step()
    assert run.regrids >= 3 and run.tt == g.scalars()["tt"]
    kw, pw = g.leaves()
    ks, ps = run.gather()
    run.close()
    g.close()
    assert np.array_equal(ks, kw) and np.array_equal(ps, pw)
