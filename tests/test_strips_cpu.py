"""Strips of one mesh with halo exchange, on CPU through the oracle: the
row split, the plan's leaf ranges, and whole runs of 2-3 strips (in one
process, and as two gloo ranks) that must end bit-identical to the same
mesh advanced whole."""
import os
import socket

import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200 import strips as SP
import oracle_strips as OS
from fdm_cell_based_amr_cartesian_b200.solver import distance_refined_keys, initial_state

BAND = [0.2, 0.15]


def riemann_mesh(base=32, levels=2):
    cfg = P.riemann4(base=base, lvl_amr=levels)
    cfg.params.iflag_amr = 0
    keys = distance_refined_keys(cfg, [("x", 0.5), ("y", 0.5)], BAND[:levels])
    return cfg, keys, initial_state(cfg, keys)


def dmr_mesh():
    cfg = P.double_mach(base_y=16, lvl_amr=2, t_end=0.2)
    cfg.params.iflag_amr = 0
    # refined bands across the shock foot and along the rows the strips cut
    keys = distance_refined_keys(cfg, [("x", 0.6), ("y", 0.5)], [0.3, 0.15])
    return cfg, keys, initial_state(cfg, keys)


def test_split_rows_balanced():
    cfg, keys, _ = riemann_mesh()
    for ns in (1, 2, 3, 5):
        r = SP.split_rows(keys, cfg.m, cfg.n, ns)
        assert r[0][0] == 3 and r[-1][1] == cfg.n - 3
        assert all(b - a >= 3 for a, b in r)
        assert all(r[i][1] == r[i + 1][0] for i in range(ns - 1))
    with pytest.raises(ValueError):
        SP.split_rows(keys, cfg.m, cfg.n, cfg.n)
    with pytest.raises(ValueError):
        SP.StripPlan(P.vortex(), distance_refined_keys(P.vortex(), [("x", 5.0)], [1.0]), 2)


def test_plan_ranges_and_gather():
    cfg, keys, prim = riemann_mesh()
    plan = SP.StripPlan(cfg, keys, 3)
    rows = SP.key_rows(keys, cfg.m)
    for st in plan.strips:
        assert st.params.window_row0 == st.row0 and st.params.window_rows == st.rows
        lr = rows[st.sel]
        a, b = st.own
        assert np.all(lr[slice(*st.recv_down)] < a) and np.all(lr[slice(*st.recv_up)] >= b)
        assert np.all((lr[slice(*st.send_up)] >= b - 3) & (lr[slice(*st.send_up)] < b))
        # local keys name roots relative to the strip
        assert np.array_equal(st.keys + np.uint64((st.row0 * cfg.m) << 34), keys[st.sel])
    assert plan.strips[0].params.kind_ymbc == cfg.params.kind_ymbc
    assert plan.strips[0].params.kind_ypbc == P.BC_EXCHANGE
    assert plan.strips[1].params.kind_ymbc == P.BC_EXCHANGE
    k, v = plan.gather([(st.keys, prim[st.sel]) for st in plan.strips])
    assert np.array_equal(k, keys) and np.array_equal(v, prim)


def whole_run(oracle_mod, cfg, keys, prim, nsteps):
    o = oracle_mod.Oracle(cfg, threads=2, initial=False)
    o.set_leaves(keys, prim)
    for _ in range(nsteps):
        assert o.solute_step() == 0
    k, v, _ = o.leaves()
    sc = o.scalars()
    o.close()
    return k, v, sc


@pytest.mark.parametrize("mesh,nstrips", [(riemann_mesh, 3), (dmr_mesh, 2)])
def test_oracle_strips_equal_whole_mesh(oracle_mod, mesh, nstrips):
    cfg, keys, prim = mesh()
    nsteps = 4
    k0, v0, sc0 = whole_run(oracle_mod, cfg, keys, prim, nsteps)
    plan = SP.StripPlan(cfg, keys, nstrips)
    engines = [OS.OracleStrip(plan, s, prim, oracle_mod) for s in range(nstrips)]
    tt, it, k = SP.run(engines, SP.LocalExchange(engines), nsteps, cfg.params.t_end)
    assert k == nsteps and tt == sc0["tt"]
    kg, vg = plan.gather([e.leaves() for e in engines])
    for e in engines:
        e.close()
    assert np.array_equal(kg, k0)
    assert np.array_equal(vg, v0)          # bit for bit


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import datetime
    import oracle as oracle_mod
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, keys, prim = riemann_mesh()
        plan = SP.StripPlan(cfg, keys, world)
        e = OS.OracleStrip(plan, rank, prim, oracle_mod)
        tt, it, k = SP.run([e], SP.DistExchange(e, rank, world), 4, cfg.params.t_end)
        lk, lv = e.leaves()
        q.put((rank, tt, lk, lv))
        e.close()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_strips_equal_whole_mesh(oracle_mod):
    import torch.multiprocessing as mp
    cfg, keys, prim = riemann_mesh()
    k0, v0, sc0 = whole_run(oracle_mod, cfg, keys, prim, 4)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=240) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == sc0["tt"]
    plan = SP.StripPlan(cfg, keys, 2)
    kg, vg = plan.gather([(o[2], o[3]) for o in out])
    assert np.array_equal(kg, k0) and np.array_equal(vg, v0)


def test_strip_parameters_validated_before_any_device_call():
    """fdm_create refuses inconsistent strip parameters before touching CUDA."""
    import ctypes
    from fdm_cell_based_amr_cartesian_b200.solver import load_library
    L = load_library()
    cfg, keys, _ = riemann_mesh()
    plan = SP.StripPlan(cfg, keys, 2)

    def create(q):
        h = ctypes.c_void_p()
        return L.fdm_create(ctypes.byref(q), ctypes.byref(h))

    def variant(s, **kw):
        q = P.FdmParams.from_buffer_copy(plan.strips[s].params)
        for k, v in kw.items():
            setattr(q, k, v)
        return q

    assert create(variant(0, window_rows=8)) == 1                       # < 3 owned rows
    assert create(variant(0, kind_ypbc=P.BC_TRANSMISSIVE)) == 1         # cut side not exchanged
    assert create(variant(1, kind_ypbc=P.BC_EXCHANGE)) == 1             # mesh edge exchanged
    assert create(variant(0, window_rows=cfg.n + 1)) == 1               # beyond the mesh
    assert create(variant(0, kind_xmbc=P.BC_EXCHANGE)) == 1             # x sides are never cut
    assert create(variant(0, kind_ymbc=P.BC_PERIODIC)) == 7             # image in another strip
    whole = P.FdmParams.from_buffer_copy(cfg.params)
    whole.kind_ypbc = P.BC_EXCHANGE
    assert create(whole) == 1                                           # exchange without a strip


def oracle_start(oracle_mod, cfg):
    """The whole mesh after creat_mesh + initial (roots, ghosts filled) as
    (keys, U(1:7)), and the oracle holding it."""
    o = oracle_mod.Oracle(cfg, threads=2)
    k, _, _ = o.leaves()
    return o, k, o.get_U(np.arange(len(k)))


@pytest.mark.parametrize("make,nstrips,nsteps", [
    (lambda: P.riemann4(base=32, lvl_amr=2), 3, 25),
    (lambda: P.double_mach(base_y=16, lvl_amr=2, t_end=0.2), 2, 12),
    (lambda: P.double_mach(base_y=16, lvl_amr=2, t_end=0.2), 3, 16),
])
def test_oracle_strip_run_with_regrids(oracle_mod, make, nstrips, nsteps):
    """The time loop with AMR on: ghost refresh after every step, regrids on
    the regrid host and a new split; leaf sets and states after every regrid
    equal the whole run's."""
    cfg = make()
    whole, keys, U = oracle_start(oracle_mod, cfg)
    run = SP.StripRun(cfg, keys, U, nstrips,
                      lambda plan, s, v: OS.OracleStrip(plan, s, v, oracle_mod),
                      lambda k, v: OS.OracleRegridHost(cfg, k, v, oracle_mod, threads=2))
    for _ in range(nsteps):
        assert whole.solute_step() == 0
        run.solute_step()
    assert run.regrids >= 2 and run.tt == whole.scalars()["tt"]
    kw, pw, Tw = whole.leaves()
    ks, Us = run.gather()
    run.close()
    whole.close()
    assert np.array_equal(ks, kw)
    assert np.array_equal(Us[:, [0, 1, 2, 4]], pw) and np.array_equal(Us[:, 3], Tw)


def _rank_amr(rank, world, port, q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import datetime
    import oracle as oracle_mod
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = P.riemann4(base=32, lvl_amr=2)
        o, keys, U = oracle_start(oracle_mod, cfg)
        o.close()
        run = SP.StripRun(cfg, keys, U, world,
                          lambda plan, s, v: OS.OracleStrip(plan, s, v, oracle_mod),
                          lambda k, v: OS.OracleRegridHost(cfg, k, v, oracle_mod), rank=rank)
        run.solute(22)
        out = run.gather()
        q.put((rank, run.tt, run.regrids, out))
        run.close()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_strip_run_with_regrids(oracle_mod):
    import torch.multiprocessing as mp
    cfg = P.riemann4(base=32, lvl_amr=2)
    whole, _, _ = oracle_start(oracle_mod, cfg)
    for _ in range(22):
        whole.solute_step()
    kw, pw, _ = whole.leaves()
    tt = whole.scalars()["tt"]
    whole.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_amr, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=240) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1] == tt and out[0][2] == 3
    ks, Us = out[0][3]
    assert out[1][3] is None
    assert np.array_equal(ks, kw) and np.array_equal(Us[:, [0, 1, 2, 4]], pw)


def test_plan_refuses_bad_leaf_sets():
    cfg, keys, _ = riemann_mesh()
    with pytest.raises(ValueError):
        SP.StripPlan(cfg, keys[::-1], 2)                       # not in key order
    with pytest.raises(ValueError):
        SP.StripPlan(cfg, np.concatenate([keys[:1], keys]), 2)  # a duplicate leaf
    plan = SP.StripPlan(cfg, keys, 2)
    with pytest.raises(ValueError):
        SP.StripPlan(plan.config(0), keys, 2)                  # already a strip
    one = SP.StripPlan(cfg, keys, 1)                           # one strip: the whole mesh
    assert one.strips[0].params.window_rows == 0 and len(one.strips[0].keys) == len(keys)
