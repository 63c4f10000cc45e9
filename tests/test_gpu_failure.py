"""Failure detection without a GPU fault.

- The batched kernel's grid barrier, made to wait for a block that never
  arrives, gives up at its time limit and the host reads FDM_ERR_TIMEOUT;
  the context stays usable (a step after it still matches the oracle).
- The same on a real batch whose wait limit is set below a phase's length.
- Device allocations refused on the host (an injected cudaMalloc failure)
  give FDM_ERR_NOMEM and leave no half-built handle that could be run."""
import ctypes

import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import Solver, load_library

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_is_reported(oracle_mod):
    L = load_library()
    secs = ctypes.c_double(-1.0)
    assert L.fdm_debug_barrier_timeout(ctypes.byref(secs)) == 4     # FDM_ERR_TIMEOUT
    assert 0.1 < secs.value < 60.0
    cfg = P.vortex()
    o = oracle_mod.Oracle(cfg)
    o.solute(3)
    keys, prim, _ = o.leaves()
    s = o.scalars()
    g = Solver(cfg)
    g.upload(keys, prim)
    g.set_scalars(s["lambda_x"], s["lambda_y"], s["tstep"], s["tt"], s["it"])
    o.solute_step()
    g.solute_step()
    assert np.array_equal(g.leaves()[1], o.leaves()[1])
    g.close()
    o.close()


def _no_regrid(cfg):
    cfg.params.nstep_adapt = 10 ** 9    # no regrid in these few steps
    return cfg


def test_batch_barrier_limit_reports_timeout():
    """A real batch with a grid-barrier wait limit of a microsecond: some
    wait of the persistent kernel runs past it, fdm_batch_solute returns
    FDM_ERR_TIMEOUT (not FDM_ERR_CUDA); the members restored by upload and
    the default limit give the steps of the same meshes advanced alone."""
    from fdm_cell_based_amr_cartesian_b200.solver import Batch, FdmError
    cfgs = [_no_regrid(P.vortex()), _no_regrid(P.riemann4(base=32, lvl_amr=2))]
    members, twins = [], []
    for c in cfgs:
        a, b = Solver(c), Solver(c)
        a.creat_mesh_and_initial()
        b.creat_mesh_and_initial()
        members.append(a)
        twins.append(b)
    batch = Batch(members)
    batch.set_blocks_per_sm(2)
    assert batch.solute(2) == 2
    saved = [(m.leaves(), m.scalars()) for m in members]
    batch.set_wait_limit(1e-6)
    with pytest.raises(FdmError) as ei:
        batch.solute(1)
    assert ei.value.code == 4, str(ei.value)             # FDM_ERR_TIMEOUT
    batch.set_wait_limit(2.0)
    for m, ((k, p), s) in zip(members, saved):
        m.upload(k, p)
        m.set_scalars(s["lambda_x"], s["lambda_y"], s["tstep"], s["tt"], s["it"])
    assert batch.solute(3) == 3
    for m, t in zip(members, twins):
        t.solute(5)
        km, pm = m.leaves()
        kt, pt = t.leaves()
        assert np.array_equal(km, kt)
        assert np.array_equal(pm, pt)
    batch.close()
    for s in members + twins:
        s.close()


def test_allocation_failure_reports_nomem(oracle_mod):
    """Host-side injection of a failing device allocation at every point of
    create / upload / regrid: the call returns FDM_ERR_NOMEM, a handle left
    half-built is refused (FDM_ERR_STATE) instead of run, and after the
    injection ends the same handle uploads again and steps as the oracle."""
    from fdm_cell_based_amr_cartesian_b200.solver import FdmError
    L = load_library()
    cfg = P.vortex()
    o = oracle_mod.Oracle(cfg)
    o.solute(12)
    keys, prim, _ = o.leaves()
    s = o.scalars()
    o.solute_step()
    ko, po, _ = o.leaves()
    o.close()
    failed = set()
    try:
        for after in range(0, 400, 2):
            if "regrid" in failed and after > 40:
                break
            L.fdm_debug_fail_alloc(after)
            try:
                g = Solver(cfg)
            except FdmError as e:
                assert e.code == 5, str(e)
                failed.add("create")
                continue
            for what, call in (("upload", lambda: g.upload(keys, prim)), ("regrid", g.amr)):
                try:
                    call()
                except FdmError as e:
                    assert e.code == 5, str(e)
                    failed.add(what)
                    assert g.num_leaves() == 0          # left not loaded
                    with pytest.raises(FdmError) as ei:
                        g.solute_step()
                    assert ei.value.code == 6, str(ei.value)   # FDM_ERR_STATE, nothing launched
                    break
            L.fdm_debug_fail_alloc(-1)
            g.upload(keys, prim)
            g.set_scalars(s["lambda_x"], s["lambda_y"], s["tstep"], s["tt"], s["it"])
            g.solute_step()
            kg, pg = g.leaves()
            assert np.array_equal(kg, ko) and np.array_equal(pg, po)
            g.close()
    finally:
        L.fdm_debug_fail_alloc(-1)
    assert {"create", "upload", "regrid"} <= failed, failed
