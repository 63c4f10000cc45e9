"""Batched ensemble path (one persistent launch per RK3 stage over many
meshes) against the same meshes advanced one by one: every member must end
bit-identical to its twin, through regrids, time-dependent boundaries, the
learned gate and members that reach t_end early."""
import os

import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import learned
from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import Batch, Solver

pytestmark = pytest.mark.gpu


def _cfgs(no_regrid=False):
    out = [P.vortex(), P.riemann4(base=32, lvl_amr=2), P.double_mach(base_y=12, lvl_amr=2),
           P.riemann4(base=40, lvl_amr=3)]
    if no_regrid:   # the first regrid would come after step 10**9
        for c in out:
            c.params.nstep_adapt = 10 ** 9
    return out


def _pair(cfg, gate=False):
    a, b = Solver(cfg), Solver(cfg)
    a.creat_mesh_and_initial()
    b.creat_mesh_and_initial()
    if gate:
        learned.enable(a)
        learned.enable(b)
    return a, b


def _assert_same(x, y):
    kx, px = x.leaves()
    ky, py = y.leaves()
    assert np.array_equal(kx, ky), "leaf sets differ"
    assert np.array_equal(px, py), f"values differ (max {np.max(np.abs(px - py)):.3e})"
    sx, sy = x.scalars(), y.scalars()
    for k in ("tt", "tstep", "lambda_x", "lambda_y", "it"):
        assert sx[k] == sy[k], (k, sx[k], sy[k])


def test_batch_solute_with_regrids_matches_single():
    cfgs = _cfgs()
    pairs = [_pair(c) for c in cfgs]
    batch = Batch([p[0] for p in pairs])
    n = batch.solute(25)
    assert n == 25
    for (bm, solo) in pairs:
        solo.solute(25)
        _assert_same(bm, solo)
    assert pairs[0][0].counters()["n_regrids"] >= 2


def test_batch_advance_matches_single_steps():
    cfgs = _cfgs(no_regrid=True)
    pairs = [_pair(c) for c in cfgs]
    batch = Batch([p[0] for p in pairs])
    batch.advance(6)
    batch.sync()
    for (bm, solo) in pairs:
        solo.solute(6)
        _assert_same(bm, solo)


@pytest.mark.skipif(not os.path.exists(learned.PARAMS_PATH), reason="no trained gate parameters")
def test_batch_with_gated_members_matches_single():
    cfgs = [P.riemann4(base=32, lvl_amr=2), P.riemann4(base=48, lvl_amr=2), P.vortex()]
    pairs = [_pair(c, gate=(k != 2)) for k, c in enumerate(cfgs)]
    batch = Batch([p[0] for p in pairs])
    assert batch.solute(23) == 23
    for (bm, solo) in pairs:
        solo.solute(23)
        _assert_same(bm, solo)
    assert learned.stats(pairs[0][0])[0] > 0


def test_members_reaching_t_end_stop():
    short = P.riemann4(base=32, lvl_amr=2, t_end=0.004)
    cfgs = [short, P.riemann4(base=32, lvl_amr=2)]
    pairs = [_pair(c) for c in cfgs]
    batch = Batch([p[0] for p in pairs])
    batch.solute(30)
    for (bm, solo) in pairs:
        solo.solute(30)
        _assert_same(bm, solo)
    assert pairs[0][0].scalars()["tt"] == pytest.approx(0.004)
    assert pairs[0][0].scalars()["it"] < 30 + 1


def test_one_and_two_blocks_per_sm_agree():
    cfgs = _cfgs(no_regrid=True)
    pa = [_pair(c) for c in cfgs]
    b1 = Batch([p[0] for p in pa])
    b2 = Batch([p[1] for p in pa])
    b1.set_blocks_per_sm(1)
    b2.set_blocks_per_sm(2)
    assert b1.info()["blocks_per_sm"] == 1
    b1.advance(4)
    b2.advance(4)
    b1.sync()
    b2.sync()
    for (x, y) in pa:
        _assert_same(x, y)


@pytest.mark.skipif(not os.path.exists(learned.PARAMS_PATH), reason="no trained gate parameters")
def test_streams_strategy_matches_single():
    """blocks_per_sm 0: no persistent kernel, each member's own step graph
    on its own stream; regrids, the gate and t_end as in the kernel path."""
    cfgs = _cfgs() + [P.riemann4(base=32, lvl_amr=2, t_end=0.004)]
    pairs = [_pair(c, gate=(k % 2 == 1)) for k, c in enumerate(cfgs)]
    batch = Batch([p[0] for p in pairs])
    batch.set_blocks_per_sm(0)
    assert batch.info()["blocks_per_sm"] == 0
    assert batch.solute(25) == 25
    for (bm, solo) in pairs:
        solo.solute(25)
        _assert_same(bm, solo)
    assert pairs[0][0].counters()["n_regrids"] >= 2


def test_streams_strategy_advance_matches_single_steps():
    cfgs = _cfgs(no_regrid=True)
    pairs = [_pair(c) for c in cfgs]
    batch = Batch([p[0] for p in pairs])
    batch.set_blocks_per_sm(0)
    batch.advance(6)
    batch.sync()
    for (bm, solo) in pairs:
        solo.solute(6)
        _assert_same(bm, solo)


@pytest.mark.skipif(not os.path.exists(learned.PARAMS_PATH), reason="no trained gate parameters")
@pytest.mark.parametrize("bps", [1, 2])
def test_branch_free_face_phases_match_single(bps):
    """The persistent kernel with the split-order, branch-free face flux
    (fdm_batch_set_face_flux(1)): plain and gated members, regrids; every
    member ends bit-identical to its twin advanced alone."""
    cfgs = _cfgs()
    pairs = [_pair(c, gate=(k % 2 == 1)) for k, c in enumerate(cfgs)]
    batch = Batch([p[0] for p in pairs])
    batch.set_blocks_per_sm(bps)
    batch.set_face_flux(True)
    assert batch.solute(25) == 25
    for (bm, solo) in pairs:
        solo.solute(25)
        _assert_same(bm, solo)
    assert pairs[0][0].counters()["n_regrids"] >= 2


@pytest.mark.skipif(not os.path.exists(learned.PARAMS_PATH), reason="no trained gate parameters")
@pytest.mark.parametrize("branch_free", [False, True])
def test_phase_kernels_match_single(branch_free):
    """blocks_per_sm 3: no persistent kernel, one launch per phase over every
    member; plain and gated members, regrids, a member reaching t_end early:
    every member ends bit-identical to its twin advanced alone."""
    cfgs = _cfgs() + [P.riemann4(base=32, lvl_amr=2, t_end=0.004)]
    pairs = [_pair(c, gate=(k % 2 == 1)) for k, c in enumerate(cfgs)]
    batch = Batch([p[0] for p in pairs])
    batch.set_blocks_per_sm(3)
    batch.set_face_flux(branch_free)
    assert batch.solute(25) == 25
    for (bm, solo) in pairs:
        solo.solute(25)
        _assert_same(bm, solo)
    assert pairs[0][0].counters()["n_regrids"] >= 2


def test_phase_kernels_advance_matches_single_steps():
    cfgs = _cfgs(no_regrid=True)
    pairs = [_pair(c) for c in cfgs]
    batch = Batch([p[0] for p in pairs])
    batch.set_blocks_per_sm(3)
    batch.advance(6)
    batch.sync()
    for (bm, solo) in pairs:
        solo.solute(6)
        _assert_same(bm, solo)
