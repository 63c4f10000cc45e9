"""Device regrid (AMR) vs the oracle: leaf set, tree and values after each
regrid bit-exact.  Both sides start from the same imported leaf set, so the
internal-node values (which gridmodify4 can copy back into leaves) start as
the same interpA means."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, cfg, pre_steps):
    o0 = oracle_mod.Oracle(cfg)
    o0.solute(pre_steps)
    keys, prim, _ = o0.leaves()
    s = o0.scalars()
    o = oracle_mod.Oracle(cfg, initial=False)
    o.set_leaves(keys, prim)
    o.set_scalars(s["lambda_x"], s["lambda_y"], s["tstep"], s["tt"], s["it"])
    g = Solver(cfg)
    g.upload(keys, prim)
    g.set_scalars(s["lambda_x"], s["lambda_y"], s["tstep"], s["tt"], s["it"])
    return o, g


def _same(g, o, what):
    kg, pg = g.leaves()
    ko, po, _ = o.leaves()
    assert len(kg) == len(ko) and np.array_equal(kg, ko), f"{what}: leaf sets differ ({len(kg)} vs {len(ko)})"
    assert np.array_equal(pg, po), f"{what}: values differ, max {np.max(np.abs(pg - po)):.3e}"


@pytest.mark.parametrize("pre", [1, 12])
def test_single_regrid_vortex(oracle_mod, pre):
    cfg = P.vortex()
    o, g = _pair(oracle_mod, cfg, pre)
    o.amr()                 # AMR + boundary refill
    g.amr()
    g.body_boundary(1)
    _same(g, o, "after regrid")
    assert np.array_equal(g.neighbors(), o.neighbors())


def test_vortex_steps_through_regrids(oracle_mod):
    cfg = P.vortex()
    o, g = _pair(oracle_mod, cfg, 12)
    for k in range(31):     # regrids at it = 21, 31, 41
        o.solute_step()
        g.solute_step()
        _same(g, o, f"step {k}")
    assert g.counters()["n_regrids"] == 3


def test_riemann4_regrids_with_nonleaf_refine(oracle_mod):
    """At 64^2 / 3 levels gridmodify4 re-refines non-leaf cells
    (src/mesh.F90:389-392); the new leaves copy the stale internal value."""
    cfg = P.riemann4(base=64, lvl_amr=3)
    o, g = _pair(oracle_mod, cfg, 20)
    for k in range(61):
        o.solute_step()
        g.solute_step()
        _same(g, o, f"step {k}")
    assert g.counters()["n_gm4_nonleaf"] == o.counters()["gm4_nonleaf"]


def test_double_mach_regrids(oracle_mod):
    cfg = P.double_mach(base_y=16, lvl_amr=2)
    o, g = _pair(oracle_mod, cfg, 5)
    for k in range(21):
        o.solute_step()
        g.solute_step()
        _same(g, o, f"step {k}")


def _l1(a, b):
    return float(np.mean(np.abs(a - b)))


def test_full_run_vortex_200_steps(oracle_mod):
    """Configuration 1: base 32^2, 2 levels, regrid every 10 steps, CFL 0.5,
    200 RK3 steps from the initial condition (host mesh + IC on both sides)."""
    cfg = P.vortex()
    o = oracle_mod.Oracle(cfg)
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    ko, po, _ = o.leaves()
    kg, pg = g.leaves()
    assert np.array_equal(ko, kg) and np.array_equal(po, pg), "initial states differ"
    assert o.solute(200) == 200
    assert g.solute(200) == 200
    kg, pg = g.leaves()
    ko, po, _ = o.leaves()
    assert np.array_equal(kg, ko)
    assert _l1(pg[:, 0], po[:, 0]) <= 1e-10
    assert np.array_equal(pg, po)
    assert g.counters()["n_regrids"] == o.counters()["regrids"] == 20
    so, sg = o.scalars(), g.scalars()
    assert sg["tt"] == so["tt"]


def test_full_run_riemann4_reduced(oracle_mod):
    """Four-quadrant problem, base 32^2, 2 levels, to t = 0.3."""
    cfg = P.riemann4(base=32, lvl_amr=2, t_end=0.3)
    o = oracle_mod.Oracle(cfg)
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    n1 = o.solute(10 ** 6)
    n2 = g.solute(10 ** 6)
    assert n1 == n2
    kg, pg = g.leaves()
    ko, po, _ = o.leaves()
    assert np.array_equal(kg, ko)
    assert _l1(pg[:, 0], po[:, 0]) <= 1e-10
    assert g.scalars()["tt"] == o.scalars()["tt"] == 0.3
