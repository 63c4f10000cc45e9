"""Whole AMR runs from a block-refined initial mesh (creat_mesh's
Block_refine): the GPU path (host generator + upload + device regrids)
against the oracle, bit for bit."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200.solver import Solver
from test_block_mesh_cpu import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,steps", [("vortex_box_l2", 40), ("riemann4_l4", 25), ("double_mach_wall_l3", 20)])
def test_block_mesh_run_matches_oracle(oracle_mod, name, steps):
    cfg = cases()[name]()
    o = oracle_mod.Oracle(cfg, threads=4)
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    ko0, po0, _ = o.leaves()
    kg0, pg0 = g.leaves()
    assert np.array_equal(kg0, ko0) and np.array_equal(pg0, po0)
    assert o.solute(steps) == steps
    assert g.solute(steps) == steps
    ko, po, _ = o.leaves()
    kg, pg = g.leaves()
    assert g.counters()["n_regrids"] == o.counters()["regrids"] >= 2
    assert np.array_equal(kg, ko) and np.array_equal(pg, po)
    o.close()
    g.close()
