"""Failure detection without a GPU fault: the batched kernel's grid barrier,
made to wait for a block that never arrives, gives up at its iteration limit
and the host reads FDM_ERR_TIMEOUT; the context stays usable (a step after
it still matches the oracle)."""
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
