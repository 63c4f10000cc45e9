"""Checkpoint/restart through the C-ABI: a run written to a file at step 250
and restored into a new handle continues bit for bit with the uninterrupted
run, through regrids that refine non-leaves (steps 261, 321, 351 of the
64^2, 3-level four-quadrant problem), because the internal-node values
travel with the leaves."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import FdmError, Solver

pytestmark = pytest.mark.gpu


def test_restart_continues_bit_for_bit(tmp_path):
    cfg = P.riemann4(base=64, lvl_amr=3)
    a = Solver(cfg)
    a.creat_mesh_and_initial()
    assert a.solute(250) == 250
    path = str(tmp_path / "run.npz")
    a.save_checkpoint(path)
    b = Solver(cfg)
    b.load_checkpoint(path)
    ka, va = a.internal_nodes()
    kb, vb = b.internal_nodes()
    assert len(ka) > 0 and np.array_equal(ka, kb) and np.array_equal(va, vb)
    assert a.scalars() == b.scalars()
    nl0 = a.counters()["n_gm4_nonleaf"]
    assert a.solute(110) == 110 and b.solute(110) == 110
    assert a.counters()["n_gm4_nonleaf"] - nl0 == b.counters()["n_gm4_nonleaf"] >= 2
    ka, pa = a.leaves()
    kb, pb = b.leaves()
    assert np.array_equal(ka, kb) and np.array_equal(pa, pb)
    assert a.scalars() == b.scalars()
    # a checkpoint only restores into the parameters it was written with
    c = Solver(P.riemann4(base=64, lvl_amr=2))
    with pytest.raises(ValueError):
        c.load_checkpoint(path)
    # internal values of another leaf set are refused
    c.creat_mesh_and_initial()
    with pytest.raises(FdmError):
        c.set_internal(kb[:3], np.zeros((3, 4)))
    for g in (a, b, c):
        g.close()
