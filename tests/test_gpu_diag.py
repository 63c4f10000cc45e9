"""Device-side diagnostics: output_error's norms formed on the device
(fdm_output_error) against the host restatement of output_error
(output.error_norms, sequential sums in cell_NS order), and asynchronous
field dumps against the leaves read back synchronously."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200 import output as O
from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import Solver

pytestmark = pytest.mark.gpu

# the vortex density uses the device's exp/pow on one side and the C
# library's on the other: they may differ in the last bit, nothing else does
REL = 1e-13


def test_device_error_norms_match_host():
    cfg = P.vortex()
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    g.solute(35)                                   # three regrids: refined leaves
    keys, prim = g.leaves()
    host = O.error_norms(cfg, keys, prim)
    dev = g.output_error_device()
    for k in ("n_res", "n_0", "n_patch"):
        assert dev[k] == host[k], k
    assert host["n_patch"] > 0 and host["n_0"] > 0
    for k in ("L1_rho", "L2_rho", "Loo_rho", "P1_rho", "P2_rho", "Poo_rho", "L1_rho0", "L2_rho0", "Loo_rho0"):
        assert abs(dev[k] - host[k]) <= REL * abs(host[k]), (k, dev[k], host[k])
    # the file records agree to the printed digits
    assert O.error_lines(35, dev, True) == O.error_lines(35, host, True)
    g.close()


def test_field_dump_matches_leaves(tmp_path):
    cfg = P.riemann4(base=32, lvl_amr=2, t_end=0.3)
    g = Solver(cfg)
    g.creat_mesh_and_initial()
    dump = O.FieldDump(str(tmp_path))
    want = {}
    for chunk in (7, 9, 15):                       # a regrid falls between the dumps
        g.solute(chunk)
        want[g.scalars()["it"]] = g.leaves()
        dump.dump(g)
    g.solute(5)                                    # steps while the last dump is in flight
    dump.close()
    assert len(dump.written) == 3
    for it, (k, p) in want.items():
        z = np.load(tmp_path / f"field_{it:08d}.npz")
        assert np.array_equal(z["keys"], k) and np.array_equal(z["prim"], p), it
    g.close()
