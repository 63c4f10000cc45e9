"""The reference's diagnostic files (src/output_ADT.F90) written on the host:
Fortran field formats, the output_Res records, and the density error norms
of output_error on known states."""
import numpy as np

from fdm_cell_based_amr_cartesian_b200 import output as O
from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import distance_refined_keys, initial_state, root_keys


def test_fortran_edit_descriptors():
    assert O.fortran_e(1.5, 14, 6) == "  0.150000E+01"
    assert O.fortran_e(-2.5e-7, 14, 6) == " -0.250000E-06"
    assert O.fortran_e(0.0, 14, 6) == "  0.000000E+00"
    assert O.fortran_e(1e-100, 14, 6) == "  0.100000E-99"
    assert O.fortran_e(1e-101, 14, 6) == "  0.100000-100"          # three-digit exponent drops the E
    assert O.fortran_e(0.9999996, 14, 6) == "  0.100000E+01"       # rounds into the next decade
    assert O.fortran_e(123.456, 16, 6) == "    0.123456E+03"
    assert O.fortran_e(-1.0, 12, 6) == "-.100000E+01"              # no room for the optional zero
    assert O.fortran_e(float("nan"), 14, 6).strip() == "NaN"
    assert O.fortran_i(42, 8) == "      42" and O.fortran_i(123456789, 8) == "********"


def test_res_lines():
    con, rec = O.res_lines(100, 4096, 1e-3, 0.25, [1, 2, 3, 4], [0.5, 0.25, 0.125, 0.0625])
    assert len(con) == 8 + 8 + 6 * 16 and len(rec) == 8 + 8 + 10 * 24
    assert con.startswith("     100    4096") and con.endswith("  0.625000E-01")
    assert rec.split()[2] == "0.1000000000E-02"


def test_error_norms_of_the_initial_vortex():
    cfg = P.vortex()
    keys = root_keys(cfg.m, cfg.n)
    e = O.error_norms(cfg, keys, initial_state(cfg, keys))
    assert e["n_res"] == 32 * 32 and e["n_patch"] == 0 and e["n_0"] == e["n_res"]
    assert e["L1_rho"] < 1e-15 and e["Loo_rho"] < 1e-15          # only the 1 + x - 1 rounding
    assert e["P1_rho"] == 0.0 and e["P2_rho"] == 0.0
    # a known perturbation on a refined mesh: +0.01 on every refined leaf
    keys = distance_refined_keys(cfg, [("x", 5.0)], [1.0, 0.5])
    prim = initial_state(cfg, keys)
    lvl = (keys & np.uint64(15)).astype(int)
    prim[lvl > 0, 0] += 0.01
    e = O.error_norms(cfg, keys, prim)
    assert abs(e["Poo_rho"] - 0.01) < 1e-12 and abs(e["P1_rho"] - 0.01) < 1e-12
    assert 0 < e["L1_rho"] < 0.01 and e["Loo_rho0"] < 1e-15
    lines = O.error_lines(200, e, first=True)
    assert lines[0].split()[0] == "nstep" and len(lines) == 3
    assert len(lines[1]) == 16 + 6 * 14 and len(lines[2]) == 16 + 3 * 14 + 8 + 3 * 14 + 8 + 3 * 14
