"""The command-line run (python -m fdm_cell_based_amr_cartesian_b200): a short
vortex run with regrids prints one JSON line with its steps and counters."""
import json

import pytest

from fdm_cell_based_amr_cartesian_b200.__main__ import main

pytestmark = pytest.mark.gpu


def test_cli_short_vortex_run(capsys):
    assert main(["--case", "vortex", "--base", "32", "--lvl-amr", "2", "--steps", "25"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["steps"] == 25
    assert out["counters"]["n_regrids"] >= 2
    assert out["tt"] > 0


def test_cli_writes_the_reference_diagnostics(tmp_path, capsys):
    d = str(tmp_path / "Output")
    assert main(["--case", "vortex", "--base", "32", "--lvl-amr", "2", "--t-end", "0.5", "--output", d]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["tt"] == 0.5
    res = open(f"{d}/Residual.dat").read().splitlines()
    assert len(res) >= 1 and all(len(r) == 16 + 10 * 24 for r in res)
    err = open(f"{d}/accuracy_error.dat").read().splitlines()
    assert err[0].split()[0] == "nstep" and len(err) == 3
    # the norms are taken against the vortex at its initial position, which
    # the flow has moved by (0.5, 0.5) at t = 0.5
    l1 = float(err[1][16:30])
    assert 0.0 < l1 < 1.0


def test_cli_ensemble_run(capsys):
    assert main(["--case", "ensemble", "--members", "4", "--steps", "20"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["members"] == 4 and out["steps"] == 20
    assert out["regrids"] >= 4 * 2 and 0 < out["tt_min"] <= out["tt_max"]


def test_cli_strips_run_matches_the_whole_run(capsys):
    args = ["--case", "riemann4", "--base", "32", "--lvl-amr", "2", "--steps", "25"]
    assert main(args) == 0
    whole = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert main(args + ["--strips", "3"]) == 0
    out = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert out["strips"] == 3 and out["steps"] == 25
    assert out["tt"] == whole["tt"] and out["regrids"] == whole["counters"]["n_regrids"] == 3
    assert out["leaves"] == whole["counters"]["n_leaves"]


def test_cli_field_dumps(tmp_path, capsys):
    d = str(tmp_path / "Output")
    assert main(["--case", "vortex", "--base", "32", "--lvl-amr", "2", "--steps", "30", "--output", d,
                 "--dump-every", "10"]) == 0
    import os

    import numpy as np
    names = sorted(f for f in os.listdir(d) if f.startswith("field_"))
    assert names == ["field_00000010.npz", "field_00000020.npz", "field_00000030.npz"]
    z = np.load(os.path.join(d, names[-1]))
    assert z["keys"].dtype == np.uint64 and z["prim"].shape == (len(z["keys"]), 4)
    assert np.isfinite(z["prim"]).all()
