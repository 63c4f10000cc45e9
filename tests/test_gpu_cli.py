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
