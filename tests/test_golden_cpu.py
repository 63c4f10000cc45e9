"""The oracle against its committed golden final states (no GPU): whole runs
with regrids from the initial condition, compared by SHA-256 of the leaf
keys and primitive states (tests/golden/oracle_runs.json, written by
tests/golden/make_golden.py)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402

GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_runs.json")))


@pytest.mark.parametrize("name", ["vortex_200_steps", "riemann4_32_l2_to_t0.3", "double_mach_64x16_l2_to_t0.2"])
def test_oracle_reproduces_golden_run(oracle_mod, name):
    make, steps = make_golden.cases()[name]
    rec = make_golden.run(make, steps)
    want = GOLDEN[name]
    for k in ("steps", "n_leaves", "regrids", "gm4_nonleaf", "sha256_keys", "sha256_prim"):
        assert rec[k] == want[k], (k, rec[k], want[k])
