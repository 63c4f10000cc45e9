"""The benchmark's statically refined mesh (no GPU): 2:1 balance across the
whole root grid, ghost cells included, and a finite, positive state after
a few RK3 steps of the oracle."""
import numpy as np

from fdm_cell_based_amr_cartesian_b200 import learned
from fdm_cell_based_amr_cartesian_b200 import params as P
from fdm_cell_based_amr_cartesian_b200.solver import distance_refined_keys, initial_state

BAND = [0.2, 0.15, 0.1, 0.05]


def _small():
    cfg = P.riemann4(base=32, lvl_amr=4, pstep_adapt=1000)
    keys = distance_refined_keys(cfg, [("x", 0.5), ("y", 0.5)], BAND)
    return cfg, keys


def test_distance_refined_mesh_is_balanced():
    cfg, keys = _small()
    lvl = (keys & np.uint64(15)).astype(np.float64)
    vals = np.zeros((len(keys), 4))
    vals[:, 0] = lvl
    F = learned.fine_density(cfg, keys, vals)
    assert F.shape == (cfg.n << 4, cfg.m << 4)
    assert F.max() == 4
    # face neighbours of every fine cell differ by at most one level
    assert np.abs(np.diff(F, axis=0)).max() <= 1
    assert np.abs(np.diff(F, axis=1)).max() <= 1
    # the mesh reaches the boundary rows: the ghost rows are refined too
    assert F[:3 << 4].max() >= 3


def test_distance_refined_mesh_stays_finite(oracle_mod):
    cfg, keys = _small()
    prim = initial_state(cfg, keys)
    o = oracle_mod.Oracle(cfg, initial=False)
    o.set_leaves(keys, prim)
    for _ in range(3):
        o.step_control()
        o.time_advance_rk()
    _, p, _ = o.leaves()
    assert np.isfinite(p).all()
    assert p[:, 0].min() > 0.1 and p[:, 3].min() > 0.02


def test_bench_golden_check(tmp_path, monkeypatch):
    """bench.matches_golden: True on the recorded digest, False on one flipped
    bit or another step count, None for an unrecorded run."""
    import hashlib
    import json
    import bench
    rng = np.random.default_rng(3)
    keys = np.sort(rng.integers(0, 1 << 40, 50, dtype=np.uint64))
    prim = rng.random((50, 4))
    rec = {"steps": 7, "regrids": 1,
           "sha256_keys": hashlib.sha256(keys.tobytes()).hexdigest(),
           "sha256_prim": hashlib.sha256(prim.tobytes()).hexdigest()}
    path = tmp_path / "runs.json"
    path.write_text(json.dumps({"case": rec}))
    monkeypatch.setattr(bench, "GOLDEN_RUNS", str(path))
    assert bench.matches_golden("case", keys, prim, 7, 1) is True
    bad = prim.copy()
    bad.view(np.uint64)[3, 2] ^= np.uint64(1)
    assert bench.matches_golden("case", keys, bad, 7, 1) is False
    assert bench.matches_golden("case", keys, prim, 8, 1) is False
    assert bench.matches_golden("other", keys, prim, 7, 1) is None
    # every full run names its configuration and golden record
    for name, (make, desc, golden) in bench.FULL_RUNS.items():
        assert make().params.t_end > 0 and desc and golden


def test_bench_summary_tolerates_missing_legs():
    """The compact summary at the end of the bench line is built from
    whatever legs ran (a leg that failed or was skipped leaves no key)."""
    import bench
    line = {"ms_per_step": 1.5, "roofline": {"ms_per_launch": 0.39, "frac": 0.04},
            "roofline_fp64": {"frac": 0.2}, "learned": {"error": "x"}, "ensemble": None, "full_run": None,
            "strips": {"error": "y"}}
    s = bench.summary(line)
    assert s["plain_ms_per_step"] == 1.5 and s["face_pair_ms"] == 0.39
    assert "gated_ms_per_step" not in s and "cfg2_full_s" not in s
    line["learned"] = {"ms_per_step": 0.75, "l1_density_vs_plain": 5e-7,
                       "rule_vs_network": {"network": {"l1_density_vs_plain": 1e-7, "stage1_gated_fraction": 0.9},
                                           "jump_rule": {"l1_density_vs_plain": 2e-7,
                                                         "stage1_gated_fraction": 0.9}}}
    s = bench.summary(line)
    assert s["gated_speedup"] == 2.0 and s["net_vs_rule_l1"] == [1e-7, 2e-7]
