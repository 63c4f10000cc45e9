"""CPU checks of the gate's reference math (no GPU): the oracle's analytic
gradient against finite differences, and the BF16 rounding helper."""
import numpy as np
import pytest

import mlp_ref
from fdm_cell_based_amr_cartesian_b200.learned import N_PARAMS, init_params


def test_bf16_rounding_is_round_to_nearest_even():
    assert mlp_ref.bf16(np.float32(1.0)) == 1.0
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert mlp_ref.bf16(np.float32(1.0 + 2.0 ** -8)) == 1.0
    assert mlp_ref.bf16(np.float32(1.0 + 3 * 2.0 ** -8)) == 1.0 + 2.0 ** -6


@pytest.mark.parametrize("neg_weight", [1.0, 4.0])
def test_oracle_gradient_matches_finite_differences(neg_weight):
    rng = np.random.default_rng(0)
    p = init_params(3).astype(np.float64)
    X = rng.uniform(-1, 1, (64, 8))
    Y = rng.uniform(0, 1, 64)
    _, g = mlp_ref.loss_and_grads(p, X, Y, rounding=False, neg_weight=neg_weight)
    assert g.shape == (N_PARAMS,)
    idx = rng.choice(N_PARAMS, 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = mlp_ref.loss_and_grads(pp, X, Y, rounding=False, neg_weight=neg_weight)
        lm, _ = mlp_ref.loss_and_grads(pm, X, Y, rounding=False, neg_weight=neg_weight)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_fine_density_paints_leaves_by_area():
    from fdm_cell_based_amr_cartesian_b200 import learned
    from fdm_cell_based_amr_cartesian_b200 import params as P
    from fdm_cell_based_amr_cartesian_b200.solver import root_keys
    cfg = P.vortex()
    p = cfg.params
    keys = root_keys(p.m, p.n)
    # refine root 0 once: children quadrants 0..3 at level 1
    kids = np.array([(0 << 34) | (q << 32) | 1 for q in range(4)], dtype=np.uint64)
    keys = np.concatenate([kids, keys[1:]])
    prim = np.zeros((len(keys), 4))
    prim[:, 0] = np.arange(len(keys)) + 1.0
    F = learned.fine_density(cfg, keys, prim)
    assert F.shape == (2 * p.n, 2 * p.m)
    assert F[0, 0] == 1.0 and F[0, 1] == 2.0 and F[1, 0] == 3.0 and F[1, 1] == 4.0
    assert F[0, 2] == F[1, 3] == 5.0          # root 1, covering 2 x 2 fine cells
    a = learned.density_errors(cfg, (keys, prim), (keys, prim))
    assert a == (0.0, 0.0)
