"""The warp-parallel left-to-right sum that forms Srot and Sdiv
(src/solution.F90:430-457) against the plain sequential sum, bit for bit,
on inputs chosen to hit every branch: halfway cases, binade crossings at
exact powers of two, long runs of zeros, subnormal and huge addends, a NaN,
and large random inputs."""
import numpy as np
import pytest

from fdm_cell_based_amr_cartesian_b200.solver import _dp, load_library

pytestmark = pytest.mark.gpu


def _seq(x):
    s = 0.0
    for v in x.tolist():
        s += v
    return s


def _device(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    out = np.zeros(2)
    assert load_library().fdm_debug_ordered_sum(_dp(a), _dp(b), len(a), _dp(out)) == 0
    return out


def _same(x, y):
    return (np.isnan(x) and np.isnan(y)) or x.tobytes() == y.tobytes()


def _cases():
    rng = np.random.default_rng(7)
    c = {
        "squares": rng.standard_normal(300_000) ** 2,
        "squares_wide": (rng.standard_normal(200_000) * 10.0 ** rng.uniform(-8, 8, 200_000)) ** 2,
        "ties": np.array([1.0] + [2.0 ** -53] * 3000 + [3 * 2.0 ** -53] * 100 + [2.0 ** -52] * 50),
        "halfway": np.array([(k + 0.5) * 2.0 ** -52 for k in range(5000)]),
        "zeros_first": np.concatenate([np.zeros(5000), rng.random(4000) * 1e-3, np.zeros(3000)]),
        "powers_of_two": np.array([0.5, 0.25, 0.25, 1.0, 1.0, 2.0, 4.0, 8.0 - 2.0 ** -49] + [2.0 ** -50] * 4000),
        "range": 10.0 ** rng.uniform(-300, 300, 6000),
        "subnormal": np.array([5e-324] * 1500 + [1e-310] * 500 + [1e-300] * 100),
        "nan": np.array([1.0] * 1500 + [np.nan] + [1.0] * 10),
        "small_ints": rng.integers(0, 8, 6000) * 2.0 ** -53,
        "one": np.array([3.0]),
        "empty": np.zeros(0),
    }
    return c


@pytest.mark.parametrize("name", list(_cases()))
def test_ordered_sum_bit_exact(name):
    x = _cases()[name]
    y = x[::-1].copy()   # the second sum sees another order of the same values
    got = _device(x, y)
    assert _same(got[0], np.float64(_seq(x))), (name, got[0], _seq(x))
    assert _same(got[1], np.float64(_seq(y))), (name, got[1], _seq(y))
