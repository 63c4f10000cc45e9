"""The method of the device's exact left-to-right sum (csrc/ordered_sum.cuh),
restated in numpy and checked against the plain sequential sum on the CPU.

While the running sum s stays in one binade [2^E, 2^(E+1)), every partial
sum is a multiple of u = 2^(E-52) and RN(s + x) = s + r*u with r = x/u
rounded to the nearest integer, unless x/u is a halfway case; so a run of
such additions is an integer prefix sum.  The run stops before the first
addition that would reach the next binade (integer total 2^53) or is a
halfway case, NaN, infinite or negative; that one addition is made as
s = s + x.  This restatement takes the runs in chunks as the block does
(any chunking gives the same result) and is compared bit for bit with
(...((0 + x0) + x1) + ...)."""
import math

import numpy as np
import pytest

TOP = 1 << 53


def _seq(x):
    s = 0.0
    for v in x.tolist():
        s += v
    return s


def _runs(x, chunk=4096):
    s, start, n = 0.0, 0, len(x)
    while start < n:
        end = min(start + chunk, n)
        if s == 0.0:
            nz = np.nonzero(x[start:end] != 0.0)[0]   # NaN counts as not zero
            if len(nz) == 0:
                start = end
                continue
            f = start + int(nz[0])
            s, start = s + float(x[f]), f + 1
            continue
        m, e = math.frexp(s)                   # s = m * 2^e, m in [0.5, 1)
        if not math.isfinite(s) or s < 0.0 or e - 1 < -970:
            s, start = s + float(x[start]), start + 1
            continue
        u = math.ldexp(1.0, e - 1 - 52)
        M = int(s / u)                         # exact: s is a multiple of u below 2^53 u
        t = x[start:end] / u                   # exact: a power-of-two scaling
        with np.errstate(invalid="ignore"):
            ok = (x[start:end] >= 0.0) & (t < 2.0 ** 52)
        tt = np.where(ok, t, 0.0)
        r = np.rint(tt)                        # nearest, ties to even
        half = np.abs(tt - np.floor(tt) - 0.5) == 0.0
        ok &= ~half
        bad = np.nonzero(~ok)[0]
        stop = int(bad[0]) if len(bad) else end - start
        pref = M + np.cumsum(r[:stop].astype(np.int64))
        over = np.nonzero(pref >= TOP)[0]
        if len(over):
            stop = int(over[0])
        R = int(pref[stop - 1]) - M if stop > 0 else 0
        s = float(M + R) * u
        a = start + stop
        if a < end:
            s, start = s + float(x[a]), a + 1
        else:
            start = end
    return s


def _cases():
    rng = np.random.default_rng(11)
    return {
        "squares": rng.standard_normal(20_000) ** 2,
        "squares_wide": (rng.standard_normal(20_000) * 10.0 ** rng.uniform(-8, 8, 20_000)) ** 2,
        "ties": np.array([1.0] + [2.0 ** -53] * 3000 + [3 * 2.0 ** -53] * 100 + [2.0 ** -52] * 50),
        "halfway": np.array([(k + 0.5) * 2.0 ** -52 for k in range(5000)]),
        "zeros_first": np.concatenate([np.zeros(5000), rng.random(4000) * 1e-3, np.zeros(3000)]),
        "powers_of_two": np.array([0.5, 0.25, 0.25, 1.0, 1.0, 2.0, 4.0, 8.0 - 2.0 ** -49] + [2.0 ** -50] * 4000),
        "range": 10.0 ** rng.uniform(-300, 300, 6000),
        "subnormal": np.array([5e-324] * 1500 + [1e-310] * 500 + [1e-300] * 100),
        "nan": np.array([1.0] * 1500 + [np.nan] + [1.0] * 10),
        "small_ints": rng.integers(0, 8, 6000) * 2.0 ** -53,
    }


@pytest.mark.parametrize("name", list(_cases()))
@pytest.mark.parametrize("chunk", [7, 1024, 4096])
def test_binade_runs_equal_sequential_sum(name, chunk):
    x = _cases()[name]
    got, want = _runs(x, chunk), _seq(x)
    assert (math.isnan(got) and math.isnan(want)) or np.float64(got).tobytes() == np.float64(want).tobytes(), \
        (name, got, want)
