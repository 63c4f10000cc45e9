"""The WLS sector test without atan2 (get_direction in csrc/build.cu),
restated in Python and checked against the reference's formula
(src/XuanGua.F90:33-43: angle = (atan2(dy, dx) + 1e-10) * 180 / pi, sector
mod(floor((angle + 22.5) / 45 + 8), 8) + 1).

Away from the sector edges the sector follows from comparing abs(dy) with
tan(22.5) abs(dx) and tan(67.5) abs(dx); a relative margin of 1e-9 on the
tangent keeps the decided points more than 3.5e-10 rad from an edge, more
than the 1e-10 rad bias plus every rounding of the formula, and the points
inside the margin take the formula itself."""
import math
import random

import numpy as np

BIAS = float(np.float32(1e-10))   # the reference's REAL(4) literal
PI = 3.1415926535897932
T1, T2 = 0.41421356237309503, 2.414213562373095
LO, HI = 1.0 - 1e-9, 1.0 + 1e-9


def formula(dx, dy):
    angle = (math.atan2(dy, dx) + BIAS) * 180.0 / PI
    f = math.floor((angle + 22.5) / 45.0 + 8)
    return ((f % 8) + 8) % 8 + 1


def fast(dx, dy):
    a, b = abs(dx), abs(dy)
    if b < a * (T1 * LO):
        return 1 if dx > 0.0 else 5
    if b > a * (T2 * HI):
        return 3 if dy > 0.0 else 7
    if a * (T1 * HI) < b < a * (T2 * LO):
        return (2 if dy > 0.0 else 8) if dx > 0.0 else (4 if dy > 0.0 else 6)
    return formula(dx, dy)


def test_dyadic_cell_offsets():
    """Offsets between cell centres: dyadic numbers at levels 0..6."""
    rng = random.Random(1)
    for _ in range(100_000):
        h = 2.0 ** -rng.randint(0, 6)
        dx = (rng.randint(-40, 40) + rng.choice((0.0, 0.5, 0.25, 0.125))) * h
        dy = (rng.randint(-40, 40) + rng.choice((0.0, 0.5, 0.25, 0.125))) * h
        assert fast(dx, dy) == formula(dx, dy), (dx, dy)


def test_points_next_to_every_edge():
    for k in range(8):
        edge = (45 * k - 22.5) * math.pi / 180
        for eps in (1e-6, 1e-9, 3e-10, 1e-10, 1e-11, 0.0, -1e-11, -1e-10, -3e-10, -1e-9, -1e-6):
            for r in (1e-3, 1.0, 7.0):
                dx, dy = r * math.cos(edge + eps), r * math.sin(edge + eps)
                assert fast(dx, dy) == formula(dx, dy), (k, eps, r)


def test_axes_and_origin():
    for dx, dy in ((1.0, 0.0), (-1.0, 0.0), (0.0, 1.0), (0.0, -1.0), (0.0, 0.0), (1.0, 1.0), (-1.0, -1.0)):
        assert fast(dx, dy) == formula(dx, dy), (dx, dy)
