"""The exact lap skip of the corrector's contour walks (skip_laps in
gragles2d_b200/csrc/gg_corrector.cuh), restated with Python floats (IEEE
binary64, round to nearest even, as the device's FP64 adds) and checked
against the step-by-step walk it replaces: the same final index, iteration
count and bit-identical distance on walks of millions of steps over tiny
contours, the case of a nearly vanished grain whose perimeter is far below
the sector radius."""
import math
import random
import sys

import pytest

DBL_MIN = sys.float_info.min


def skip_laps(d, limit, seg, p, step, n, max_laps):
    if not (d >= DBL_MIN) or not (d < limit) or n <= 0 or max_laps < 1:
        return d, 0
    _, e = math.frexp(d)
    u = math.ldexp(1.0, e - 53)
    top = math.ldexp(1.0, e)
    q = 0.0
    k = p
    for _ in range(n):
        r = seg[k] / u
        if r - math.floor(r) == 0.5:
            return d, 0
        q += float(round(r)) * u  # round() is round-half-even, as rint
        k = (k + step) % n
    if not q > 0:
        return d, 0
    mm = math.floor((min(limit, top) - d) / q) - 2
    mm = min(mm, max_laps)
    if mm < 1:
        return d, 0
    return d + mm * q, mm


def walk_plain(d, limit, seg, p, step, strict=True):
    n = len(seg)
    it = 0
    while (d < limit) if strict else (d <= limit):
        d += seg[p]
        p = (p + step) % n
        it += 1
    return d, p, it


def walk_skipping(d, limit, seg, p, step, guard, strict=True):
    n = len(seg)
    it = 0
    while (d < limit) if strict else (d <= limit):
        if it >= 64 and it % 64 == 0:
            d, m = skip_laps(d, limit, seg, p, step, n, (guard - it) // n - 2)
            it += m * n
        d += seg[p]
        p = (p + step) % n
        it += 1
        assert it <= guard
    return d, p, it


@pytest.mark.parametrize("seed", range(12))
def test_skipping_walk_is_bit_identical(seed):
    rng = random.Random(seed)
    n = rng.choice([3, 4, 5, 7])
    scale = 10.0 ** rng.uniform(-11, -8)
    seg = [scale * rng.uniform(0.2, 1.5) for _ in range(n)]
    limit = rng.uniform(2.0, 4.0) / 3600.0
    d0 = scale * rng.uniform(0.0, 1.0)
    p0 = rng.randrange(n)
    step = rng.choice([1, -1])
    strict = rng.random() < 0.5
    ref = walk_plain(d0, limit, seg, p0, step, strict)
    assert ref[2] > 10_000  # a long walk
    guard = (math.ceil(limit / sum(seg)) + 2) * (n + 2) + 8
    got = walk_skipping(d0, limit, seg, p0, step, guard, strict)
    assert got[1:] == ref[1:]
    assert got[0] == ref[0] and got[0].hex() == ref[0].hex()


def test_ordinary_walks_do_not_skip():
    seg = [0.7 / 3600] * 40
    d, m = skip_laps(0.1 / 3600, 3.0 / 3600, seg, 0, 1, 40, 100)
    assert m == 0 and d == 0.1 / 3600
