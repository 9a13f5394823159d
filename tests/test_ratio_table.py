"""The reciprocal-table quotient of the device transforms (rnj_device.cuh,
ratio_f32): for integers 0 <= num <= den < 2^24, rounding num * rn to float,
with rn the double nearest to 1 / den, gives the float quotient num / den that
the reference computes with float division (JCdistance.cpp:171-176,
KimuraDistance.cpp:324) and with a double division rounded to float
(KimuraDistance.cpp:341-342).  numpy's float32 division and float64
arithmetic are IEEE, correctly rounded, so they restate both sides exactly.
Exhaustive for den <= 3000 and random beyond, up to the tensor-core path's
2^21 - 1 columns and the 2^24 bound of the proof."""
import numpy as np


def table_quotient(num, den):
    rn = 1.0 / den.astype(np.float64)
    return (num.astype(np.float64) * rn).astype(np.float32)


def float_quotient(num, den):
    return num.astype(np.float32) / den.astype(np.float32)


def double_quotient(num, den):
    return (num.astype(np.float64) / den.astype(np.float64)).astype(np.float32)


def check(num, den):
    t = table_quotient(num, den)
    assert np.array_equal(t.view(np.uint32), float_quotient(num, den).view(np.uint32))
    assert np.array_equal(t.view(np.uint32), double_quotient(num, den).view(np.uint32))


def test_exhaustive_small_denominators():
    for lo in range(1, 3001, 500):
        den = np.arange(lo, min(lo + 500, 3001), dtype=np.int64)
        num = np.concatenate([np.arange(d + 1) for d in den])
        dd = np.concatenate([np.full(d + 1, d) for d in den])
        check(num, dd)


def test_random_large_denominators():
    rng = np.random.default_rng(7)
    for hi in ((1 << 16), (1 << 21) - 1, (1 << 24) - 1):
        den = rng.integers(1, hi + 1, 2_000_000)
        num = (rng.random(den.size) * (den + 1)).astype(np.int64)
        num = np.minimum(num, den)
        check(num, den)
        # the edges: 0, 1, den - 1, den
        for k in (0, 1):
            check(np.full(den.size, k), den)
        check(den - 1, den)
        check(den, den)
