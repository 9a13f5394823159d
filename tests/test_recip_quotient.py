"""The quotients of the device transforms by the valid count (rnj_device.cuh,
recip_nr and ratio_f32): for integers 0 <= num <= den < 2^24, rounding
num * r to float, with r the Newton-Raphson reciprocal of den (a float seed
within four ulps of 1 / den, then two steps r + r (1 - den r) as fused
multiply-adds in double), gives the float quotient num / den that the reference computes with a
float division (JCdistance.cpp:171-176, KimuraDistance.cpp:324) and with a
double division rounded to float (KimuraDistance.cpp:341-342).

The reciprocal is restated exactly: each fused multiply-add is the exact
rational a * b + c rounded once to double (Python's float() of a Fraction is
correctly rounded).  numpy's float32 division and float64 products are IEEE,
correctly rounded.  Every den below 2^16 (the fused kernel's 16-bit counts) is
checked for its error bound, with every num for den <= 2000 and samples beyond;
random den up to 2^24 exercise the general statement."""
from fractions import Fraction

import numpy as np


def fma(a: float, b: float, c: float) -> float:
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def seed(n: int, ulps: int = 0) -> float:
    """A float reciprocal seed: the correctly rounded 1/n moved by `ulps` floats
    (the device seeds with the PTX fast reciprocal, within a couple of ulps;
    the proof needs a seed within 2^-21, four ulps)."""
    r = np.float32(1.0) / np.float32(n)
    step = np.inf if ulps > 0 else -np.inf
    for _ in range(abs(ulps)):
        r = np.nextafter(r, np.float32(step))
    return float(r)


def recip_nr(n: int, ulps: int = 0) -> float:
    r0 = seed(n, ulps)
    r1 = fma(r0, fma(-float(n), r0, 1.0), r0)
    return fma(r1, fma(-float(n), r1, 1.0), r1)


def quotient(num: np.ndarray, r: np.ndarray) -> np.ndarray:
    return (num.astype(np.float64) * r).astype(np.float32)


def check(num, den, r):
    got = quotient(num, r)
    want_f = num.astype(np.float32) / den.astype(np.float32)
    want_d = (num.astype(np.float64) / den.astype(np.float64)).astype(np.float32)
    assert np.array_equal(got.view(np.uint32), want_f.view(np.uint32))
    assert np.array_equal(got.view(np.uint32), want_d.view(np.uint32))


def test_reciprocal_error_bound_for_16_bit_counts():
    dens = np.arange(1, 1 << 16)
    r = np.array([recip_nr(int(d)) for d in dens])
    # |r - 1/n| <= 2^-52.9 / n, checked exactly
    worst = max(abs(Fraction(float(x)) * int(d) - 1) for d, x in zip(dens[::97], r[::97]))
    assert worst < Fraction(1, 2 ** 52)
    rel = np.abs(r * dens - 1.0)
    assert rel.max() <= 2.0 ** -51


def test_reciprocal_error_bound_from_any_seed_within_four_ulps():
    rng = np.random.default_rng(5)
    dens = np.concatenate([np.arange(1, 300), rng.integers(300, 1 << 24, 400)])
    for d in dens:
        for u in (-4, -3, -2, -1, 1, 2, 3, 4):
            x = recip_nr(int(d), u)
            assert abs(Fraction(x) * int(d) - 1) < Fraction(1, 2 ** 52)


def test_quotients_exhaustive_small_and_sampled_16_bit():
    for lo in range(1, 2001, 250):
        den = np.arange(lo, min(lo + 250, 2001), dtype=np.int64)
        num = np.concatenate([np.arange(d + 1) for d in den])
        dd = np.concatenate([np.full(d + 1, d) for d in den])
        r = np.array([recip_nr(int(d)) for d in den])
        rr = np.concatenate([np.full(d + 1, x) for d, x in zip(den, r)])
        check(num, dd, rr)
    rng = np.random.default_rng(3)
    den = rng.integers(2001, 1 << 16, 200_000)
    r_all = {int(d): recip_nr(int(d)) for d in np.unique(den)}
    r = np.array([r_all[int(d)] for d in den])
    num = np.minimum((rng.random(den.size) * (den + 1)).astype(np.int64), den)
    check(num, den, r)
    for edge in (np.zeros_like(den), np.ones_like(den), den - 1, den):
        check(edge, den, r)


def test_quotients_random_up_to_2_24():
    rng = np.random.default_rng(11)
    den = rng.integers(1 << 16, 1 << 24, 3000)
    r = np.array([recip_nr(int(d)) for d in den])
    for _ in range(20):
        num = np.minimum((rng.random(den.size) * (den + 1)).astype(np.int64), den)
        check(num, den, r)


def round_to_float_bits(y: np.ndarray) -> np.ndarray:
    """rnj_device.cuh round_to_float_bits: Veltkamp splitting with C = 2^29 + 1
    (two roundings per operation, as the device's explicitly rounded ops)."""
    g = y * 536870913.0
    return g - (g - y)


def check_k2p16(num, den, r):
    """k2p_decide16's ts: the 24-bit rounding of fl(num * r) in double equals the
    double of the float quotient the reference computes."""
    y = num.astype(np.float64) * r
    got = round_to_float_bits(y)
    want = (num.astype(np.float32) / den.astype(np.float32)).astype(np.float64)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_veltkamp_rounding_of_16_bit_quotients():
    for lo in range(1, 2001, 250):
        den = np.arange(lo, min(lo + 250, 2001), dtype=np.int64)
        num = np.concatenate([np.arange(d + 1) for d in den])
        dd = np.concatenate([np.full(d + 1, d) for d in den])
        r = np.array([recip_nr(int(d)) for d in den])
        check_k2p16(num, dd, np.concatenate([np.full(d + 1, x) for d, x in zip(den, r)]))
    rng = np.random.default_rng(5)
    den = rng.integers(2001, 1 << 16, 300_000)
    r_all = {int(d): recip_nr(int(d)) for d in np.unique(den)}
    r = np.array([r_all[int(d)] for d in den])
    for _ in range(3):
        num = np.minimum((rng.random(den.size) * (den + 1)).astype(np.int64), den)
        check_k2p16(num, den, r)
    for edge in (np.zeros_like(den), np.ones_like(den), den - 1, den):
        check_k2p16(edge, den, r)


# --- the fused epilogue's float quotients (rnj_device.cuh: recip16, quotient16)
#
# y = fma(r0, fma(-d, r0, 1), r0) from a seed r0 within four ulps of 1 / d, then
# q0 = fl(num y), r = fma(-q0, d, num), q = fma(r, y, q0), all in float.  The
# fused multiply-adds are restated exactly (Fraction) where rounding matters:
# the Newton-Raphson step and the final correction.

def f32(x) -> float:
    return float(np.float32(x))


def fma32(a: float, b: float, c: float) -> float:
    """fma in float: the exact a * b + c rounded once to float (through a
    correctly rounded double, exact here unless the sum needs more than 53 bits;
    the rational is then rounded to float directly)."""
    exact = Fraction(a) * Fraction(b) + Fraction(c)
    d = float(exact)
    if Fraction(d) == exact:
        return f32(d)
    lo = np.float32(d)
    # round the rational to the nearest float, ties to even
    cands = [np.nextafter(lo, np.float32(-np.inf)), lo, np.nextafter(lo, np.float32(np.inf))]
    best = min(cands, key=lambda c: (abs(Fraction(float(c)) - exact),
                                     int(np.array(c, np.float32).view(np.uint32)) & 1))
    return float(best)


def quotient16(num: int, d: int, ulps: int) -> float:
    r0 = seed(d, ulps)
    y = fma32(r0, fma32(-float(d), r0, 1.0), r0)
    q0 = f32(np.float32(num) * np.float32(y))
    return fma32(fma32(-q0, float(d), float(num)), y, q0)


def test_float_quotient_of_16_bit_counts():
    """Sampled restatement; the device checks every 0 <= num <= d < 2^16
    itself (tests/test_gpu_quotient16.py)."""
    rng = np.random.default_rng(16)
    dens = np.concatenate([np.arange(1, 80), rng.integers(80, 1 << 16, 60), [65535, 65534, 49152]])
    for d in dens:
        d = int(d)
        nums = set(range(min(d, 40) + 1)) | {d, d - 1, d // 2, d // 3} | set(
            int(x) for x in rng.integers(0, d + 1, 25))
        for ulps in (-4, -1, 0, 1, 4):
            for num in nums:
                if num < 0:
                    continue
                want = f32(Fraction(num, d))
                assert quotient16(num, d, ulps) == want, (num, d, ulps)
