"""The one-logarithm fast path of the device K2P transform (rnj_device.cuh,
k2p_distance), restated in numpy with its table logarithm, checked against the
reference's two-logarithm arithmetic (KimuraDistance.cpp:339-349, as the oracle
computes it): whenever the fast path's rounding check accepts, its float must
be the reference's float.  This pins the error bound the check relies on; the
device path itself is compared with the oracle by the GPU parity tests.
"""
import numpy as np
import pytest

from oracle import oracle


def reference_k2p(P, Q, n):
    """KimuraDistance.cpp:339-349 in numpy (float ratios, double logs)."""
    ts = (P.astype(np.float64) / n).astype(np.float32)
    tv = (Q.astype(np.float64) / n).astype(np.float32)
    a = 1.0 - 2.0 * ts.astype(np.float64) - tv.astype(np.float64)
    b = 1.0 - 2.0 * tv.astype(np.float64)
    ok = (a.astype(np.float32) > 0) & (b.astype(np.float32) > 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        d = (-0.5 * np.log(a) - 0.25 * np.log(b)).astype(np.float32)
    return np.where(ok, d, np.float32(-1.0)), a, b, ok


def _log_table():
    """The table of rnj_logtab.h (its header, generated by gen_log_table.py)."""
    import os
    import re
    path = os.path.join(os.path.dirname(__file__), "..", "rapidnj_b200", "csrc", "rnj_logtab.h")
    text = open(path).read()
    rows = re.findall(r"\{(-?0x[0-9a-fp.+-]+), (0x[0-9a-fp.+-]+)\}", text)
    tab = np.array([[float.fromhex(a), float.fromhex(b)] for a, b in rows])
    hi = float.fromhex(re.search(r"kLn2Hi = (\S+);", text).group(1))
    lo = float.fromhex(re.search(r"kLn2Lo = (\S+);", text).group(1))
    return tab, hi, lo


def ln_table(x):
    """rnj_device.cuh ln_table in numpy (each fused multiply-add done as a multiply
    and an add: two roundings, within the same error bound)."""
    tab, hi, lo = _log_table()
    bits = x.view(np.int64)
    k = ((bits >> 52) & 0x7FF) - 1023
    j = (bits >> 45) & 127
    m = ((bits & 0x000FFFFFFFFFFFFF) | 0x3FF0000000000000).view(np.float64)
    F = (0x3FF0000000000000 | (j << 45)).view(np.float64)
    r = (m - F) * tab[j, 1]
    p = np.full_like(r, -1.0 / 6.0)
    for c in (0.2, -0.25, 1.0 / 3.0, -0.5, 1.0):
        p = p * r + c
    p = p * r
    dk = k.astype(np.float64)
    return dk * hi + ((dk * lo + tab[j, 0]) + p)


def fast_k2p(a, b):
    """The device fast path: (accepted, float)."""
    with np.errstate(divide="ignore", invalid="ignore"):
        x = (a * a) * b
        dd = -0.25 * ln_table(x)
        # fma(2^-47, dd, 2^-49): the product is exact, the sum rounded once
        eps = dd * 2.0 ** -47 + 2.0 ** -49
        lo = (dd - eps).astype(np.float32)
        hi = (dd + eps).astype(np.float32)
    return lo.view(np.int32) == hi.view(np.int32), lo


def test_ln_table_error_bound():
    # |ln_table(x) - ln x| < 2^-50.5 + 2^-53 |ln x| over x in [2^-138, 1]
    rng = np.random.default_rng(1)
    x = np.exp2(-rng.random(2_000_000) * 138.0)
    x = np.concatenate([x, 1.0 - rng.random(200_000) * 2.0 ** -7, [1.0, 0.5, 2.0 ** -138]])
    err = np.abs(ln_table(x) - np.log(x))
    bound = 2.0 ** -50.5 + 2.0 ** -53 * np.abs(np.log(x)) + 2.0 ** -52 * np.abs(np.log(x))
    assert (err <= bound).all()  # np.log itself within 1 ulp: the last term


@pytest.mark.parametrize("n", [7, 100, 997, 1000, 2048])
def test_fast_path_agrees_with_reference_exhaustive(n):
    P, Q = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = (P + Q <= n) & ((P + Q) > 0)
    P, Q = P[keep], Q[keep]
    ref, a, b, ok = reference_k2p(P, Q, float(n))
    acc, got = fast_k2p(a[ok], b[ok])
    r = ref[ok]
    assert np.array_equal(got[acc].view(np.int32), r[acc].view(np.int32))
    # the check rejects only a tiny fraction (then the two-log formula runs)
    assert (~acc).mean() < 1e-4


def test_fast_path_agrees_with_reference_random_large_n():
    rng = np.random.default_rng(0)
    n = rng.integers(1000, 2_000_000, size=2_000_000)
    P = (rng.random(n.size) * 0.4 * n).astype(np.int64)
    Q = (rng.random(n.size) * 0.45 * n).astype(np.int64)
    ref, a, b, ok = reference_k2p(P, Q, n.astype(np.float64))
    acc, got = fast_k2p(a[ok], b[ok])
    r = ref[ok]
    assert np.array_equal(got[acc].view(np.int32), r[acc].view(np.int32))
    assert (~acc).mean() < 1e-5


def test_fast_path_matches_oracle_transform():
    # The oracle's C transform (the reference's arithmetic, glibc log) on count
    # triples near the saturation boundary 1 - 2P/n - Q/n -> 0.
    rng = np.random.default_rng(1)
    n = rng.integers(50, 50_000, size=50_000).astype(np.uint32)
    Q = (rng.random(n.size) * 0.5 * n).astype(np.uint32)
    P = ((n - Q).astype(np.float64) / 2 * (0.9 + 0.1 * rng.random(n.size))).astype(np.uint32)
    k2p = oracle.lib().orc_k2p
    want = np.array([k2p(int(p), int(q), int(v)) for p, q, v in zip(P, Q, n)], dtype=np.float32)
    ref, a, b, ok = reference_k2p(P, Q, n.astype(np.float64))
    assert np.array_equal(want.view(np.int32), ref.view(np.int32))
    acc, got = fast_k2p(a[ok], b[ok])
    assert np.array_equal(got[acc].view(np.int32), ref[ok][acc].view(np.int32))


def neg_log_checked(c, arg):
    """rnj_device.cuh neg_log_checked in numpy: (accepted, float)."""
    dd = -c * ln_table(arg)
    eps = 2.0 ** -49 * (1.0 + 4.0 * dd)
    lo = (dd - eps).astype(np.float32)
    hi = (dd + eps).astype(np.float32)
    return lo.view(np.int32) == hi.view(np.int32), lo


@pytest.mark.parametrize("n", [1, 7, 100, 997, 10000, 65536])
@pytest.mark.parametrize("alpha", [4, 20])
def test_jc_checked_log_agrees_with_reference(n, alpha):
    # JCdistance.cpp:171-183: p = (float) total / valid, q = p / b in double,
    # (float)(-b log(1 - q)) unless q >= 1
    b = (alpha - 1.0) / alpha
    total = np.arange(n + 1)
    p = (total.astype(np.float32) / np.float32(n)).astype(np.float32)
    q = p.astype(np.float64) / b
    keep = (q < 1.0) & (q > 0.0)
    arg = 1.0 - q[keep]
    ref = (-b * np.log(arg)).astype(np.float32)
    acc, got = neg_log_checked(b, arg)
    assert np.array_equal(got[acc].view(np.int32), ref[acc].view(np.int32))
    if acc.size:  # n = 1 leaves no pair with 0 < q < 1
        assert (~acc).mean() < 1e-3


def test_protein_kimura_checked_log_agrees_with_reference():
    # KimuraDistance.cpp:322-338, p < 0.75: (float)(-log(1 - p - (float)(p*p) * 0.2))
    rng = np.random.default_rng(3)
    v = rng.integers(1, 200_000, size=3_000_000)
    m = (rng.random(v.size) * 0.75 * v).astype(np.int64)
    p = (m.astype(np.float32) / v.astype(np.float32)).astype(np.float32)
    keep = (p > 0) & (p.astype(np.float64) < 0.75)
    p = p[keep]
    sq = (p * p).astype(np.float32).astype(np.float64)
    arg = (1.0 - p.astype(np.float64)) - sq * 0.2
    ref = (-np.log(arg)).astype(np.float32)
    acc, got = neg_log_checked(1.0, arg)
    assert np.array_equal(got[acc].view(np.int32), ref[acc].view(np.int32))
    assert (~acc).mean() < 1e-5
