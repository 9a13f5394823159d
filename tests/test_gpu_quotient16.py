"""The fused epilogue's float quotients by the valid count (rnj_device.cuh:
recip16, quotient16) over their whole domain, on the device: every
0 <= num <= n < 2^16 (2.1e9 pairs) against correctly rounded float division
and against the reference's double division rounded to float
(KimuraDistance.cpp:341-342, JCdistance.cpp:171-176)."""
import pytest

pytestmark = pytest.mark.gpu


def test_every_16_bit_quotient_is_correctly_rounded(ctx):
    assert ctx.check_quotient16() == 0
