"""The fused epilogue's quotients over their whole domains, on the device:
the float quotients by the valid count (rnj_device.cuh: recip16, quotient16)
for every 0 <= num <= n < 2^16 (2.1e9 pairs) against correctly rounded float
division and against the reference's double division rounded to float
(KimuraDistance.cpp:341-342, JCdistance.cpp:171-176); and JC's (double)p / b
(div_by_b, Markstein's correction from the correctly rounded 1 / b) for every
float p in [0, 1] and b = 3/4, 19/20 against the correctly rounded double
division (JCdistance.cpp:177)."""
import pytest

pytestmark = pytest.mark.gpu


def test_every_16_bit_quotient_is_correctly_rounded(ctx):
    assert ctx.check_quotient16() == 0
