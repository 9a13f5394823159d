"""Writes rnj_logtab.h: the table of the transform's logarithm (rnj_device.cuh,
ln_table).  Tang's table-driven method (P. T. P. Tang, "Table-driven
implementation of the logarithm function in IEEE floating-point arithmetic", ACM
TOMS 16(4), 1990): for F_j = 1 + j/128, j = 0..127, the double nearest to
ln(F_j) and to 1/F_j.  Exact values come from Python's Fraction/Decimal
arithmetic, not from a library logarithm, so each entry is correctly rounded.

Usage: python rapidnj_b200/csrc/gen_log_table.py > rapidnj_b200/csrc/rnj_logtab.h
"""
import struct
from decimal import Decimal, getcontext
from fractions import Fraction

getcontext().prec = 80


def ln_decimal(x: Decimal) -> Decimal:
    """ln(x) for x in [1, 2): 2 atanh((x - 1) / (x + 1)) by its series."""
    y = (x - 1) / (x + 1)
    y2 = y * y
    term, s, k = y, Decimal(0), 1
    while True:
        t = term / k
        if abs(t) < Decimal(10) ** -75:
            break
        s += t
        term *= y2
        k += 2
    return 2 * s


def nearest_double(v: Decimal) -> float:
    """The double nearest to v (float() of a Fraction rounds correctly)."""
    return float(Fraction(v))


def main():
    rows = []
    for j in range(128):
        F = Decimal(128 + j) / Decimal(128)
        lnF = nearest_double(ln_decimal(F))
        inv = float(Fraction(128, 128 + j))
        rows.append((lnF, inv))
    # ln 2 = ln(2) split: hi with 42 significant bits (k * hi exact for |k| < 2^11)
    ln2 = 2 * ln_decimal(Decimal(2).sqrt())  # ln 2 = 2 ln sqrt 2, sqrt 2 in [1, 2)
    ln2_d = Fraction(ln2)
    hi = float(ln2_d)
    bits = struct.unpack("<Q", struct.pack("<d", hi))[0] & ~((1 << 11) - 1)
    hi = struct.unpack("<d", struct.pack("<Q", bits))[0]
    lo = float(ln2_d - Fraction(hi))
    print("// rnj_logtab.h -- generated by gen_log_table.py; do not edit.")
    print("// Tang's table for ln(x) (ACM TOMS 16(4), 1990): {ln(1 + j/128), 1/(1 + j/128)},")
    print("// each the double nearest to the exact value; ln 2 = kLn2Hi + kLn2Lo, kLn2Hi with")
    print("// 42 significant bits so that k * kLn2Hi is exact for |k| < 2^11.")
    print("#pragma once")
    print(f"constexpr double kLn2Hi = {hi.hex()};")
    print(f"constexpr double kLn2Lo = {lo.hex()};")
    print("static __device__ __align__(16) const double c_log_tab[128][2] = {")
    for lnF, inv in rows:
        print(f"    {{{lnF.hex()}, {inv.hex()}}},")
    print("};")


if __name__ == "__main__":
    main()
