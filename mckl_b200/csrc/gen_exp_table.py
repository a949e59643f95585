"""Writes exp_table.inc: the table of dd::exp's quick phase in crmath.cuh.

Entry j (0..63) is 2^(j/64) split into a double-double (hi, lo), computed with
80 decimal digits.  The header comment also carries the Cody-Waite split of
ln2/64 the quick phase reduces with: L1 rounded to 36 significant bits (so
k * L1 is exact for |k| < 2^17) and L2 = RN(ln2/64 - L1).

    python mckl_b200/csrc/gen_exp_table.py > mckl_b200/csrc/exp_table.inc
"""
import math
from decimal import Decimal, getcontext

getcontext().prec = 80


def split36(v):
    """v rounded to 36 significant bits (v > 0)."""
    e = math.frexp(float(v))[1]  # v = m 2^e, m in [0.5, 1)
    scale = Decimal(2) ** (36 - e)
    return float((v * scale).to_integral_value() / scale)


def main():
    l64 = Decimal(2).ln() / 64
    L1 = split36(l64)
    L2 = float(l64 - Decimal(L1))
    print(f"// generated by gen_exp_table.py: {{2^(j/64) hi, lo}} for j = 0..63;")
    print(f"// ln2/64 = L1 + L2 with L1 = {L1.hex()} (36 bits), L2 = {L2.hex()}")
    for j in range(64):
        v = Decimal(2) ** (Decimal(j) / 64)
        hi = float(v)
        lo = float(v - Decimal(hi))
        print(f"    {{{hi.hex()}, {lo.hex()}}},")


if __name__ == "__main__":
    main()
