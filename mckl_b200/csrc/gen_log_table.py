"""Writes log_table.inc: the reduction table of dd::log in crmath.cuh.

Entry i (0..127) serves mantissas m in [1 + i/128, 1 + (i+1)/128): inv_i =
a_i / 256 with a_i = round(256 / (1 + (i + 0.5)/128)) (a_0 = 256, a_127 =
128, so that m near 1 and near 2 reduce without cancellation), and
-ln(inv_i) split into a double-double (hi, lo), computed with 80 decimal
digits.  r = m inv_i - 1 is then exact in one fma (|r| <= 2^-7, and m inv_i
has at most 62 significant bits above 2^-60).

    python mckl_b200/csrc/gen_log_table.py > mckl_b200/csrc/log_table.inc
"""
from decimal import Decimal, getcontext

getcontext().prec = 80


def main():
    print("// generated by gen_log_table.py: {inv_i, -ln(inv_i) hi, lo} for i = 0..127")
    for i in range(128):
        if i == 0:
            a = 256
        elif i == 127:
            a = 128
        else:
            a = int((Decimal(256) / (Decimal(1) + (Decimal(i) + Decimal("0.5")) / 128)).to_integral_value())
        inv = Decimal(a) / 256
        L = -inv.ln()
        hi = float(L)
        lo = float(L - Decimal(hi))
        print(f"    {{{float(inv).hex()}, {hi.hex()}, {lo.hex()}}},")


if __name__ == "__main__":
    main()
