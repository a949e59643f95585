"""Writes sincos_table.inc: the table of dd::sincos's quick phase in crmath.cuh.

Entry j (0..51) is {sin(j/64) hi, lo, cos(j/64) hi, lo}, each split into a
double-double, from Taylor series summed with 80 decimal digits.

    python mckl_b200/csrc/gen_sincos_table.py > mckl_b200/csrc/sincos_table.inc
"""
from decimal import Decimal, getcontext

getcontext().prec = 80


def sin_cos(a):
    """sin a and cos a by their Taylor series (|a| < 1)."""
    s, c = Decimal(0), Decimal(0)
    term = Decimal(1)  # a^n / n!
    n = 0
    eps = Decimal(10) ** -78
    while True:
        if n % 4 == 0:
            c += term
        elif n % 4 == 1:
            s += term
        elif n % 4 == 2:
            c -= term
        else:
            s -= term
        n += 1
        term = term * a / n
        if abs(term) < eps:
            return s, c


def split(v):
    hi = float(v)
    return hi, float(v - Decimal(hi))


def main():
    print("// generated by gen_sincos_table.py: {sin(j/64) hi, lo, cos(j/64) hi, lo} for j = 0..51")
    for j in range(52):
        s, c = sin_cos(Decimal(j) / 64)
        sh, sl = split(s)
        ch, cl = split(c)
        print(f"    {{{sh.hex()}, {sl.hex()}, {ch.hex()}, {cl.hex()}}},")


if __name__ == "__main__":
    main()
