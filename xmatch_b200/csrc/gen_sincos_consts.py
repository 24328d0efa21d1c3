"""Derive the constants of the project's FP64 sincos from first principles.

The method is Cody & Waite (1980) argument reduction by pi/2 split into three
doubles, followed by truncated Taylor series of sin and cos on |r| <= pi/4.
pi is computed here with Machin's formula in 100-digit decimal arithmetic and
the Taylor coefficients are exact rationals 1/n!, so every constant is the
double nearest to a mathematically defined number.  Running this script prints
the C literals used by ``xm_sincos.h`` (product) and ``oracle/xm_oracle.c``.
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 110


def arctan_inv(n):
    # arctan(1/n) by its alternating Taylor series
    x = Decimal(1) / n
    x2 = x * x
    term, total, k = x, Decimal(0), 0
    while True:
        t = term / (2 * k + 1)
        if t == 0 or abs(t) < Decimal(10) ** -105:
            break
        total += t if k % 2 == 0 else -t
        term *= x2
        k += 1
    return total


PI = 16 * arctan_inv(5) - 4 * arctan_inv(239)   # Machin (1706)


def nearest_double(d):
    """Double nearest to the Decimal d (round-half-even via Fraction)."""
    fr = Fraction(d)
    f = float(fr)            # float(Fraction) is correctly rounded
    return f


def hexlit(f):
    return f.hex()


def main():
    pio2 = PI / 2
    p1 = nearest_double(pio2)
    p2 = nearest_double(pio2 - Decimal(Fraction(p1).numerator) / Decimal(Fraction(p1).denominator))
    rem = pio2 - Decimal(Fraction(p1).numerator) / Decimal(Fraction(p1).denominator) \
        - Decimal(Fraction(p2).numerator) / Decimal(Fraction(p2).denominator)
    p3 = nearest_double(rem)
    two_over_pi = nearest_double(2 / PI)
    print("/* pi/2 = P1 + P2 + P3 (Cody-Waite split), 2/pi */")
    for name, v in (("XM_PIO2_1", p1), ("XM_PIO2_2", p2), ("XM_PIO2_3", p3), ("XM_2_OVER_PI", two_over_pi)):
        print(f"#define {name} {hexlit(v)}  /* {v!r} */")
    print("/* sin r = r + r^3 * (S1 + r^2 (S2 + ...)),  S_k = (-1)^k / (2k+1)! */")
    for k in range(1, 9):
        v = float(Fraction((-1) ** k, math.factorial(2 * k + 1)))
        print(f"#define XM_S{k} {hexlit(v)}  /* {v!r} */")
    print("/* cos r = 1 + r^2 * (C1 + r^2 (C2 + ...)),  C_k = (-1)^k / (2k)! */")
    for k in range(1, 10):
        v = float(Fraction((-1) ** k, math.factorial(2 * k)))
        print(f"#define XM_C{k} {hexlit(v)}  /* {v!r} */")


if __name__ == "__main__":
    main()
