"""Derives the constants of the double-precision sine used by the oracle
(mercury_oracle.c: or_sin) and by the CUDA actuation table
(mercury_b200/csrc/mb_sin.cuh).

Method: Cody & Waite (1980) argument reduction x = k*(pi/2) + r with pi/2
split into three parts, C1 and C2 carrying 33 significant bits each (so that
k*C1 and k*C2 are exact for |k| < 2^20) and C3 the rounded remainder; then
the Taylor series of sin and cos on |r| <= pi/4.

pi is computed from Machin's formula pi = 16 atan(1/5) - 4 atan(1/239) in
exact integer arithmetic; every constant is the correctly rounded double of
an exact rational.  Run: python oracle/sin_constants.py
"""
from fractions import Fraction
from math import factorial

DIGITS = 80  # decimal digits of working precision for pi


def _atan_inv(n: int, scale: int) -> int:
    """atan(1/n) * scale by its alternating series, in integers."""
    total, term, k, sign = 0, scale // n, 1, 1
    n2 = n * n
    while term:
        total += sign * (term // k)
        term //= n2
        k += 2
        sign = -sign
    return total


def pi_fraction() -> Fraction:
    scale = 10 ** (DIGITS + 10)
    return Fraction(16 * _atan_inv(5, scale) - 4 * _atan_inv(239, scale), scale)


def round_bits(x: Fraction, bits: int) -> Fraction:
    """x rounded to `bits` significant binary digits (nearest)."""
    if x == 0:
        return x
    e = 0
    ax = abs(x)
    while ax >= 2:
        ax /= 2
        e += 1
    while ax < 1:
        ax *= 2
        e -= 1
    m = round(ax * (1 << (bits - 1)))
    return Fraction(m, 1 << (bits - 1)) * (Fraction(2) ** e) * (1 if x > 0 else -1)


def constants():
    pi = pi_fraction()
    half_pi = pi / 2
    c1 = round_bits(half_pi, 33)
    c2 = round_bits(half_pi - c1, 33)
    c3 = float(half_pi - c1 - c2)
    two_over_pi = float(2 / pi)
    sin_c = [float(Fraction((-1) ** k, factorial(2 * k + 1))) for k in range(10)]
    cos_c = [float(Fraction((-1) ** k, factorial(2 * k))) for k in range(11)]
    return two_over_pi, float(c1), float(c2), c3, sin_c, cos_c


if __name__ == "__main__":
    t, c1, c2, c3, s, c = constants()
    print(f"2/pi     = {t!r}")
    print(f"pi/2 C1  = {c1!r}")
    print(f"pi/2 C2  = {c2!r}")
    print(f"pi/2 C3  = {c3!r}")
    print("sin coef = " + ", ".join(repr(v) for v in s))
    print("cos coef = " + ", ".join(repr(v) for v in c))
