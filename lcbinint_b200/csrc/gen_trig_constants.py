"""Prints the constants of lcbi_trig.cuh: pi/2 split into four 33-bit parts
and a 53-bit remainder, 2/pi, and the Taylor coefficients (-1)^n/(2n+1)!
and (-1)^n/(2n)! as double-double pairs (hi, lo), all from exact rational
arithmetic (pi from mpmath at 400 bits).  Run it to check the header."""
from fractions import Fraction
from math import factorial

import mpmath

mpmath.mp.prec = 400


def exact(x) -> Fraction:
    m, e = mpmath.mpf(x).man_exp
    return Fraction(m) * Fraction(2) ** e if e >= 0 else Fraction(m, 2 ** -e)


def split_dd(fr: Fraction):
    hi = float(fr)
    return hi, float(fr - Fraction(hi))


def head(fr: Fraction, bits: int) -> float:
    """fr truncated to its leading `bits` significant bits (an exact double)."""
    e = fr.numerator.bit_length() - fr.denominator.bit_length()
    while Fraction(2) ** e > fr:
        e -= 1
    while Fraction(2) ** (e + 1) <= fr:
        e += 1
    scale = Fraction(2) ** (bits - 1 - e)
    v = Fraction(int(fr * scale)) / scale
    assert Fraction(float(v)) == v
    return float(v)


def main():
    half_pi = exact(mpmath.pi) / 2
    rest = half_pi
    parts = []
    for _ in range(4):
        c = head(rest, 33)
        parts.append(c)
        rest -= Fraction(c)
    parts.append(float(rest))
    print("// pi/2 = kP1 + kP2 + kP3 + kP4 + kP5 (kP1..kP4: 33 significant bits each)")
    for i, p in enumerate(parts, 1):
        print(f"constexpr double kP{i} = {p.hex()};")
    print(f"constexpr double kTwoOverPi = {float(2 / exact(mpmath.pi)).hex()};")
    print("// (-1)^n / (2n+1)!, n = 0..13")
    for n in range(14):
        hi, lo = split_dd(Fraction((-1) ** n, factorial(2 * n + 1)))
        print(f"    {{{hi.hex()}, {lo.hex()}}},")
    print("// (-1)^n / (2n)!, n = 0..14")
    for n in range(15):
        hi, lo = split_dd(Fraction((-1) ** n, factorial(2 * n)))
        print(f"    {{{hi.hex()}, {lo.hex()}}},")


if __name__ == "__main__":
    main()
