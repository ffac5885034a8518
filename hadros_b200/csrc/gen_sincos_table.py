"""Generates hadros_sincos_table.h: sin and cos of j/128 (j = 0..kTabN-1)
as double-double pairs, and pi/2 in three parts, for the correctly rounded
sin/cos of hadros_cr_math.cuh.  Values come from Python's decimal module at
60 significant digits (pi by Machin's formula, sin/cos by their Taylor
series), so every pair carries its value to about 106 bits.

    python hadros_b200/csrc/gen_sincos_table.py   # rewrites the header beside it
"""
from __future__ import annotations

from decimal import Decimal, getcontext
from fractions import Fraction
from pathlib import Path

getcontext().prec = 60
N = 104   # j/128 up to 103/128 = 0.805 > pi/4 + 1/256


def arctan_inv(x: int) -> Decimal:
    """arctan(1/x) by its series."""
    x2 = x * x
    term = Decimal(1) / x
    total, k, sign = term, 1, 1
    while True:
        term /= x2
        k += 2
        sign = -sign
        t = term / k
        if t < Decimal(10) ** -65:
            return total
        total += sign * t


PI = 16 * arctan_inv(5) - 4 * arctan_inv(239)


def sin_cos(x: Decimal) -> tuple[Decimal, Decimal]:
    s, c, term, n = Decimal(0), Decimal(0), Decimal(1), 0
    while True:   # term = x^n / n!
        if n % 4 == 0:
            c += term
        elif n % 4 == 1:
            s += term
        elif n % 4 == 2:
            c -= term
        else:
            s -= term
        n += 1
        term = term * x / n
        if abs(term) < Decimal(10) ** -64:
            return s, c


def split(v: Decimal) -> tuple[float, float]:
    """v as hi + lo, hi = v rounded to double, lo = (v - hi) rounded."""
    hi = float(v)
    lo = float(v - Decimal(Fraction(hi).numerator) / Decimal(Fraction(hi).denominator))
    return hi, lo


def truncated(v: Decimal, bits: int) -> float:
    """v truncated to `bits` significant bits (exactly representable)."""
    e = 0
    a = abs(v)
    while a >= 1:
        a /= 2
        e += 1
    while a < Decimal("0.5"):
        a *= 2
        e -= 1
    m = int(a * (1 << bits))
    return float(Fraction(m * (1 if v > 0 else -1), 1 << bits) * Fraction(2) ** e)


def main() -> None:
    half_pi = PI / 2
    p1 = truncated(half_pi, 33)
    r = half_pi - Decimal(Fraction(p1).numerator) / Decimal(Fraction(p1).denominator)
    p2 = truncated(r, 33)
    r -= Decimal(Fraction(p2).numerator) / Decimal(Fraction(p2).denominator)
    p3 = float(r)
    rows = []
    for j in range(N):
        s, c = sin_cos(Decimal(j) / 128)
        rows.append((*split(s), *split(c)))
    lines = ["// hadros_sincos_table.h — generated by gen_sincos_table.py; do not edit.",
             "// sin(j/128) and cos(j/128) as double-double pairs (hi, lo, hi, lo), and",
             "// pi/2 = P1 + P2 + P3 with P1, P2 of 33 significant bits.",
             "#pragma once", "",
             f"#define HADROS_SC_N {N}",
             f"#define HADROS_PIO2_1 {p1!r}",
             f"#define HADROS_PIO2_2 {p2!r}",
             f"#define HADROS_PIO2_3 {p3!r}",
             f"#define HADROS_2_OVER_PI {float(2 / PI)!r}",
             "#define HADROS_SC_TABLE \\", "    { \\"]
    for j, (sh, sl, ch, cl) in enumerate(rows):
        lines.append(f"        {sh!r}, {sl!r}, {ch!r}, {cl!r}, \\")
    lines.append("    }")
    lines.append("")
    Path(__file__).with_name("hadros_sincos_table.h").write_text("\n".join(lines))


if __name__ == "__main__":
    main()
