"""JavaScript number formatting, for the reports the reference writes from JavaScript.

to_fixed(x, f)   Number.prototype.toFixed (ECMA-262 21.1.3.3): the exact binary value
                 rounded to f decimals, ties away from zero; "-" for negatives, so
                 (-0.001).toFixed(2) is "-0.00" and (-0).toFixed(2) is "0.00"; values
                 of magnitude 1e21 and up are printed by Number::toString.
to_string(x)     Number::toString (ECMA-262 6.1.6.1.20): the shortest digits that read
                 back as x, plain notation for 1e-7 < |x| < 1e21, exponent form
                 ("1e+21", "1.5e-7") outside.
"""
from __future__ import annotations

import math
from decimal import ROUND_HALF_UP, Decimal


def to_string(x: float) -> str:
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    if x == 0:
        return "0"
    if x < 0:
        return "-" + to_string(-x)
    # repr gives the shortest round-tripping digits: value = D x 10^(exp - len(B)) for
    # repr = "A.B" or "A.Be<exp>"; re-lay them out as JavaScript does
    mant, _, exp = repr(x).partition("e")
    a, _, b = mant.partition(".")
    d = (a + b).lstrip("0")
    scale = (int(exp) if exp else 0) - len(b)
    stripped = d.rstrip("0")
    scale += len(d) - len(stripped)
    digits = stripped
    k = len(digits)
    n = k + scale  # value = digits x 10^(n - k)
    if k <= n <= 21:
        return digits + "0" * (n - k)
    if 0 < n <= 21:
        return digits[:n] + "." + digits[n:]
    if -6 < n <= 0:
        return "0." + "0" * (-n) + digits
    e = n - 1
    sign = "+" if e >= 0 else "-"
    return (digits if k == 1 else digits[0] + "." + digits[1:]) + "e" + sign + str(abs(e))


def to_fixed(x: float, digits: int) -> str:
    x = float(x)
    if math.isnan(x):
        return "NaN"
    sign = "-" if x < 0 else ""
    x = abs(x)
    if x >= 1e21:
        return sign + to_string(x)
    q = Decimal(x).quantize(Decimal(1).scaleb(-digits), rounding=ROUND_HALF_UP)
    return sign + format(q, "f")
