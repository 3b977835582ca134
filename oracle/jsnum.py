"""JavaScript number-to-text conversions restated from ECMA-262 -- TEST INFRASTRUCTURE ONLY.

An independent check of aerosim_b200.jsfmt, which the telemetry writer
(src/solver/domainWorkflows.ts:323-402) prints through:
  to_fixed   Number.prototype.toFixed (21.1.3.3) with exact rational arithmetic: n is
             the integer nearest x * 10^f, the larger one on a tie.
  to_string  Number::toString (6.1.6.1.20): the fewest significant digits k that read
             back as x (found by trying k = 1..17 correctly rounded), laid out by the
             spec's four cases.
Pinned by known outputs of the JavaScript functions in tests/test_telemetry.py.
"""
from __future__ import annotations

import math
from fractions import Fraction


def to_string(x: float) -> str:
    if math.isnan(x):
        return "NaN"
    if x == 0:
        return "0"
    if x < 0:
        return "-" + to_string(-x)
    if math.isinf(x):
        return "Infinity"
    for k in range(1, 18):
        s = f"{x:.{k - 1}e}"
        if float(s) == x:
            break
    mant, exp = s.split("e")
    digits = mant.replace(".", "").rstrip("0") or "0"
    k = len(digits)
    n = int(exp) + 1
    if k <= n <= 21:
        return digits + "0" * (n - k)
    if 0 < n <= 21:
        return digits[:n] + "." + digits[n:]
    if -6 < n <= 0:
        return "0." + "0" * (-n) + digits
    e = n - 1
    return (digits[0] + ("." + digits[1:] if k > 1 else "")) + ("e+" if e >= 0 else "e-") + str(abs(e))


def to_fixed(x: float, f: int) -> str:
    if math.isnan(x):
        return "NaN"
    s = ""
    if x < 0:
        s, x = "-", -x
    if x >= 1e21:
        return s + to_string(x)
    v = Fraction(x) * 10 ** f
    n = math.floor(v + Fraction(1, 2))
    m = str(n)
    if f:
        m = m.rjust(f + 1, "0")
        m = m[:-f] + "." + m[-f:]
    return s + m
