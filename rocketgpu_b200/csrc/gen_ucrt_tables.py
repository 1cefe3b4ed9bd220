"""Generates rg_ucrt_tables.inc: the lookup tables of the single-precision atan2 / pow algorithms the reference uses
(reference include/rocketgpu/detail/math.hpp:65-457, the UCRT-compatible float routines).

The tables are mathematical constants, computed here to 60 significant digits and rounded to double (to nearest unless noted):
  atan_tab[k]  = atan((k + 16) / 256), rounded toward zero,   k = 0..240
  pow_inv_c[i] = 512 / (256 + i)  (= 1 / c_i, c_i = (256 + i) / 512),  i = 0..256
  pow_log_c[i] = ln((256 + i) / 256)  (= ln(2 c_i)),  i = 0..256
  pow_exp2[j]  = 2^(j / 64),                          j = 0..63
Run:  python rocketgpu_b200/csrc/gen_ucrt_tables.py > rocketgpu_b200/csrc/rg_ucrt_tables.inc
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 60


def to_double_hex(d: Decimal) -> str:
    # exact rational -> nearest double (ties to even), via Python's float(Fraction) which rounds correctly
    return float(Fraction(d)).hex()


def to_double_hex_trunc(d: Decimal) -> str:
    f = Fraction(d)
    x = float(f)
    if abs(Fraction(x)) > abs(f):
        x = math.nextafter(x, 0.0)
    return x.hex()


def atan(x: Decimal) -> Decimal:
    # argument reduction atan(x) = 2 atan(x / (1 + sqrt(1 + x^2))) until small, then the Taylor series
    k = 0
    while x > Decimal("0.05"):
        x = x / (1 + (1 + x * x).sqrt())
        k += 1
    s, term, n = Decimal(0), x, 1
    x2 = x * x
    while True:
        t = term / n
        if abs(t) < Decimal(10) ** -70:
            break
        s += t if (n // 2) % 2 == 0 else -t
        term *= x2
        n += 2
    return s * (2 ** k)


def ln(x: Decimal) -> Decimal:
    return x.ln()


def exp2(q: Fraction) -> Decimal:
    return (Decimal(q.numerator) / Decimal(q.denominator) * Decimal(2).ln()).exp()


def emit(name, vals):
    print(f"RG_UCRT_TABLE({name}, {len(vals)}) = {{")
    for i in range(0, len(vals), 3):
        print("    " + ", ".join(vals[i:i + 3]) + ",")
    print("};")


print("// Generated by gen_ucrt_tables.py: atan / pow lookup tables (see that script). Do not edit.")
emit("kAtanTab", [to_double_hex_trunc(atan(Decimal(k + 16) / Decimal(256))) for k in range(241)])
emit("kPowInvC", [to_double_hex(Decimal(512) / Decimal(256 + i)) for i in range(257)])
emit("kPowLogC", [to_double_hex(ln(Decimal(256 + i) / Decimal(256))) if i else "0x0.0p+0" for i in range(257)])
emit("kPowExp2", [to_double_hex(exp2(Fraction(j, 64))) for j in range(64)])
