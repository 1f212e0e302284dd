"""Generate dd_tables.h: double-double constants for the correctly rounded
exp/log in dd_math.cuh.

Every constant is computed here from its definition with Python's exact
rational / 60-digit decimal arithmetic and split as hi = RN(value),
lo = RN(value - hi).  Run:  python gen_dd_tables.py > dd_tables.h
"""
from decimal import Decimal, getcontext
from fractions import Fraction
import math

getcontext().prec = 80


def dd(value: Decimal):
    hi = float(value)
    lo = float(value - Decimal(hi))
    return hi, lo


def ln(x: Decimal) -> Decimal:
    return x.ln()


def emit(name, pairs):
    print(f"#define {name.upper()}_N {len(pairs)}")
    body = ", ".join(f"{{{hi.hex()}, {lo.hex()}}}" for hi, lo in pairs)
    print(f"#define {name.upper()}_INIT {{ {body} }}")


print("/* Generated by gen_dd_tables.py -- do not edit. */")
print("#pragma once")
ln2 = ln(Decimal(2))
h, l = dd(ln2)
print(f"#define DD_LN2_HI {h.hex()}")
print(f"#define DD_LN2_LO {l.hex()}")
print(f"#define DD_INV_LN2 {float(1 / ln2).hex()}")
# 1/k! for the exp Taylor series, k = 0..14
emit("dd_inv_fact", [dd(Decimal(Fraction(1, math.factorial(k)).numerator) /
                        Decimal(Fraction(1, math.factorial(k)).denominator)) for k in range(15)])
# 1/(2k+1) for the atanh series, k = 0..8
emit("dd_inv_odd", [dd(Decimal(1) / Decimal(2 * k + 1)) for k in range(9)])
# log(j/64) for j = 48..96 (table points of the log reduction)
emit("dd_log_j64", [dd(ln(Decimal(j) / Decimal(64))) for j in range(48, 97)])
