"""Writes pow_tables.h: the constants of pow_ in math.h (run from any directory).

Every value is computed here in 60-digit decimal arithmetic and rounded once
to the nearest double, so the header can be regenerated and checked:

  kPowInv[j]   = 128 / (129 + 2j) rounded to double: the reciprocal of the
                 midpoint of the j-th of 64 equal mantissa intervals of [1, 2);
  kPowLogInv[j] = -ln(kPowInv[j]) of that double;
  kPowExp2[j]  = 2^(j/64);
  ln 2 and ln 2 / 64 split into a head of 32 significant bits (so products with
  small integers are exact) and the rounded remainder; 64 / ln 2.
"""
from __future__ import annotations

import sys
from decimal import Decimal, getcontext
from pathlib import Path

getcontext().prec = 60
OUT = Path(__file__).resolve().parent / "pow_tables.h"


def head(x: Decimal, bits: int = 32) -> float:
    """x rounded to `bits` significant bits (a double whose low bits are zero)."""
    f = float(x)
    m, e = __import__("math").frexp(f)
    scale = 2 ** bits
    return __import__("math").ldexp(round(m * scale) / scale, e)


def render() -> str:
    ln2 = Decimal(2).ln()
    inv = [128.0 / (129 + 2 * j) for j in range(64)]
    log_inv = [float(-Decimal(v).ln()) for v in inv]
    exp2 = [float(Decimal(2) ** (Decimal(j) / Decimal(64))) for j in range(64)]
    ln2_hi = head(ln2)
    ln2_lo = float(ln2 - Decimal(ln2_hi))
    l64 = ln2 / 64
    l64_hi = head(l64)
    l64_lo = float(l64 - Decimal(l64_hi))
    inv_l64 = float(64 / ln2)

    def table(name, vals):
        rows = [", ".join(float.hex(v) for v in vals[i:i + 4]) for i in range(0, len(vals), 4)]
        return f"#define {name} {{ \\\n    " + ", \\\n    ".join(rows) + " }\n"

    return ("// Generated by gen_pow_tables.py (the constants of pow_ in math.h); do not edit.\n"
            "#pragma once\n\n"
            + table("SOL_POW_INV", inv) + "\n"
            + table("SOL_POW_LOG_INV", log_inv) + "\n"
            + table("SOL_POW_EXP2", exp2) + "\n"
            + f"#define SOL_POW_LN2_HI {float.hex(ln2_hi)}\n"
            + f"#define SOL_POW_LN2_LO {float.hex(ln2_lo)}\n"
            + f"#define SOL_POW_LN2_64_HI {float.hex(l64_hi)}\n"
            + f"#define SOL_POW_LN2_64_LO {float.hex(l64_lo)}\n"
            + f"#define SOL_POW_INV_LN2_64 {float.hex(inv_l64)}\n")


if __name__ == "__main__":
    text = render()
    if "--check" in sys.argv:
        sys.exit(0 if OUT.read_text() == text else 1)
    OUT.write_text(text)
    print(OUT)
