"""Generates drift_math_tables.h: the lookup tables of the contraction
unit's natural log and exp (drift_math.cuh, log_tab / exp_tab).

    python astrodrift_b200/csrc/gen_math_tables.py > astrodrift_b200/csrc/drift_math_tables.h

Every entry is computed with 60-digit decimal arithmetic and rounded once to
the nearest double:
  LOG_INV_C[i] = RN(1 / c_i),  c_i = 1 + i / 128            (i = 0 .. 127)
  LOG_L[i]     = RN(-ln(LOG_INV_C[i]))  (of the rounded reciprocal, so that
                 ln m = LOG_L[i] + ln(m * LOG_INV_C[i]) holds exactly)
  EXP_T[j]     = RN(2^(j / 64))                               (j = 0 .. 63)
stored in MATH_TABLE_INIT as (LOG_INV_C[i], LOG_L[i]) pairs, then EXP_T, so
that one 16-byte load fetches both log entries.
"""

from __future__ import annotations

from decimal import Decimal, getcontext

getcontext().prec = 60


def rn(d: Decimal) -> float:
    return float(d)  # Decimal -> float rounds correctly to nearest


def hexlit(v: float) -> str:
    return v.hex() if v != 0.0 else "0x0p+0"


def main() -> None:
    inv_c = [rn(Decimal(1) / (Decimal(1) + Decimal(i) / 128)) for i in range(128)]
    log_l = [rn(-Decimal(v).ln()) for v in inv_c]
    exp_t = [rn((Decimal(2).ln() * Decimal(j) / 64).exp()) for j in range(64)]
    print("// drift_math_tables.h -- generated by gen_math_tables.py; do not edit.")
    print("// Lookup tables of the contraction unit's log and exp (drift_math.cuh), in")
    print("// constant memory; kernels stage them into shared memory once per block.")
    print("#pragma once")
    print()
    print("namespace drift {")
    print("constexpr int LOG_TABLE_N = 128;")
    print("constexpr int EXP_TABLE_N = 64;")
    print("// [(LOG_INV_C[i], LOG_L[i]) pairs (128 x 2)][EXP_T (64)]")
    vals = [v for pair in zip(inv_c, log_l) for v in pair] + exp_t
    print(f"static __constant__ const double MATH_TABLE_INIT[{len(vals)}] = {{")
    for k in range(0, len(vals), 3):
        print("    " + ", ".join(hexlit(v) for v in vals[k:k + 3]) + ",")
    print("};")
    print("}  // namespace drift")


if __name__ == "__main__":
    main()
