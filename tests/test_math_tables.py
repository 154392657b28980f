"""The contraction unit's table-driven ln and exp (drift_math.cuh log_tab,
exp_tab), checked on the host.

* drift_math_tables.h is what gen_math_tables.py generates, and every entry
  is the correctly rounded value it documents (60-digit decimal reference).
* The two functions, emulated step by step in exact rational arithmetic
  (every fused multiply-add rounded once, as the device rounds it), stay
  within a few ulps of the true ln and exp on the ranges the Bovy force uses:
  ln(1 + u) for the halo and exp(s ln x) for the bulge (where ln x needs
  only absolute accuracy).
"""

from __future__ import annotations

import math
import struct
import subprocess
import sys
from decimal import Decimal, getcontext
from fractions import Fraction
from pathlib import Path

import numpy as np

CSRC = Path(__file__).resolve().parent.parent / "astrodrift_b200" / "csrc"
getcontext().prec = 60


def _table():
    text = (CSRC / "drift_math_tables.h").read_text()
    body = text[text.index("MATH_TABLE_INIT"):]
    body = body[body.index("{") + 1:body.index("}")]
    return [float.fromhex(v.strip()) for v in body.split(",") if v.strip()]


def test_header_is_the_generator_output_and_correctly_rounded():
    gen = subprocess.run([sys.executable, str(CSRC / "gen_math_tables.py")], capture_output=True, text=True,
                         check=True).stdout
    assert gen == (CSRC / "drift_math_tables.h").read_text()
    t = _table()
    assert len(t) == 2 * 128 + 64
    for i in range(128):
        inv_c, l_i = t[2 * i], t[2 * i + 1]
        assert inv_c == float(Decimal(1) / (Decimal(1) + Decimal(i) / 128))
        assert l_i == float(-Decimal(inv_c).ln())
    for j in range(64):
        assert t[256 + j] == float((Decimal(2).ln() * j / 64).exp())


def _fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _bits(x):
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _from_bits(b):
    return struct.unpack("<d", struct.pack("<q", b))[0]


LN2_HI, LN2_LO = 0.6931471805599453, 2.3190468138462996e-17
LN2_64_HI, LN2_64_LO = float.fromhex("0x1.62e42fefa0000p-7"), float.fromhex("0x1.cf79abc9e3b3ap-46")
INV_LN2_64 = float.fromhex("0x1.71547652b82fep+6")


def log_tab(t, x):
    bits = _bits(x)
    k = (bits >> 52) - 1023
    i = (bits >> 45) & 127
    m = _from_bits((bits & 0x000FFFFFFFFFFFFF) | 0x3FF0000000000000)
    r = _fma(m, t[2 * i], -1.0)
    p = -1.0 / 8.0
    for c in (1.0 / 7.0, -1.0 / 6.0, 1.0 / 5.0, -1.0 / 4.0, 1.0 / 3.0, -1.0 / 2.0):
        p = _fma(p, r, c)
    lp = _fma(p * r, r, r)
    kd = float(k)
    return _fma(kd, LN2_HI, t[2 * i + 1] + _fma(kd, LN2_LO, lp))


def exp_tab(t, x):
    kd = float(np.rint(x * INV_LN2_64))
    r = _fma(-kd, LN2_64_LO, _fma(-kd, LN2_64_HI, x))
    k = int(kd)
    j, e = k & 63, k >> 6
    p = 1.0 / 120.0
    for c in (1.0 / 24.0, 1.0 / 6.0, 0.5):
        p = _fma(p, r, c)
    p = _fma(p, r, 1.0) * r
    tj = t[256 + j]
    return _fma(tj, p, tj) * math.ldexp(1.0, e)


def _ulps(got, ref: Decimal):
    r = float(ref)
    return float(abs(Decimal(got) - ref)) / (math.nextafter(abs(r), math.inf) - abs(r))


def test_log_and_exp_within_a_few_ulps():
    t = _table()
    rng = np.random.default_rng(7)
    worst_log = worst_exp = worst_abs = 0.0
    for u in np.exp(rng.uniform(np.log(1e-8), np.log(50.0), 1500)):  # halo: ln(1 + u)
        a = 1.0 + float(u)
        worst_log = max(worst_log, _ulps(log_tab(t, a), Decimal(a).ln()))
    for x in np.exp(rng.uniform(np.log(1e-12), np.log(40.0), 1500)):  # bulge: ln x, absolute
        x = float(x)
        worst_abs = max(worst_abs, float(abs(Decimal(log_tab(t, x)) - Decimal(x).ln())))
    for x in np.concatenate([rng.uniform(-700.0, 700.0, 1000), rng.uniform(-20.0, 5.0, 1000)]):
        x = float(x)
        worst_exp = max(worst_exp, _ulps(exp_tab(t, x), Decimal(x).exp()))
    assert worst_log < 2.0, worst_log
    assert worst_exp < 2.0, worst_exp
    assert worst_abs < 2e-15, worst_abs
