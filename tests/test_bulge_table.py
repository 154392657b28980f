"""The bulge's incomplete-gamma table (drift_bulge_table.h), evaluated on the
host the way the device evaluates it -- gamma(s, x) = x^s E(x) with E from
the piece around the nearest odd centre -- against scipy's regularised lower
incomplete gamma, for the bulge exponents the potential admits."""

from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parent.parent / "astrodrift_b200" / "csrc"
PIECES, DEG = 20, 17  # BULGE_PIECES, BULGE_PIECE_DEG in drift_potentials.cuh


@pytest.fixture(scope="module")
def table_tool(tmp_path_factory):
    d = tmp_path_factory.mktemp("bulge")
    src = d / "table.cpp"
    src.write_text(
        '#include <cstdio>\n#include <cstdlib>\n#include "drift_bulge_table.h"\n'
        "int main(int argc, char **argv) {\n"
        f"  double out[{PIECES * (DEG + 1)}];\n"
        f"  drift::fill_bulge_table_impl(std::atof(argv[1]), out, {PIECES}, {DEG});\n"
        f"  for (int i = 0; i < {PIECES * (DEG + 1)}; i++) std::printf(\"%.17g\\n\", out[i]);\n"
        "  return 0;\n}\n")
    exe = d / "table"
    subprocess.run(["g++", "-O2", "-I", str(CSRC), str(src), "-o", str(exe)], check=True)
    return exe


def _table(exe, s):
    out = subprocess.run([str(exe), repr(s)], capture_output=True, text=True, check=True).stdout
    return np.array([float(v) for v in out.split()]).reshape(PIECES, DEG + 1)


def _evaluate(table, s, x):
    j = np.minimum((x * 0.5).astype(int), PIECES - 1)
    t = x - (2.0 * j + 1.0)
    p = table[j, DEG]
    for k in range(DEG - 1, -1, -1):
        p = p * t + table[j, k]
    return np.exp(s * np.log(x)) * p


@pytest.mark.parametrize("alpha", [0.1, 1.0, 1.8, 2.5, 2.9])
def test_table_reproduces_the_lower_incomplete_gamma(table_tool, alpha):
    from scipy.special import gamma, gammainc

    s = 1.5 - 0.5 * alpha
    table = _table(table_tool, s)
    rng = np.random.default_rng(3)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e-8), np.log(40.0), 20000)),
                        np.arange(0.0, 40.0, 2.0)[1:], np.arange(1.0, 40.0, 2.0), [39.999999]])
    got = _evaluate(table, s, x)
    ref = gammainc(s, x) * gamma(s)
    rel = np.abs(got - ref) / ref
    assert rel.max() < 1e-14, (rel.max(), x[rel.argmax()])
    # beyond the table the device returns Gamma(s): the tail it drops is tiny
    assert (1.0 - gammainc(s, 40.0)) < 1e-15
