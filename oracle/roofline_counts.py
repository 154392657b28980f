"""Exact algorithmic work per unit from the oracle's own arithmetic (test
infrastructure).

Builds oracle/opcount.cpp (the oracle compiled with a counting scalar),
runs it over seeded particles at several tolerances and output grids, and
fits, for each integrator and force, the operations per accepted step, per
rejected step, per emitted sample and per particle.  The integrators'
per-unit costs are constant (no data-dependent loops), so the least-squares
fit must be exact: the script fails unless every run is reproduced to the
operation (the Bovy force's counts to within 1e-4 of each run).  Writes
astrodrift_b200/roofline_counts.json, which bench.py uses
for roofline.achieved.

    python oracle/roofline_counts.py
"""

from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "astrodrift_b200" / "roofline_counts.json"
FIELDS = ("flops", "pow", "exp", "log", "sqrt", "gamma")


def run_counts() -> dict:
    with tempfile.TemporaryDirectory() as d:
        exe = Path(d) / "opcount"
        subprocess.run(["g++", "-O1", "-std=c++17", "-fpermissive", "-ffp-contract=off", "-w",
                        "-I", str(HERE), str(HERE / "opcount.cpp"), "-o", str(exe)], check=True)
        lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows: dict[str, list] = {}
    for line in lines:
        if not line.strip():
            continue
        name, *vals = line.split()
        rows.setdefault(name, []).append([int(v) for v in vals])
    return {k: np.array(v, dtype=np.int64) for k, v in rows.items()}


def fit(rows: np.ndarray) -> dict:
    # columns: accepted, rejected, samples, then the FIELDS.  With a single
    # sample count (DOPR54's one-interval runs) its column merges into the
    # per-particle constant and per_sample is not determined.
    single = len(np.unique(rows[:, 2])) == 1
    cols = [rows[:, 0], rows[:, 1]] + ([] if single else [rows[:, 2]]) + [np.ones(len(rows))]
    design = np.column_stack(cols).astype(float)
    out = {}
    for j, name in enumerate(FIELDS):
        y = rows[:, 3 + j].astype(float)
        coef, *_ = np.linalg.lstsq(design, y, rcond=None)
        coef = np.round(coef).astype(np.int64)
        resid = np.abs(design @ coef - y)
        # Exact for Kepler and Plummer.  With the Bovy force a few runs are
        # off by a handful of operations in 10^5 (consecutive rejections cost
        # one multiplication fewer than isolated ones; a particle whose
        # initial-step estimate takes Hairer's fallback skips one pow); the
        # residual is recorded and must stay within 1e-4 of the run's count
        # or one operation per particle.
        rel = float((resid / np.maximum(y, 1.0)).max())
        if (resid > np.maximum(1e-4 * y, 1.0)).any():
            raise SystemExit(f"{name}: the linear model does not reproduce the counts (max residual "
                             f"{resid.max()}, {rel:.2e} relative)")
        out[name] = {"per_accepted": int(coef[0]), "per_rejected": int(coef[1]),
                     "per_sample": None if single else int(coef[2]), "per_particle": int(coef[-1])}
        if rel > 0.0:
            out[name]["max_rel_residual"] = rel
    out["runs"] = int(len(rows))
    return out


def main() -> int:
    rows = run_counts()
    result = {
        "convention": "+ - * / and sqrt = 1 flop each (the oracle has no fused multiply-add); pow, exp, "
                      "log and the Bovy bulge's lower incomplete gamma counted as calls, pow(x, 2) as one "
                      "multiplication; comparisons, fabs, fmin/fmax, floor/ceil/round not counted",
        "source": "oracle/drift_oracle.c compiled with a counting scalar (oracle/opcount.cpp), "
                  "exact least-squares fit over seeded runs (oracle/roofline_counts.py)",
        "units": "accepted step, rejected step and emitted sample of one particle; per_particle is the "
                 "set-up (initial step size and first force evaluation)",
    }
    for name, rows_k in sorted(rows.items()):
        result[name] = fit(rows_k)
    OUT.write_text(json.dumps(result, indent=2) + "\n")
    for name in sorted(rows):
        f = result[name]["flops"]
        print(f"{name}: {f['per_accepted']} flops/accepted, {f['per_rejected']}/rejected, "
              f"{f['per_sample']}/sample, {f['per_particle']}/particle; pow per accepted "
              f"{result[name]['pow']['per_accepted']}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
