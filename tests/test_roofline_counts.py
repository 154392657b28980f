"""The committed operation counts (astrodrift_b200/roofline_counts.json, which
the benchmark's roofline divides by) are reproduced by counting the oracle's
arithmetic again, and the per-unit model fits every run exactly."""

from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def test_committed_counts_match_a_fresh_count():
    sys.path.insert(0, str(ROOT / "oracle"))
    try:
        import roofline_counts
    finally:
        sys.path.pop(0)
    rows = roofline_counts.run_counts()
    committed = json.loads((ROOT / "astrodrift_b200" / "roofline_counts.json").read_text())
    for name, r in rows.items():
        assert roofline_counts.fit(r) == committed[name], name  # fit() raises unless exact
    plummer = committed["dop853_plummer"]["flops"]
    # counting the reference's DOP853 step and Plummer force by hand gives about 2,065 per accepted step
    assert abs(plummer["per_accepted"] - 2065) < 50
    assert committed["dop853_plummer"]["pow"]["per_accepted"] == 17  # 15 forces + 2 controller pows


def test_bovy_counts_cover_the_composite_force():
    """The Bovy composite has a count: per force evaluation one disk power,
    one halo log and one bulge incomplete gamma (tallied as calls), 15
    evaluations per accepted step and 11 per rejected one."""
    committed = json.loads((ROOT / "astrodrift_b200" / "roofline_counts.json").read_text())
    bovy = committed["dop853_bovy"]
    for field in ("log", "gamma"):
        assert bovy[field]["per_accepted"] == 15 and bovy[field]["per_rejected"] == 11
    assert bovy["pow"]["per_accepted"] == 17  # 15 disk powers + 2 controller powers
    # the composite's arithmetic outside those calls: tens of flops per force
    extra = bovy["flops"]["per_accepted"] - committed["dop853_plummer"]["flops"]["per_accepted"]
    assert 15 * 30 < extra < 15 * 80
    assert bovy["flops"].get("max_rel_residual", 0.0) < 1e-4
