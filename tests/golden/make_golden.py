"""Generate the golden fixtures in tests/golden/ from the CPU oracle.

The oracle is pinned to the reference's own golden vectors (the DOPR54 tails
of tests/galpy_integrator_tests.rs:26-42, checked bit for bit in
tests/test_oracle.py).  The reference's galpy fixture corpus is not
committed upstream (tests/fixtures/galpy_native/README.md), so its inputs are
regenerated here with the reference's own recipe
(scripts/generate_galpy_fixtures.py:347-401: reference orbit, seed
0xA57D0F54, 100 cases) and the oracle's outputs stand in for galpy's dumps,
which the reference asserts its CPU port reproduces bit for bit
(tests/galpy_integrator_tests.rs:104-131, 339-365).

Run: python tests/golden/make_golden.py   (writes *.npz next to this file)
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

SEED = 0xA57D0F54
N_CASES = 100
CORPUS_STEPS = 1000
REFERENCE_STEPS = 1001


def cyl_to_rect(orbit):
    """[R, vR, vT, z, vz, phi] -> [x, y, z, vx, vy, vz]."""
    R, vR, vT, z, vz, phi = orbit
    c, s = np.cos(phi), np.sin(phi)
    return np.array([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz])


def seeded_cases():
    """scripts/generate_galpy_fixtures.py:383-401."""
    rng = np.random.default_rng(SEED)
    for _ in range(N_CASES):
        radius = rng.uniform(0.75, 2.25)
        phi = rng.uniform(-np.pi, np.pi)
        z = rng.uniform(-0.35, 0.35)
        radial_velocity = rng.uniform(-0.35, 0.35)
        tangential_velocity = rng.uniform(0.65, 1.25) / np.sqrt(radius)
        z_velocity = rng.uniform(-0.25, 0.25)
        end_time = rng.uniform(0.75, 1.50)
        orbit = [radius, radial_velocity, tangential_velocity, z, z_velocity, phi]
        yield cyl_to_rect(orbit), end_time


def reference_cases():
    """The reference orbit (1,0,0,0,1,0) over linspace(0, 10, 1001) at ln(1e-12)."""
    yo = np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0])
    t = np.linspace(0.0, 10.0, REFERENCE_STEPS)
    tol = float(np.log(1e-12))
    kep = oracle.kepler(1.0)
    r54, err, st, s54 = oracle.dopr54(kep, yo, t, tol, tol)
    assert err == 0 and st == 0
    r853, st, s853 = oracle.dop853(kep, yo, t, tol, tol)
    assert st == 0
    return dict(yo=yo, t=t, tol_ln=tol, dopr54=r54, dop853=r853,
                dopr54_steps=np.array([s54.accepted, s54.rejected, s54.rhs]),
                dop853_steps=np.array([s853.accepted, s853.rejected, s853.rhs]))


def corpus():
    """Seeded Kepler corpus: final state, step counts and 4 full trajectories per method."""
    cases = list(seeded_cases())
    y0 = np.stack([c[0] for c in cases])
    t_end = np.array([c[1] for c in cases])
    tol = float(np.log(1e-12))
    kep = oracle.kepler(1.0)
    out = dict(y0=y0, t_end=t_end, tol_ln=tol)
    for name, fn in (("dopr54", oracle.dopr54), ("dop853", oracle.dop853)):
        finals, steps, full = [], [], []
        for i, (yo, te) in enumerate(cases):
            t = np.linspace(0.0, te, CORPUS_STEPS)
            if name == "dopr54":
                res, err, st, stats = fn(kep, yo, t, tol, tol)
                assert err == 0
            else:
                res, st, stats = fn(kep, yo, t, tol, tol)
            assert st == 0
            finals.append(res[-1])
            steps.append([stats.accepted, stats.rejected])
            if i < 4:
                full.append(res)
        out[f"{name}_final"] = np.array(finals)
        out[f"{name}_steps"] = np.array(steps)
        out[f"{name}_full4"] = np.array(full)
    return out


def potential_batches():
    """Small seeded Plummer and Bovy batches for both methods (final states)."""
    rng = np.random.default_rng(20261203)
    out = {}
    n = 64
    # Plummer: near-bound orbits in r in [0.2, 3]
    r = rng.uniform(0.2, 3.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = rng.normal(size=(n, 3))
    v -= (v * u).sum(1, keepdims=True) * u
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    vc = np.sqrt(r * r / (r * r + 1.0) ** 1.5)
    yp = np.hstack([u * r[:, None], v * (vc * rng.uniform(0.6, 1.1, n))[:, None]])
    # Bovy: disk-like orbits, R in [0.2, 5]
    R = np.exp(rng.uniform(np.log(0.2), np.log(5.0), n))
    phi = rng.uniform(0, 2 * np.pi, n)
    z = rng.normal(0, 0.1, n) * R
    bov = oracle.bovy()
    vcb = np.array([np.sqrt(Ri * abs(oracle.force(bov, Ri, 0.0, 0.0)[0])) for Ri in R])
    vT = vcb * (1 + 0.1 * rng.normal(size=n))
    vR = 0.1 * vcb * rng.normal(size=n)
    vz = 0.1 * vcb * rng.normal(size=n)
    yb = np.stack([R * np.cos(phi), R * np.sin(phi), z,
                   vR * np.cos(phi) - vT * np.sin(phi), vR * np.sin(phi) + vT * np.cos(phi), vz], 1)
    ts = np.linspace(0.0, 20.0, 41)
    for pname, pot, y0 in (("plummer", oracle.plummer(1.0, 1.0), yp), ("bovy", bov, yb)):
        out[f"{pname}_y0"] = y0
        for mname, m in (("dopr54", oracle.DOPR54), ("dop853", oracle.DOP853)):
            res = oracle.integrate_batch(m, pot, y0, ts=ts, rtol=1e-10, atol=1e-10, threads=8)
            assert res["failures"] == 0
            out[f"{pname}_{mname}_final"] = res["out"][-1]
            out[f"{pname}_{mname}_mid"] = res["out"][20]
            out[f"{pname}_{mname}_accepted"] = res["accepted"]
            out[f"{pname}_{mname}_rejected"] = res["rejected"]
    out["ts"] = ts
    return out


def main():
    oracle.build()
    np.savez_compressed(HERE / "reference_orbit.npz", **reference_cases())
    np.savez_compressed(HERE / "kepler_corpus.npz", **corpus())
    np.savez_compressed(HERE / "potential_batches.npz", **potential_batches())
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
