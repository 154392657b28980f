"""The CPU oracle against the reference's golden vectors and force properties.

The oracle (oracle/drift_oracle.c) restates src/integrators/galpy/dopr54.rs and
dop853.rs.  These tests pin it: bit-exact against the DOPR54 tails recorded in
tests/galpy_integrator_tests.rs:26-42, bit-exact against the committed golden
fixtures (tests/golden/make_golden.py), and against the Plummer force
properties of shared/tests/plummer_potential_tests.rs.
"""

from __future__ import annotations

import struct
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"

# tests/galpy_integrator_tests.rs:35-42 (galpy cylindrical Kepler force)
DOPR54_EXPECTED_TAIL_BITS = [
    0xBFEAD9AC890CBF36, 0xBFE1689EF5F2F535, 0x0,
    0x3FE1689EF5F2DA37, 0xBFEAD9AC890CA90A, 0x0,
]
# tests/galpy_integrator_tests.rs:26-33 (the earlier Cartesian Kepler force)
DOPR54_CARTESIAN_TAIL_BITS = [
    0xBFEAD9AC890CBF34, 0xBFE1689EF5F2F595, 0x0,
    0x3FE1689EF5F2DA49, 0xBFEAD9AC890CA8BE, 0x0,
]


def bits(v):
    return [struct.unpack("<Q", struct.pack("<d", float(x)))[0] for x in v]


def reference_input():
    # scripts/generate_galpy_fixtures.py:347-373
    yo = np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0])
    t = np.linspace(0.0, 10.0, 1001)
    return yo, t


@pytest.mark.parametrize("tol_ln", [float(np.log(1e-12)), float("%.16g" % np.log(1e-12))])
def test_dopr54_reproduces_reference_tail_bits(oracle, tol_ln):
    yo, t = reference_input()
    res, err, status, stats = oracle.dopr54(oracle.kepler(1.0), yo, t, tol_ln, tol_ln)
    assert err == 0 and status == 0
    assert bits(res[-1]) == DOPR54_EXPECTED_TAIL_BITS
    assert stats.accepted == 1000 and stats.rejected == 0


def test_dopr54_cartesian_force_reproduces_earlier_tail_bits(oracle):
    yo, t = reference_input()
    pot = oracle.Potential(kind=oracle.POT_KEPLER_CARTESIAN if hasattr(oracle, "POT_KEPLER_CARTESIAN") else 3,
                           amp=1.0)
    tol = float(np.log(1e-12))
    res, err, status, _ = oracle.dopr54(pot, yo, t, tol, tol)
    assert err == 0 and status == 0
    assert bits(res[-1]) == DOPR54_CARTESIAN_TAIL_BITS


def test_oracle_reproduces_committed_reference_orbit(oracle):
    g = np.load(GOLDEN / "reference_orbit.npz")
    kep = oracle.kepler(1.0)
    r54, err, _, s54 = oracle.dopr54(kep, g["yo"], g["t"], float(g["tol_ln"]), float(g["tol_ln"]))
    r853, _, s853 = oracle.dop853(kep, g["yo"], g["t"], float(g["tol_ln"]), float(g["tol_ln"]))
    np.testing.assert_array_equal(r54, g["dopr54"])
    np.testing.assert_array_equal(r853, g["dop853"])
    assert [s853.accepted, s853.rejected, s853.rhs] == list(g["dop853_steps"])


def test_oracle_reproduces_committed_kepler_corpus(oracle):
    g = np.load(GOLDEN / "kepler_corpus.npz")
    kep = oracle.kepler(1.0)
    tol = float(g["tol_ln"])
    for i in range(len(g["y0"])):
        t = np.linspace(0.0, g["t_end"][i], 1000)
        r54, err, _, s54 = oracle.dopr54(kep, g["y0"][i], t, tol, tol)
        r853, _, s853 = oracle.dop853(kep, g["y0"][i], t, tol, tol)
        assert err == 0
        np.testing.assert_array_equal(r54[-1], g["dopr54_final"][i])
        np.testing.assert_array_equal(r853[-1], g["dop853_final"][i])
        assert [s54.accepted, s54.rejected] == list(g["dopr54_steps"][i])
        assert [s853.accepted, s853.rejected] == list(g["dop853_steps"][i])


def test_oracle_reproduces_committed_potential_batches(oracle):
    g = np.load(GOLDEN / "potential_batches.npz")
    for pname, pot in (("plummer", oracle.plummer(1.0, 1.0)), ("bovy", oracle.bovy())):
        for mname, m in (("dopr54", oracle.DOPR54), ("dop853", oracle.DOP853)):
            res = oracle.integrate_batch(m, pot, g[f"{pname}_y0"], ts=g["ts"], rtol=1e-10,
                                         atol=1e-10, threads=4)
            np.testing.assert_array_equal(res["out"][-1], g[f"{pname}_{mname}_final"])
            np.testing.assert_array_equal(res["accepted"], g[f"{pname}_{mname}_accepted"])


def test_reference_orbit_closes_after_one_period(oracle):
    # tests/test_python_smoke.py:159-173: circular unit Kepler orbit, one
    # period, tolerance 1e-12, closure within 2e-10.
    yo = np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0])
    t = np.linspace(0.0, 2.0 * np.pi, 100)
    tol = float(np.log(1e-12))
    for fn in (oracle.dopr54, oracle.dop853):
        res = fn(oracle.kepler(1.0), yo, t, tol, tol)[0]
        np.testing.assert_allclose(res[-1], yo, rtol=0.0, atol=2e-10)


def test_dopr54_plunge_sets_odd_error_code(oracle):
    # tests/test_python_errors.py:8-37: a radial plunge at 1e-13 forces the
    # minimum step and returns an odd error code.
    yo = np.array([1.0, 0.0, 0.0, -3.0, 0.0, 0.0])
    t = np.linspace(0.0, 5.0, 64)
    tol = float(np.log(1e-13))
    _, err, status, _ = oracle.dopr54(oracle.kepler(1.0), yo, t, tol, tol, max_steps=2_000_000)
    assert err % 2 == 1


def test_max_steps_cap_ends_integration(oracle):
    yo = np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0])
    t = np.linspace(0.0, 100.0, 11)
    tol = float(np.log(1e-12))
    _, status, stats = oracle.dop853(oracle.kepler(1.0), yo, t, tol, tol, max_steps=10)
    assert status == 2 and stats.accepted + stats.rejected == 10


# --- force properties (shared/tests/plummer_potential_tests.rs) ---------

def _norm(v):
    return float(np.sqrt(sum(x * x for x in v)))


def test_plummer_force_properties(oracle):
    p = oracle.plummer(1.0, 0.6)
    assert oracle.force(p, 0.0, 0.0, 0.0) == (0.0, 0.0, 0.0) or all(
        abs(v) <= 1e-15 for v in oracle.force(p, 0.0, 0.0, 0.0))
    assert _norm(oracle.force(p, 1e-6, -1e-6, 2e-6)) < 1.0
    p = oracle.plummer(1.0, 0.5)
    f, g = oracle.force(p, 0.7, -0.3, 1.1), oracle.force(p, -0.7, 0.3, -1.1)
    np.testing.assert_allclose(f, -np.array(g), atol=1e-12)
    p = oracle.plummer(1.0, 0.4)
    r = np.array([0.8, 1.2, -0.5])
    f = np.array(oracle.force(p, *r))
    assert abs(f @ r / (_norm(f) * _norm(r)) + 1.0) < 1e-12
    p = oracle.plummer(1.0, 0.5)
    for r1, r2 in [((1.0, 0.0, 0.0), (0.0, 1.0, 0.0)), ((2.0, -1.0, 0.5), (-1.0, 2.0, 0.5))]:
        s = _norm(r1)
        r2s = np.array(r2) * s / _norm(r2)
        assert abs(_norm(oracle.force(p, *r1)) / _norm(oracle.force(p, *r2s)) - 1) < 1e-12
    d = np.array([0.6, -0.2, 0.77])
    d /= _norm(d)
    rp = 0.5 / np.sqrt(2.0)
    mags = [_norm(oracle.force(p, *(d * r))) for r in (0.2 * rp, 0.5 * rp, 0.9 * rp)]
    assert mags[0] < mags[1] < mags[2]
    mags = [_norm(oracle.force(p, *(d * r))) for r in (1.1 * rp, 2.0 * rp, 4.0 * rp)]
    assert mags[0] > mags[1] > mags[2]
    f1 = np.array(oracle.force(oracle.plummer(1.0, 0.5), 0.3, -1.7, 2.2))
    f3 = np.array(oracle.force(oracle.plummer(3.0, 0.5), 0.3, -1.7, 2.2))
    np.testing.assert_allclose(f3, 3.0 * f1, atol=1e-12)
    p = oracle.plummer(2.0, 0.4)
    r1 = np.array([50.0 / 3.0, 100.0 / 3.0, 0.0])
    ratio = _norm(oracle.force(p, *(2.5 * r1))) / _norm(oracle.force(p, *r1))
    assert abs(ratio / (1 / 6.25) - 1) < 3e-3


def test_bovy_normalisation(oracle):
    # Radial forces at R = 1, z = 0: bulge 0.05, disk 0.60, halo 0.35 (vc = 1).
    b = oracle.bovy()
    fx, fy, fz = oracle.force(b, 1.0, 0.0, 0.0)
    assert abs(fx + 1.0) < 1e-9 and fy == 0.0 and fz == 0.0


def test_lower_gamma_matches_scipy(oracle):
    from scipy.special import gamma, gammainc

    lib = oracle.lib()
    s = 0.6
    gs = float(gamma(s))
    for x in np.concatenate([np.geomspace(1e-8, 1.59, 40), np.geomspace(1.61, 800.0, 40)]):
        got = lib.oracle_lower_gamma(s, float(x), gs)
        want = float(gammainc(s, x) * gs)
        assert abs(got - want) <= 4e-15 * want, (x, got, want)


def test_grid_sample_matches_output_grid(oracle):
    # shared/src/config.rs:69-85
    assert [oracle.grid_sample(0.0, 1.0, 3, i) for i in range(3)] == [0.0, 0.5, 1.0]
    assert [oracle.grid_sample(1.0, -1.0, 3, i) for i in range(3)] == [1.0, 0.0, -1.0]


def test_origin_table_matches_samples_and_forces(oracle):
    """Each quintic segment passes through its end samples with their
    velocities and the source force's accelerations."""
    sat = np.array([[1.2, 0.0, 0.05, 0.0, 1.0, 0.02]])
    ts = np.linspace(0.0, 4.0, 9)
    traj = oracle.integrate_batch(1, oracle.bovy(), sat, ts=ts, rtol=1e-12, atol=1e-12)["out"]
    dt = ts[1] - ts[0]
    table = oracle.origin_table(oracle.bovy(), traj, ts[0], dt)
    assert table.shape == (8, 1, 18)
    for k in range(8):
        for axis in range(3):
            c = table[k, 0, 6 * axis: 6 * axis + 6]
            x0, v0 = traj[k, 0, axis], traj[k, 0, 3 + axis]
            x1, v1 = traj[k + 1, 0, axis], traj[k + 1, 0, 3 + axis]
            a0 = oracle.force(oracle.bovy(), *traj[k, 0, :3])[axis]
            a1 = oracle.force(oracle.bovy(), *traj[k + 1, 0, :3])[axis]
            assert c[0] == x0
            assert abs(c[1] / dt - v0) < 1e-15 * max(1, abs(v0))
            assert abs(2 * c[2] / dt ** 2 - a0) < 1e-14 * max(1, abs(a0))
            assert abs(c.sum() - x1) < 1e-14
            assert abs((c[1] + 2 * c[2] + 3 * c[3] + 4 * c[4] + 5 * c[5]) / dt - v1) < 1e-13
            assert abs((2 * c[2] + 6 * c[3] + 12 * c[4] + 20 * c[5]) / dt ** 2 - a1) < 1e-11


def test_single_part_model_is_the_potential(oracle):
    y0 = np.array([[1.0, 0.1, 0.05, 0.0, 0.9, 0.02]])
    ts = np.linspace(0.0, 5.0, 11)
    for pot in (oracle.plummer(1.0, 1.0), oracle.bovy(), oracle.kepler(1.0)):
        for method in (0, 1):
            a = oracle.integrate_batch(method, pot, y0, ts=ts, rtol=1e-10, atol=1e-10)["out"]
            b = oracle.integrate_batch(method, oracle.model([pot]), y0, ts=ts, rtol=1e-10, atol=1e-10)["out"]
            np.testing.assert_array_equal(a, b)


def test_arbitrary_output_times(oracle):
    """DOPR54 with arbitrary_times lands every interval on the requested time:
    on a logarithmic grid it agrees with DOP853's dense output to the
    integration tolerance, and on a uniform grid with the galpy semantics."""
    y0 = np.array([[1.0, 0.1, 0.05, 0.0, 0.9, 0.02], [0.7, -0.3, 0.0, 0.4, 0.8, 0.1]])
    ts = np.concatenate([[0.0], np.logspace(-2, 1, 12)])
    a = oracle.integrate_batch(0, oracle.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-12, atol=1e-12,
                               arbitrary_times=True)["out"]
    b = oracle.integrate_batch(1, oracle.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-12, atol=1e-12)["out"]
    assert np.abs(a - b).max() < 1e-9
    u = np.linspace(0.0, 10.0, 11)
    c = oracle.integrate_batch(0, oracle.plummer(1.0, 1.0), y0, ts=u, rtol=1e-12, atol=1e-12,
                               arbitrary_times=True)["out"]
    d = oracle.integrate_batch(0, oracle.plummer(1.0, 1.0), y0, ts=u, rtol=1e-12, atol=1e-12)["out"]
    assert np.abs(c - d).max() < 1e-10
