"""The potentials used for energy-drift reports are the antiderivatives of
the integrated forces: -grad Phi (central differences) equals the oracle's
force at random points, for every potential kind."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.energy import potential_energy


@pytest.mark.parametrize("kind", ["kepler", "plummer", "bovy"])
def test_minus_gradient_of_phi_is_the_force(oracle, kind):
    pot = {"kepler": capi.kepler(1.0), "plummer": capi.plummer(1.3, 0.7), "bovy": capi.bovy()}[kind]
    opot = {"kepler": oracle.kepler(1.0), "plummer": oracle.plummer(1.3, 0.7), "bovy": oracle.bovy()}[kind]
    rng = np.random.default_rng(0)
    pts = rng.uniform(-3.0, 3.0, (50, 3))
    pts = pts[np.linalg.norm(pts[:, :2], axis=1) > 0.05]
    h = 1e-5
    for p in pts:
        grad = np.empty(3)
        for c in range(3):
            e = np.zeros(3)
            e[c] = h
            grad[c] = (potential_energy(pot, (p + e)[None])[0] - potential_energy(pot, (p - e)[None])[0]) / (2 * h)
        f = np.array(oracle.force(opot, *p))
        assert np.abs(-grad - f).max() <= 1e-7 * max(1.0, np.abs(f).max()), (p, -grad, f)


def test_angular_momentum_drift_measures_the_conserved_part():
    from astrodrift_b200 import capi
    from astrodrift_b200.energy import angular_momentum_drift

    rng = np.random.default_rng(4)
    first = rng.normal(size=(1000, 6))
    # a rotation about z conserves L_z and |L| but turns L: no drift for Bovy
    # (L_z), and for a spherical potential the vector L changes
    c, s = np.cos(0.3), np.sin(0.3)
    rot = np.array([[c, -s, 0], [s, c, 0], [0, 0, 1.0]])
    last = np.hstack([first[:, :3] @ rot.T, first[:, 3:] @ rot.T])
    bovy = angular_momentum_drift(capi.bovy(), first, last)
    assert bovy["quantity"] == "L_z" and bovy["max"] < 1e-13
    plummer = angular_momentum_drift(capi.plummer(), first, last)
    assert plummer["quantity"] == "L" and plummer["median"] > 0.1
    # scaling the velocities by (1 + 1e-9) drifts L by 1e-9 in both measures
    scaled = np.hstack([first[:, :3], first[:, 3:] * (1 + 1e-9)])
    got = angular_momentum_drift(capi.plummer(), first, scaled)
    assert abs(got["median"] - 1e-9) < 1e-14 and got["particles"] == 1000
