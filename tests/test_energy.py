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
