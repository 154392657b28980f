"""Potentials Phi of the integrated forces, for energy-conservation checks.

The reference has no potential evaluation (shared/src/potential.rs:41-44
declares only `force`), so these are derived from the forces in
drift_potentials.cuh with Phi(inf) = 0:
  Kepler:  -amp / r
  Plummer: -amp / sqrt(r^2 + b^2)
  disk:    -amp / sqrt(R^2 + (a + sqrt(z^2 + b^2))^2)           (Miyamoto-Nagai)
  halo:    -amp ln(1 + r/a) / r                                  (NFW)
  bulge:   -k (gamma(s, u) / r + Gamma(s - 1/2, u) / rc),  u = r^2 / rc^2
           (F = -k gamma(s, u) / r^2 integrated from r to infinity; Gamma(., u)
           is the upper incomplete gamma function).
Host-side numpy; used to report the relative energy drift |E(t)/E(0) - 1|.
"""

from __future__ import annotations

import numpy as np

from . import capi


def potential_energy(pot: capi.DriftPotential, xyz: np.ndarray) -> np.ndarray:
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    r2 = x * x + y * y + z * z
    if pot.kind in (capi.POT_KEPLER, capi.POT_KEPLER_CARTESIAN):
        return -pot.amp / np.sqrt(r2)
    if pot.kind == capi.POT_PLUMMER:
        return -pot.amp / np.sqrt(r2 + pot.b * pot.b)
    from scipy.special import gamma, gammainc, gammaincc

    r = np.sqrt(r2)
    R2 = x * x + y * y
    disk = -pot.mn_amp / np.sqrt(R2 + (pot.mn_a + np.sqrt(z * z + pot.mn_b * pot.mn_b)) ** 2)
    halo = -pot.nfw_amp * np.log1p(r / pot.nfw_a) / r
    s = 1.5 - 0.5 * pot.bulge_alpha
    u = r2 / (pot.bulge_rc * pot.bulge_rc)
    bulge = -pot.bulge_k * (gamma(s) * gammainc(s, u) / r + gamma(s - 0.5) * gammaincc(s - 0.5, u) / pot.bulge_rc)
    return bulge + disk + halo


def energy(pot: capi.DriftPotential, y: np.ndarray) -> np.ndarray:
    """Specific energy of states y (..., 6)."""
    return 0.5 * (y[..., 3:] ** 2).sum(-1) + potential_energy(pot, y[..., :3])


def drift_summary(pot: capi.DriftPotential, first: np.ndarray, last: np.ndarray) -> dict:
    """Median / p99 / max of |E(last)/E(first) - 1| over particles (finite rows)."""
    de = np.abs(energy(pot, last) / energy(pot, first) - 1.0)
    de = de[np.isfinite(de)]
    return {"median": float(np.median(de)), "p99": float(np.quantile(de, 0.99)), "max": float(de.max()),
            "particles": int(de.size)}


def angular_momentum_drift(pot: capi.DriftPotential, first: np.ndarray, last: np.ndarray) -> dict:
    """Median / p99 / max over particles (finite rows) of the drift of the
    conserved angular momentum between states ``first`` and ``last`` (N, 6):
    the full vector L = x x v for the spherical potentials (Kepler, Plummer),
    |L(last) - L(first)| / |L(first)|; only L_z for the axisymmetric Bovy
    potential, |L_z(last) - L_z(first)| / |L(first)| (normalised by |L| so
    that orbits with L_z near 0 stay meaningful)."""
    l0 = np.cross(first[:, :3], first[:, 3:])
    l1 = np.cross(last[:, :3], last[:, 3:])
    norm = np.linalg.norm(l0, axis=1)
    if pot.kind == capi.POT_BOVY:
        d, quantity = np.abs(l1[:, 2] - l0[:, 2]) / norm, "L_z"
    else:
        d, quantity = np.linalg.norm(l1 - l0, axis=1) / norm, "L"
    d = d[np.isfinite(d)]
    return {"quantity": quantity, "median": float(np.median(d)), "p99": float(np.quantile(d, 0.99)),
            "max": float(d.max()), "particles": int(d.size)}
