"""``drift.drift_rs``: the native module under the reference's name.

The reference's ``drift.drift_rs`` is its compiled extension
(python/drift/drift_rs.pyi).  Here it is astrodrift_b200's pybind11 host module,
``astrodrift_b200._drift``, which serves the same names.
"""

from __future__ import annotations

import astrodrift_b200

_native = astrodrift_b200._load_native()
_native.DriftError.__module__ = "drift"
_native.IntegrationError.__module__ = "drift"

Potential = _native.Potential
Container = _native.Container
Config = _native.Config
particles = _native.particles
test_particles = _native.test_particles
background = _native.background
DriftError = _native.DriftError
IntegrationError = _native.IntegrationError

__all__ = [
    "Potential",
    "Container",
    "Config",
    "particles",
    "test_particles",
    "background",
    "DriftError",
    "IntegrationError",
]
