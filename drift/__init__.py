"""``drift``: the reference's import name for astrodrift_b200.

lbparticles/astrodrift is imported as ``import drift as dft`` with the native
module at ``drift.drift_rs`` (python/drift/__init__.py).  This package gives
astrodrift_b200 the same two names, so host code and tests written against the
reference import it unchanged:

    import drift as dft
    sim = dft.Config(method=dft.Method.DOP853, ts=(0.0, 10.0, 101))

Every name is the one ``astrodrift_b200`` exports (the same classes and
functions, not copies).  Importing ``drift`` names the exception classes
``drift.DriftError`` and ``drift.IntegrationError``, as the reference does.
"""

from __future__ import annotations

from astrodrift_b200.selectors import Engine, Implementation, Method

from . import drift_rs
from .drift_rs import (
    Config,
    Container,
    DriftError,
    IntegrationError,
    Potential,
    background,
    particles,
    test_particles,
)

__all__ = [
    "Potential",
    "Container",
    "Config",
    "Implementation",
    "Method",
    "Engine",
    "DriftError",
    "IntegrationError",
    "particles",
    "test_particles",
    "background",
    "drift_rs",
]
