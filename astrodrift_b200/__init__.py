"""B200-native batched Dormand-Prince test-particle integration.

The public API mirrors lbparticles/astrodrift's ``drift`` package
(python/drift/__init__.py): build potentials and containers, register force
edges with ``Config.add(node, *requires)`` and integrate with
``Config.run()``.  Integration runs on the GPU through the sm_100a kernels of
``libdrift_b200.so``; importing works without a GPU, integrating does not.

    import astrodrift_b200 as dft
    kp = dft.Potential.kepler(1.0)
    sim = dft.Config(method=dft.Method.DOP853, ts=(0.0, 10.0, 101))
    sim.add(dft.test_particles(istate), dft.background(kp))
    trajectory, _ = sim.run()            # (101, N, 6) float64
"""

from __future__ import annotations

from .selectors import Engine, Implementation, Method

try:
    from . import _drift
except ImportError as exc:  # pragma: no cover - exercised only without a build
    raise ImportError(
        "astrodrift_b200's native extension is not built; run "
        "`python -m astrodrift_b200.build` (needs nvcc for sm_100a)"
    ) from exc

Potential = _drift.Potential
Container = _drift.Container
Config = _drift.Config
particles = _drift.particles
test_particles = _drift.test_particles
background = _drift.background
DriftError = _drift.DriftError
IntegrationError = _drift.IntegrationError

# Exceptions are part of the package's public surface.
DriftError.__module__ = __name__
IntegrationError.__module__ = __name__

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
]
