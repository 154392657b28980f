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

# Names served by the pybind11 host module.  It is loaded on first use, so
# importing a pure-Python submodule (workloads, sharding) maps no native code.
_NATIVE_NAMES = (
    "Potential",
    "Container",
    "Config",
    "particles",
    "test_particles",
    "background",
    "DriftError",
    "IntegrationError",
)


def _load_native():
    try:
        from . import _drift
    except ImportError as exc:
        raise ImportError(
            "astrodrift_b200's native extension is not built; run "
            "`python -m astrodrift_b200.build` (needs nvcc for sm_100a)"
        ) from exc
    # Exceptions are part of the package's public surface.
    if _drift.DriftError.__module__ != "drift":
        _drift.DriftError.__module__ = __name__
        _drift.IntegrationError.__module__ = __name__
    for name in _NATIVE_NAMES:
        globals()[name] = getattr(_drift, name)
    return _drift


def __getattr__(name: str):
    if name in _NATIVE_NAMES:
        _load_native()
        return globals()[name]
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def __dir__():
    return sorted(set(globals()) | set(_NATIVE_NAMES))


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
