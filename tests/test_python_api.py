"""The drift Python surface on CPU (no device work).

Follows the reference's Python tests (tests/test_python_containers.py,
test_python_selectors.py, test_python_time_grids.py, test_python_errors.py
and the host-only parts of test_python_smoke.py) with this package's
deliberate differences: particle and output-time caps are lifted
(2^30 particles, 2^24 times) and the engine is the GPU.
"""

from __future__ import annotations

import warnings
from collections.abc import Callable
from enum import StrEnum
from typing import Any, cast

import numpy as np
import pytest

import astrodrift_b200 as dft
from astrodrift_b200 import _drift

INITIAL_STATE = np.zeros((1, 6), dtype=np.float64)
MAX_MODEL_COMPONENTS = 11
MAX_OUTPUT_TIMES = _drift.MAX_OUTPUT_TIMES


# --- containers (tests/test_python_containers.py) -------------------------

@pytest.mark.parametrize(
    ("factory", "args"),
    ((dft.Potential.kepler, ()), (dft.Potential.plummer, ()), (dft.Potential.plummer, (1.0,))),
)
def test_potential_parameters_are_required(factory: Callable[..., Any], args: tuple) -> None:
    with pytest.raises(TypeError):
        factory(*args)


@pytest.mark.parametrize("potential", (dft.Potential.kepler(1.0), dft.Potential.plummer(1.0, 0.5)))
def test_supported_potentials_can_be_attached_to_particles(potential) -> None:
    assert isinstance(dft.particles(potential, INITIAL_STATE), dft.Container)


@pytest.mark.parametrize(
    ("potential", "expected"),
    (
        (dft.Potential.kepler(2.5), "Potential.kepler(amp=2.5)"),
        (dft.Potential.plummer(3.5, 0.25), "Potential.plummer(amp=3.5, radius=0.25)"),
        (dft.Potential.bovy(), "Potential.bovy()"),
    ),
)
def test_potential_reprs_use_public_constructors(potential, expected) -> None:
    assert repr(potential) == expected


def test_container_reprs_describe_only_public_properties() -> None:
    potential = dft.Potential.kepler(1.0)
    assert repr(dft.background(potential)) == (
        "Container(kind='background', potential=Potential.kepler(amp=1.0))")
    assert repr(dft.test_particles(np.zeros((2, 6)))) == (
        "Container(kind='test_particles', num_particles=2)")
    assert repr(dft.particles(potential, INITIAL_STATE)) == (
        "Container(kind='particles', num_particles=1, potential=Potential.kepler(amp=1.0))")


@pytest.mark.parametrize("state", (np.zeros((2, 6)), np.zeros(12)))
def test_initial_state_accepts_particle_records(state) -> None:
    assert dft.test_particles(state).num_particles == 2


@pytest.mark.parametrize("state", (np.zeros(7), np.zeros((2, 5)), np.zeros((1, 2, 3))))
def test_initial_state_rejects_partial_or_misdimensioned_records(state) -> None:
    with pytest.raises(ValueError, match=r"shape \(N, 6\)"):
        dft.test_particles(state)


@pytest.mark.parametrize("state", (np.empty((0, 6)), np.empty(0)))
def test_initial_state_rejects_empty_particle_groups(state) -> None:
    with pytest.raises(ValueError, match="at least one particle"):
        dft.test_particles(state)


def test_particle_capacity_is_lifted_beyond_the_reference_cap() -> None:
    # The reference caps a container at 1000 particles (shared/src/lib.rs:25).
    assert dft.test_particles(np.zeros((4096, 6))).num_particles == 4096
    assert _drift.MAX_PARTICLES == 1 << 30


@pytest.mark.parametrize("value", (np.nan, np.inf, -np.inf))
def test_initial_state_rejects_non_finite_values(value) -> None:
    state = INITIAL_STATE.copy()
    state[0, 0] = value
    with pytest.raises(ValueError, match="must be finite"):
        dft.test_particles(state)


def test_container_particle_counts_are_read_only() -> None:
    particles = dft.test_particles(np.zeros((2, 6)))
    background = dft.background(dft.Potential.kepler(1.0))
    assert particles.num_particles == 2
    assert background.num_particles is None
    for container in (particles, background):
        with pytest.raises(AttributeError):
            setattr(container, "num_particles", 3)


def test_unsupported_potential_cannot_be_attached_to_particles() -> None:
    with pytest.raises(NotImplementedError, match="only Kepler and Plummer"):
        dft.particles(dft.Potential.bovy(), INITIAL_STATE)


def test_container_creation_is_not_limited_by_process_lifetime() -> None:
    potential = dft.Potential.kepler(1.0)
    for _ in range(2 * MAX_MODEL_COMPONENTS):
        dft.background(potential)


def test_add_rejects_more_containers_than_one_model_can_hold() -> None:
    background = dft.background(dft.Potential.kepler(1.0))
    state = np.array([[1.0, 0.0, 0.0, 0.0, 1.0, 0.0]])
    groups = [dft.test_particles(state) for _ in range(MAX_MODEL_COMPONENTS)]
    config = dft.Config()
    for group in groups[:-1]:
        config.add(group, background)
    with pytest.raises(ValueError, match="at most 11"):
        config.add(groups[-1], background)
    assert "containers=11" in config.info()


def test_per_particle_end_times_are_validated() -> None:
    state = np.zeros((3, 6))
    assert dft.test_particles(state, t_end=np.array([1.0, 2.0, 3.0])).num_particles == 3
    with pytest.raises(ValueError, match="one end time per particle"):
        dft.test_particles(state, t_end=np.array([1.0, 2.0]))
    with pytest.raises(ValueError, match="finite"):
        dft.test_particles(state, t_end=np.array([1.0, np.nan, 3.0]))


# --- selectors (tests/test_python_selectors.py) ---------------------------

@pytest.mark.parametrize(
    ("selector", "value", "expected"),
    ((dft.Engine, "CPU", dft.Engine.CPU), (dft.Method, "DOP853", dft.Method.DOP853),
     (dft.Implementation, "GALPY", dft.Implementation.GALPY)),
)
def test_selectors_support_value_construction(selector: type[StrEnum], value, expected) -> None:
    assert selector(value) is expected


@pytest.mark.parametrize("keyword", ({"engine": "GPU"}, {"method": "DOPR54"}, {"implementation": "GALPY"}))
def test_config_rejects_raw_strings(keyword) -> None:
    config = cast(Any, dft.Config)
    with pytest.raises(TypeError, match="expected a drift.* member"):
        config(**keyword)


# --- time grids (tests/test_python_time_grids.py) -------------------------

@pytest.mark.parametrize(
    "ts",
    ((0.0, 1.0, 2), (1.0, -1.0, 7), np.linspace(0.0, 1.0, 7), np.linspace(0.0, 1.0e-12, 7),
     np.linspace(1.0e12, 1.0e12 + 1.0e6, 7), np.linspace(1.0, -1.0, 7), (0.0, 1.0, 1025),
     np.linspace(0.0, 1.0, 1025)),
)
def test_valid_time_grids_are_accepted(ts) -> None:
    dft.Config(ts=ts)


def test_read_only_time_array_is_accepted() -> None:
    times = np.linspace(0.0, 1.0, 7)
    times.flags.writeable = False
    dft.Config(ts=times)


@pytest.mark.parametrize(
    ("ts", "message"),
    (
        ([0.0, 1.0e-12, 3.0e-12], "uniformly spaced"),
        ([0.0, 0.25, 0.500_000_000_001, 0.75, 1.0], "uniformly spaced"),
        (np.logspace(0.0, 1.0, 7), "uniformly spaced"),
        ([0.0, 0.5, 0.5, 1.0], "strictly increasing or strictly decreasing"),
        ([0.0, 0.5, 0.25, 1.0], "strictly increasing or strictly decreasing"),
        ((float("nan"), 1.0, 3), "finite"),
        ([0.0, float("inf")], "finite"),
        ((0.0, 1.0, 1), f"between 2 and {MAX_OUTPUT_TIMES}"),
        ((0.0, 1.0, MAX_OUTPUT_TIMES + 1), f"between 2 and {MAX_OUTPUT_TIMES}"),
        ([0.0], f"between 2 and {MAX_OUTPUT_TIMES}"),
        ((1.0, 1.0, 2), "non-zero"),
        ([1.0, 1.0], "non-zero"),
        (np.linspace(0.0, 1.0, 7)[::2], "contiguous"),
    ),
)
def test_invalid_time_grids_are_rejected(ts, message) -> None:
    with pytest.raises(ValueError, match=message):
        dft.Config(ts=ts)


# --- errors (tests/test_python_errors.py) ---------------------------------

def test_exception_hierarchy() -> None:
    assert issubclass(dft.IntegrationError, dft.DriftError)
    assert issubclass(dft.DriftError, RuntimeError)
    assert dft.DriftError.__module__ == "astrodrift_b200"
    assert dft.IntegrationError.__module__ == "astrodrift_b200"


def test_unsupported_configuration_uses_not_implemented_error() -> None:
    with pytest.raises(NotImplementedError) as raised:
        dft.Config(method=dft.Method.DOPR54, implementation=dft.Implementation.SCIPY)
    assert not isinstance(raised.value, dft.DriftError)


@pytest.mark.parametrize("engine", dft.Engine)
@pytest.mark.parametrize("method", (dft.Method.DOPR54, dft.Method.DOP853))
@pytest.mark.parametrize("implementation", (dft.Implementation.SCIPY, dft.Implementation.DRIFT))
def test_unimplemented_integrator_is_rejected_before_execution(engine, method, implementation) -> None:
    message = rf"{engine.value} \+ {implementation.value} {method.value} is not implemented"
    with pytest.raises(NotImplementedError, match=message):
        dft.Config(engine=engine, method=method, implementation=implementation)


def test_cpu_engine_is_not_a_product_path() -> None:
    # The reference's CPU engine is its host port; this package keeps that port
    # as the test oracle and integrates on the GPU only.
    with pytest.raises(NotImplementedError, match=r"CPU \+ GALPY DOP853 is not implemented"):
        dft.Config(engine=dft.Engine.CPU, method=dft.Method.DOP853)


def test_input_validation_still_raises_plain_value_error() -> None:
    with pytest.raises(ValueError) as raised:
        dft.Config(tolerance=-1.0)
    assert not isinstance(raised.value, dft.DriftError)


@pytest.mark.parametrize("tolerance", (0.0, -1.0, float("nan"), float("inf"), (1.0e-12, 0.0)))
def test_invalid_tolerances_are_rejected(tolerance) -> None:
    with pytest.raises(ValueError, match="finite and greater than zero"):
        dft.Config(tolerance=tolerance)


# --- configuration and graph (tests/test_python_smoke.py, host-only) ------

def _model():
    kp = dft.Potential.kepler(1.0)
    gal = dft.background(kp)
    gmc = dft.particles(kp, np.tile([1.0, 0.0, 0.0, 0.0, 1.0, 0.0], (20, 1)))
    iso = dft.test_particles(np.tile([-1.0, 0.0, 0.0, 0.0, -1.0, 0.0], (20, 1)))
    return gal, gmc, iso


def test_empty_config_returns_no_results() -> None:
    assert dft.Config().run() == []


def test_extension_reports_cuda_compiler() -> None:
    assert _drift._cuda_compiler == "nvcc-sm_100a"


def test_config_construction_does_not_print(capsys) -> None:
    dft.Config()
    captured = capsys.readouterr()
    assert captured.out == "" and captured.err == ""


def test_info_and_repr_return_a_bounded_summary_without_printing(capsys) -> None:
    gal, gmc, _ = _model()
    sim = dft.Config()
    sim.add(gmc, gal)
    capsys.readouterr()
    summary = sim.info()
    assert capsys.readouterr().out == ""
    assert repr(sim) == summary
    assert summary.startswith("Config(engine=GPU, method=DOPR54")
    assert "implementation=GALPY" in summary
    assert "containers=2" in summary and "dependencies=1" in summary
    assert len(summary) < 300


def test_particle_group_requires_a_registered_force_source() -> None:
    _, gmc, iso = _model()
    sim = dft.Config()
    sim.add(iso, gmc)
    with pytest.raises(ValueError, match="registered with add"):
        sim.run()


def test_add_rejects_empty_and_cyclic_dependencies() -> None:
    gal, gmc, iso = _model()
    sim = dft.Config()
    with pytest.raises(ValueError, match="at least one dependency"):
        sim.add(iso)
    with pytest.raises(ValueError, match="cycle"):
        sim.add(iso, iso)
    sim.add(gmc, gal)
    sim.add(iso, gmc)
    with pytest.raises(ValueError, match="cycle"):
        sim.add(gal, iso)
    sim.add(gmc, gal, gal)  # duplicates are harmless
    assert "dependencies=2" in sim.info()


def test_dependency_alias_warns_at_the_call_site() -> None:
    gal, gmc, _ = _model()
    sim = dft.Config()
    with pytest.warns(DeprecationWarning, match="use Config.add") as caught:
        sim.dependency(gmc, gal)
    assert caught[0].filename == __file__


def test_run_without_a_device_fails_loudly() -> None:
    # On a machine without a CUDA device the GPU path raises; it never falls
    # back to a CPU integrator.
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    gal, gmc, _ = _model()
    sim = dft.Config()
    sim.add(gmc, gal)
    with pytest.raises(dft.DriftError, match="CUDA device"):
        sim.run()


def test_moving_sources_need_the_shared_output_grid() -> None:
    # A particle group with an attached potential is a moving force source;
    # its origin table follows the shared grid, so per-particle end times are
    # refused before any device work.
    kp = dft.Potential.kepler(1.0)
    gal = dft.background(kp)
    sat = dft.particles(dft.Potential.plummer(0.1, 0.05), np.array([[1.0, 0.0, 0.0, 0.0, 1.0, 0.0]]),
                        t_end=np.array([5.0]))
    stars = dft.test_particles(np.tile([-1.0, 0.0, 0.0, 0.0, -1.0, 0.0], (4, 1)))
    sim = dft.Config(ts=(0.0, 5.0, 11), attached_potentials=True)
    sim.add(sat, gal)
    sim.add(stars, gal, sat)
    with pytest.raises(NotImplementedError, match="shared output grid"):
        sim.run()


def test_a_stage_without_force_source_is_refused() -> None:
    _, gmc, iso = _model()
    sim = dft.Config()
    sim.add(gmc, iso)  # iso carries no potential; gmc has no background
    sim.add(iso, dft.background(dft.Potential.kepler(1.0)))
    with pytest.raises(NotImplementedError, match="no force source"):
        sim.run()


def test_arbitrary_times_are_accepted_only_when_asked() -> None:
    times = np.logspace(0.0, 1.0, 7)
    with pytest.raises(ValueError, match="uniformly spaced"):
        dft.Config(ts=times)
    dft.Config(ts=times, arbitrary_times=True)
    dft.Config(ts=[0.0, 0.1, 0.5, 2.0], arbitrary_times=True)
    with pytest.raises(ValueError, match="strictly increasing or strictly decreasing"):
        dft.Config(ts=[0.0, 1.0, 0.5], arbitrary_times=True)
    with pytest.raises(ValueError, match="finite"):
        dft.Config(ts=[0.0, float("nan"), 1.0], arbitrary_times=True)
