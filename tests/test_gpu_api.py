"""The drift Python surface integrating on the GPU.

Follows the reference's tests/test_python_smoke.py (registration order,
time-major shapes, one-orbit closure at 2e-10), tests/test_python_errors.py
(a radial plunge raises IntegrationError with galpy's error code) and
tests/test_python_logging.py (logger names, message prefixes, levels, a
broken handler does not abort the run), with the GPU as the engine.
"""

from __future__ import annotations

import logging
import sys
from collections.abc import Iterator
from pathlib import Path

import numpy as np
import pytest

import astrodrift_b200 as dft

pytestmark = pytest.mark.gpu

N_PARTICLES = 20
SUPPORTED_METHODS = (dft.Method.DOPR54, dft.Method.DOP853)
GMC_INITIAL_STATE = np.tile(np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0]), (N_PARTICLES, 1))
ISO_INITIAL_STATE = np.tile(np.array([-1.0, 0.0, 0.0, 0.0, -1.0, 0.0]), (N_PARTICLES, 1))


def _make_model():
    kp = dft.Potential.kepler(1.0)
    gal = dft.background(kp)
    gmc = dft.particles(kp, GMC_INITIAL_STATE)
    iso = dft.test_particles(ISO_INITIAL_STATE)
    return gal, gmc, iso


def _run(method, **kw):
    gal, gmc, iso = _make_model()
    sim = dft.Config(engine=dft.Engine.GPU, method=method, implementation=dft.Implementation.GALPY, **kw)
    sim.add(gmc, gal)
    sim.add(iso, gmc, gal)
    return sim.run()


@pytest.fixture(scope="module")
def gpu_results(cuda_device):
    return {m: _run(m) for m in SUPPORTED_METHODS}


@pytest.mark.parametrize("method", SUPPORTED_METHODS)
def test_results_follow_registration_order(gpu_results, method) -> None:
    gmc_trajectory, background_result, iso_trajectory = gpu_results[method]
    assert isinstance(iso_trajectory, np.ndarray)
    assert background_result is None
    assert isinstance(gmc_trajectory, np.ndarray)


@pytest.mark.parametrize("method", SUPPORTED_METHODS)
def test_particle_results_are_time_major_trajectories(gpu_results, method) -> None:
    gmc, _, iso = gpu_results[method]
    for trajectory in (gmc, iso):
        assert trajectory.shape == (100, N_PARTICLES, 6)
        assert trajectory.dtype == np.float64


@pytest.mark.parametrize("method", SUPPORTED_METHODS)
def test_gpu_trajectories_are_accurate_over_one_orbit(gpu_results, method) -> None:
    gmc, _, iso = gpu_results[method]
    for trajectory, initial_state in ((iso, ISO_INITIAL_STATE), (gmc, GMC_INITIAL_STATE)):
        np.testing.assert_array_equal(trajectory[0], initial_state)
        assert not np.array_equal(trajectory[1], initial_state)
        np.testing.assert_allclose(trajectory[-1], initial_state, rtol=0.0, atol=2.0e-10)


@pytest.mark.parametrize("method", SUPPORTED_METHODS)
def test_gpu_results_agree_with_the_reference_cpu_algorithm(gpu_results, oracle, method) -> None:
    # tests/test_python_smoke.py:214-225 compares the CPU and GPU engines at
    # rtol = atol = 1e-12; here the CPU side is the oracle.
    gmc, _, iso = gpu_results[method]
    ts = np.linspace(0.0, 2.0 * np.pi, 100)
    for traj, y0 in ((gmc, GMC_INITIAL_STATE), (iso, ISO_INITIAL_STATE)):
        ref = oracle.integrate_batch(0 if method == dft.Method.DOPR54 else 1, oracle.kepler(1.0), y0,
                                     ts=ts, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(traj, ref["out"], rtol=1e-12, atol=1e-12)


def test_default_config_integrates_with_dopr54(gpu_results) -> None:
    default = _run(dft.Method.DOPR54)
    for a, b in zip(default, gpu_results[dft.Method.DOPR54]):
        if a is None:
            assert b is None
        else:
            np.testing.assert_array_equal(a, b)


def test_precision_and_schedule_options(cuda_device) -> None:
    base = _run(dft.Method.DOP853)
    plain = _run(dft.Method.DOP853, schedule="plain")
    fma = _run(dft.Method.DOP853, precision="fma")
    np.testing.assert_array_equal(plain[0], base[0])
    np.testing.assert_allclose(fma[0], base[0], rtol=0.0, atol=1e-10)


def test_run_stats_report_step_counts(cuda_device) -> None:
    gal, gmc, _ = _make_model()
    sim = dft.Config(method=dft.Method.DOP853)
    sim.add(gmc, gal)
    results, stats = sim.run(stats=True)
    assert stats[1] is None
    assert (stats[0]["accepted"] > 0).all() and (stats[0]["status"] == 0).all()
    n = len(stats[0]["accepted"])
    assert stats[0]["bytes_written"] == results[0].shape[0] * n * 6 * 8
    assert stats[0]["bytes_in"] >= n * 6 * 8 and stats[0]["seconds"] > 0


def test_plummer_and_bovy_backgrounds(cuda_device, oracle) -> None:
    rng = np.random.default_rng(5)
    y0 = np.hstack([rng.uniform(0.5, 2.0, (64, 3)), rng.uniform(-0.4, 0.4, (64, 3))])
    ts = (0.0, 10.0, 21)
    for pot, opot in ((dft.Potential.plummer(1.0, 1.0), oracle.plummer(1.0, 1.0)),
                      (dft.Potential.bovy(), oracle.bovy())):
        sim = dft.Config(method=dft.Method.DOP853, ts=ts, tolerance=1e-11)
        sim.add(dft.test_particles(y0), dft.background(pot))
        traj, _ = sim.run()
        ref = oracle.integrate_batch(1, opot, y0, ts=np.linspace(*ts[:2], ts[2]), rtol=1e-11, atol=1e-11)
        scale = np.abs(ref["out"]).max(axis=2, keepdims=True)
        assert (np.abs(traj - ref["out"]) / scale).max() < 1e-9


def test_per_particle_end_times(cuda_device, oracle) -> None:
    y0 = np.tile([1.0, 0.0, 0.1, 0.0, 1.0, 0.0], (4, 1))
    t_end = np.array([1.0, 2.0, 5.0, 10.0])
    sim = dft.Config(method=dft.Method.DOP853, ts=(0.0, 1.0, 11))
    sim.add(dft.test_particles(y0, t_end=t_end), dft.background(dft.Potential.plummer(1.0, 1.0)))
    traj, _ = sim.run()
    ref = oracle.integrate_batch(1, oracle.plummer(1.0, 1.0), y0, t0=0.0, t_end=t_end, nt=11,
                                 rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(traj, ref["out"], rtol=1e-9, atol=1e-12)


# --- errors (tests/test_python_errors.py) ---------------------------------

def test_failed_integration_raises_drift_integration_error(cuda_device) -> None:
    plunge = np.array([[1.0, 0.0, 0.0, -3.0, 0.0, 0.0]])
    sim = dft.Config(method=dft.Method.DOPR54, ts=(0.0, 5.0, 64), tolerance=(1.0e-13, 1.0e-13),
                     max_steps=2_000_000)
    sim.add(dft.test_particles(plunge), dft.background(dft.Potential.kepler(1.0)))
    with pytest.raises(dft.IntegrationError, match="error code|step limit") as raised:
        sim.run()
    assert isinstance(raised.value, dft.DriftError)
    assert isinstance(raised.value, RuntimeError)


# --- logging (tests/test_python_logging.py) -------------------------------

GPU_LOGGER_NAME = "drift.dispatch.gpu"
BACKEND_LOGGER_NAME = "drift.dispatch.gpu.b200"
LOG_STATE = np.tile(np.array([1.0, 0.0, 0.0, 0.0, 1.0, 0.0]), (50, 1))


def _log_config():
    sim = dft.Config(ts=(0.0, 2.0 * np.pi, 16))
    sim.add(dft.test_particles(LOG_STATE), dft.background(dft.Potential.kepler(1.0)))
    return sim


@pytest.fixture(autouse=False)
def restore_drift_logger() -> Iterator[None]:
    logger = logging.getLogger("drift")
    saved = (logger.level, logger.propagate, list(logger.handlers))
    try:
        yield
    finally:
        logger.setLevel(saved[0])
        logger.propagate = saved[1]
        logger.handlers[:] = saved[2]


def test_gpu_run_emits_info_records_on_the_drift_logger(cuda_device, caplog, restore_drift_logger) -> None:
    with caplog.at_level(logging.INFO, logger="drift"):
        _log_config().run()
    records = [r for r in caplog.records if r.name == GPU_LOGGER_NAME]
    messages = [r.getMessage() for r in records]
    assert any(m.startswith("GPU integration starting") for m in messages)
    assert any(m.startswith("GPU integration finished") for m in messages)
    assert all(r.levelno == logging.INFO for r in records)
    assert all(r.filename == "gpu_dispatch.cpp" for r in records)


def test_gpu_debug_records_include_dispatch_and_backend_phases(cuda_device, caplog,
                                                               restore_drift_logger) -> None:
    with caplog.at_level(logging.DEBUG, logger="drift"):
        _log_config().run()
    dispatch = [r.getMessage() for r in caplog.records if r.name == GPU_LOGGER_NAME]
    assert any(m.startswith("launching GALPY DOPR54 kernel") for m in dispatch)
    assert any(m.startswith("stage 1: dispatching") for m in dispatch)
    assert any(m.startswith("stage 1: 50 particles finished") for m in dispatch)
    backend = [r.getMessage() for r in caplog.records if r.name == BACKEND_LOGGER_NAME]
    assert any("bytes of host data to the device" in m for m in backend)
    assert any("result bytes to the host" in m for m in backend)


def test_standard_python_levels_can_be_reconfigured(cuda_device, caplog, restore_drift_logger) -> None:
    caplog.clear()
    with caplog.at_level(logging.WARNING, logger="drift"):
        _log_config().run()
    assert [r for r in caplog.records if r.name == GPU_LOGGER_NAME] == []


@pytest.mark.filterwarnings("ignore::pytest.PytestUnraisableExceptionWarning")
def test_broken_handler_does_not_abort_integration(cuda_device, restore_drift_logger) -> None:
    class BrokenHandler(logging.Handler):
        def emit(self, record):
            raise RuntimeError("handler failed")

    logger = logging.getLogger("drift")
    logger.handlers[:] = [BrokenHandler()]
    logger.propagate = False
    logger.setLevel(logging.INFO)
    trajectory, _ = _log_config().run()
    assert trajectory.shape == (16, 50, 6)


@pytest.mark.parametrize("method", SUPPORTED_METHODS)
def test_attached_potentials_move_with_their_group(cuda_device, oracle, method) -> None:
    """Config(attached_potentials=True): stars feel the Bovy background plus
    the Plummer potentials carried by two satellites, placed along the
    satellites' own trajectories (integrated in the stage before).  The
    oracle repeats the chain: satellites, origin table, stars."""
    sat_state = np.array([[1.2, 0.0, 0.05, 0.0, 1.0, 0.02], [0.0, -1.6, 0.0, 0.95, 0.0, 0.0]])
    rng = np.random.default_rng(9)
    stars_state = sat_state[0] + np.hstack([rng.normal(0, 0.05, (40, 3)), rng.normal(0, 0.05, (40, 3))])
    gal = dft.background(dft.Potential.bovy())
    sats = dft.particles(dft.Potential.plummer(0.02, 0.05), sat_state)
    stars = dft.test_particles(stars_state)
    sim = dft.Config(method=method, ts=(0.0, 8.0, 41), tolerance=1e-10, attached_potentials=True)
    sim.add(sats, gal)
    sim.add(stars, gal, sats)
    sat_traj, background_result, star_traj = sim.run()
    assert background_result is None

    ts = np.array([oracle.grid_sample(0.0, 8.0, 41, k) for k in range(41)])
    om = 0 if method == dft.Method.DOPR54 else 1
    sat_ref = oracle.integrate_batch(om, oracle.bovy(), sat_state, ts=ts, rtol=1e-10, atol=1e-10)["out"]
    assert np.abs(sat_traj - sat_ref).max() < 1e-9
    table = oracle.origin_table(oracle.bovy(), sat_traj, 0.0, 8.0 / 40)
    omodel = oracle.model([oracle.bovy()], [(oracle.POT_PLUMMER, 0.02, 0.05, 0, 2)], origins=table,
                          t0=0.0, dt=8.0 / 40)
    ref = oracle.integrate_batch(om, omodel, stars_state, ts=ts, rtol=1e-10, atol=1e-10)["out"]
    scale = np.abs(ref).max(axis=2)
    assert (np.abs(star_traj - ref).max(axis=2) / scale).max() < 1e-9

    # without the flag the satellites exert no force (the reference's behaviour)
    sim2 = dft.Config(method=method, ts=(0.0, 8.0, 41), tolerance=1e-10)
    sats2 = dft.particles(dft.Potential.plummer(0.02, 0.05), sat_state)
    stars2 = dft.test_particles(stars_state)
    sim2.add(sats2, gal)
    sim2.add(stars2, gal, sats2)
    _, _, star_plain = sim2.run()
    plain_ref = oracle.integrate_batch(om, oracle.bovy(), stars_state, ts=ts, rtol=1e-10, atol=1e-10)["out"]
    assert np.abs(star_plain - plain_ref).max() < 1e-9
    assert np.abs(star_plain[-1] - star_traj[-1]).max() > 1e-4


def test_device_results_stay_on_the_gpu_and_equal_host_results(cuda_device) -> None:
    """run(device=True): trajectories are torch CUDA tensors written in place
    by the kernels, bit-identical to run()'s host arrays, exportable through
    DLPack -- also through a satellite -> stream chain whose origin table is
    built on the device from the satellite's device trajectory."""
    import torch

    sat_state = np.array([[1.2, 0.0, 0.05, 0.0, 1.0, 0.02]])
    rng = np.random.default_rng(12)
    stars_state = sat_state[0] + np.hstack([rng.normal(0, 0.05, (30, 3)), rng.normal(0, 0.05, (30, 3))])

    def build():
        gal = dft.background(dft.Potential.bovy())
        sats = dft.particles(dft.Potential.plummer(0.02, 0.05), sat_state)
        stars = dft.test_particles(stars_state)
        sim = dft.Config(method=dft.Method.DOP853, ts=(0.0, 6.0, 31), tolerance=1e-10, attached_potentials=True)
        sim.add(sats, gal)
        sim.add(stars, gal, sats)
        return sim

    host = build().run()
    dev, stats = build().run(device=True, stats=True)
    assert dev[1] is None
    for h, d in zip((host[0], host[2]), (dev[0], dev[2])):
        assert isinstance(d, torch.Tensor) and d.is_cuda and d.dtype == torch.float64
        np.testing.assert_array_equal(d.cpu().numpy(), h)
    assert (stats[2]["status"] == 0).all() and stats[2]["accepted"].min() > 0
    # zero-copy hand-off to any DLPack consumer
    capsule = torch.utils.dlpack.to_dlpack(dev[2])
    back = torch.utils.dlpack.from_dlpack(capsule)
    assert back.data_ptr() == dev[2].data_ptr()
