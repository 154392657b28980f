"""Parity at each benchmark configuration's own inputs, against the oracle.

* Configuration 1 exactly: the seeded 1,024 Kepler particles, ts = (0, 20 pi,
  1001), DOPR54 at rtol = atol = 1e-10; every particle, every sample and the
  accepted-step counts, in both precision units.
* Configuration 5's forward pass: a seeded 1,024-particle subsample of the
  65,536 stream particles in the Bovy composite, DOP853 at 1e-10 to t = 50.
* Configuration 3 over full spans: a seeded 256-particle subsample of the
  2^22 uneven Bovy particles (t_end up to 1000, 101 outputs each), DOP853 at
  1e-10.  Over hundreds of dynamical times some of these orbits amplify
  last-bit differences (a different libm rounding, a fused multiply-add)
  exponentially.  The test therefore measures each particle's own
  sensitivity: the oracle integrates it again from initial conditions moved
  by one ulp (three directions), and the GPU's deviation from the oracle must
  stay within 1e-9 or within a bounded factor of that intrinsic spread.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.workloads import bovy_disc, bovy_radial_force, kepler_disc, stream_progenitor

pytestmark = pytest.mark.gpu


def _sample_err(got, ref):
    """Per particle: max over samples of the largest component error over the
    sample's largest component."""
    scale = np.maximum(np.abs(ref).max(axis=2), 1e-300)
    return (np.abs(got - ref).max(axis=2) / scale).max(axis=0)


@pytest.mark.parametrize("precision", [capi.EXACT, capi.FMA])
def test_configuration_1_exact_inputs(cuda_device, oracle, precision):
    y0 = kepler_disc(1024, seed=1)
    ts = np.linspace(0.0, 20.0 * np.pi, 1001)
    got = capi.integrate_host(capi.DOPR54, capi.kepler(1.0), y0, ts=ts, rtol=1e-10, atol=1e-10,
                              precision=precision, schedule=capi.ORDERED)
    ref = oracle.integrate_batch(oracle.DOPR54, oracle.kepler(1.0), y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert (got["status"] == 0).all() and (np.asarray(ref["status"]) == 0).all()
    err = _sample_err(got["out"], ref["out"])
    same_steps = float((got["accepted"].astype(np.int64) == ref["accepted"]).mean())
    print(f"C1 precision {precision}: max rel err {err.max():.3e}, median {np.median(err):.3e}, "
          f"identical step counts {same_steps:.4f}")
    assert err.max() < 1e-9
    assert same_steps >= 0.99


@pytest.mark.parametrize("precision", [capi.EXACT, capi.FMA])
def test_configuration_5_forward_subsample(cuda_device, oracle, precision):
    vc = float(np.sqrt(1.5 * abs(float(bovy_radial_force(np.array([1.5]))[0]))))
    _, y0_all = stream_progenitor(65536, vc, seed=5)
    idx = np.sort(np.random.default_rng(55).choice(len(y0_all), 1024, replace=False))
    y0 = y0_all[idx]
    ts = np.array([0.0, 50.0])
    got = capi.integrate_host(capi.DOP853, capi.bovy(), y0, ts=ts, rtol=1e-10, atol=1e-10,
                              precision=precision, schedule=capi.ORDERED)
    ref = oracle.integrate_batch(oracle.DOP853, oracle.bovy(), y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert (got["status"] == 0).all() and (np.asarray(ref["status"]) == 0).all()
    err = _sample_err(got["out"], ref["out"])
    same_steps = float((got["accepted"].astype(np.int64) == ref["accepted"]).mean())
    print(f"C5 forward precision {precision}: max rel err {err.max():.3e}, median {np.median(err):.3e}, "
          f"identical step counts {same_steps:.4f}")
    assert err.max() < 1e-9


@pytest.mark.parametrize("precision", [capi.EXACT, capi.FMA])
def test_configuration_3_full_spans_subsample(cuda_device, oracle, precision):
    y0_all, te_all = bovy_disc(1 << 22, seed=3)
    idx = np.sort(np.random.default_rng(333).choice(len(y0_all), 256, replace=False))
    y0, t_end = y0_all[idx], te_all[idx]
    nt = 101

    def ref_run(y):
        return oracle.integrate_batch(oracle.DOP853, oracle.bovy(), y, t_end=t_end, nt=nt, rtol=1e-10, atol=1e-10)

    got = capi.integrate_host(capi.DOP853, capi.bovy(), y0, t_end=t_end, nt=nt, rtol=1e-10, atol=1e-10,
                              precision=precision, schedule=capi.ORDERED)
    ref = ref_run(y0)
    assert (got["status"] == 0).all() and (np.asarray(ref["status"]) == 0).all()
    err = _sample_err(got["out"], ref["out"])
    # the oracle's own spread: the same particles from initial conditions one
    # ulp away, in three directions (all components up, all down, positions
    # up and velocities down)
    flip = np.concatenate([np.full((len(y0), 3), np.inf), np.full((len(y0), 3), -np.inf)], axis=1)
    spread = np.zeros(len(y0))
    for direction in (np.inf, -np.inf, flip):
        spread = np.maximum(spread, _sample_err(ref_run(np.nextafter(y0, direction))["out"], ref["out"]))
    same_steps = float((got["accepted"].astype(np.int64) == ref["accepted"]).mean())
    within = float((err < 1e-9).mean())
    print(f"C3 precision {precision}: max rel err {err.max():.3e}, median {np.median(err):.3e}, "
          f"within 1e-9 {within:.4f}, identical step counts {same_steps:.4f}; one-ulp spread of the "
          f"oracle itself: max {spread.max():.3e}, median {np.median(spread):.3e}")
    # Every particle within 1e-9 or within 1e3 of its own one-ulp spread; the
    # spread in three directions can miss the one direction the GPU's
    # rounding pushes a sensitive orbit along, so up to 2 of the 256 may
    # exceed that (still below 1e-5, far from any real defect).
    bound = np.maximum(1e-9, 1e3 * spread)
    bad = np.flatnonzero(err > bound)
    assert bad.size <= 2 and (err < 1e-5).all(), [(int(i), float(err[i]), float(spread[i]), float(t_end[i]))
                                                  for i in bad[:8]]
