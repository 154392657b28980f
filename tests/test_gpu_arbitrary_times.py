"""Arbitrary (non-uniform) output times on the GPU against the oracle.

DOP853's dense output serves any strictly monotone grid; DOPR54 needs
drift_launch.arbitrary_times so that each interval ends exactly at the next
requested time (the default keeps galpy's uniform-grid semantics).  The
Python surface accepts such grids with Config(arbitrary_times=True).
Exact arithmetic; 1e-9 relative per sample, as the other parity tests.
"""

from __future__ import annotations

import numpy as np
import pytest

import astrodrift_b200 as dft
from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    a = np.asarray(a).reshape(-1, 6)
    b = np.asarray(b).reshape(-1, 6)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def _ics(n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.4, 2.0, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    v = np.sqrt(r * r / (r * r + 1.0) ** 1.5) * rng.uniform(0.6, 1.1, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(0, 0.1, n),
                     -v * np.sin(phi), v * np.cos(phi), rng.normal(0, 0.05, n)], axis=1)


GRIDS = {
    "log": np.concatenate([[0.0], np.logspace(-2, 1.2, 30)]),
    "ragged": np.array([0.0, 0.001, 0.3, 0.31, 2.0, 2.5, 7.0, 7.0001, 9.0]),
    "backward": -np.concatenate([[0.0], np.logspace(-1, 1, 9)]),
}


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
@pytest.mark.parametrize("grid", list(GRIDS))
def test_arbitrary_grids_match_oracle(cuda_device, oracle, method, grid):
    ts = GRIDS[grid]
    y0 = _ics(400, 3)
    got = capi.integrate_host(method, capi.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-11, atol=1e-11,
                              arbitrary_times=True)
    ref = oracle.integrate_batch(method, oracle.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-11, atol=1e-11,
                                 arbitrary_times=True)
    assert (got["status"] == 0).all()
    assert rel_err(got["out"], ref["out"]) < 1e-9
    if method == capi.DOPR54:
        np.testing.assert_array_equal(got["accepted"], ref["accepted"].astype(np.uint32))


def test_uniform_grid_default_semantics_unchanged(cuda_device, oracle):
    ts = np.linspace(0.0, 10.0, 21)
    y0 = _ics(300, 4)
    a = capi.integrate_host(capi.DOPR54, capi.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-11, atol=1e-11)
    b = oracle.integrate_batch(0, oracle.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-11, atol=1e-11)
    assert rel_err(a["out"], b["out"]) < 1e-9


def test_python_surface_with_arbitrary_times(cuda_device, oracle):
    ts = np.concatenate([[0.0], np.logspace(-1, 1, 15)])
    y0 = _ics(50, 5)
    for method, om in ((dft.Method.DOPR54, 0), (dft.Method.DOP853, 1)):
        gal = dft.background(dft.Potential.plummer(1.0, 1.0))
        stars = dft.test_particles(y0)
        sim = dft.Config(method=method, ts=ts, tolerance=1e-11, arbitrary_times=True)
        sim.add(stars, gal)
        out, _ = sim.run()
        ref = oracle.integrate_batch(om, oracle.plummer(1.0, 1.0), y0, ts=ts, rtol=1e-11, atol=1e-11,
                                     arbitrary_times=True)["out"]
        assert out.shape == (len(ts), 50, 6)
        assert rel_err(out, ref) < 1e-9
