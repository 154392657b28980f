"""Explicit host-path contexts (drift_context_*): the same results as the
implicit per-device context, their buffers reported and freed, and separate
contexts used from two host threads at once."""

from __future__ import annotations

import threading

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


def _states(n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 2.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(u, rng.normal(size=(n, 3)))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return np.hstack([u * r[:, None], v * (0.7 / np.sqrt(r))[:, None]])


def test_context_matches_the_implicit_context_and_frees_its_memory(cuda_device):
    import torch

    y0 = _states(70000, 1)  # above the host path's chunking threshold
    ts = np.linspace(0.0, 5.0, 41)
    ref = capi.integrate_host(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10)
    free_before, _ = torch.cuda.mem_get_info()
    ctx = capi.Context(device=0)
    got = capi.integrate_host(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10, context=ctx)
    for k in ("out", "y_final", "status", "accepted", "rejected"):
        np.testing.assert_array_equal(got[k], ref[k])
    dev_bytes, pinned = ctx.memory()
    assert dev_bytes >= 70000 * 41 * 48 // 4  # at least one trajectory chunk
    assert pinned > 0  # pageable numpy outputs are staged through page-locked buffers
    free_used, _ = torch.cuda.mem_get_info()
    ctx.close()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after - free_used >= dev_bytes * 0.9
    assert abs(free_after - free_before) < 64 << 20
    with pytest.raises(RuntimeError, match="closed"):
        ctx.memory()


def test_two_threads_with_their_own_contexts(cuda_device):
    ts = np.linspace(0.0, 8.0, 17)
    jobs = [(capi.DOP853, capi.bovy(), _states(20000, 2)), (capi.DOPR54, capi.kepler(1.0), _states(30000, 3))]
    refs = [capi.integrate_host(m, p, y, ts=ts, rtol=1e-10, atol=1e-10) for m, p, y in jobs]
    results = [None, None]
    errors = []

    def work(i):
        try:
            with capi.Context() as ctx:
                m, p, y = jobs[i]
                results[i] = capi.integrate_host(m, p, y, ts=ts, rtol=1e-10, atol=1e-10, context=ctx)
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for got, ref in zip(results, refs):
        np.testing.assert_array_equal(got["out"], ref["out"])
        np.testing.assert_array_equal(got["accepted"], ref["accepted"])


def test_context_on_a_missing_device_is_refused(cuda_device):
    with pytest.raises(RuntimeError, match="no such CUDA device"):
        capi.Context(device=1 << 20)
