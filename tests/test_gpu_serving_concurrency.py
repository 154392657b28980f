"""The request server's concurrency: no lock is held across a CUDA call.

* A large request whose result buffer is pageable host memory (its copy back
  returns only once its kernel has finished) holds up only its own stream:
  small requests submitted after it are admitted on the other streams and
  finish long before it.
* drift_server_cancel stops a request's remaining particles; the wait that
  follows reports the cancellation within a bounded time, and the server
  keeps serving.
* The host path (drift_integrate_host, whose buffer growth frees device
  memory) runs to completion while a server batch is in flight.
* drift_server_wait_any hands back whichever request finishes first: small
  requests submitted after a large one are retired before it.
* Destroying a server while another thread waits: drift_server_destroy lets
  the thread inside drift_server_wait return before it frees the server, and
  Server.close() cancels what other threads wait for and lets their calls
  return first.
Every wait here has a time limit, so a stall fails the test instead of
holding the run.
"""

from __future__ import annotations

import ctypes
import threading
import time

import numpy as np
import pytest

from astrodrift_b200 import capi, serving
from astrodrift_b200.serving import RequestCancelled, Server

pytestmark = pytest.mark.gpu

WAIT_S = 120.0


def _disc(n, seed, vscale=1.0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 2.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    vt = vscale * rng.uniform(0.7, 1.0, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), 0.1 * r * rng.normal(size=n),
                     -vt * np.sin(phi), vt * np.cos(phi), 0.05 * rng.normal(size=n)], axis=1)


def _small(seed):
    return dict(method=capi.DOP853, pot=capi.plummer(1.0, 1.0), y0=_disc(64, seed, 0.5),
                ts=np.linspace(0.0, 10.0, 11), rtol=1e-10, atol=1e-10)


@pytest.fixture(scope="module")
def warm(cuda_device):
    """Launches the kernels these tests time once, small, before any of them
    runs: a kernel's first launch in a process loads its code (lazy module
    loading), which waits for the device, so a first small batch launched
    beside a running large one would measure that wait instead of serving."""
    kw = _small(0)
    for schedule in (capi.PLAIN, capi.ORDERED):
        capi.integrate_host(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"], atol=kw["atol"],
                            schedule=schedule)
        capi.integrate_host(capi.DOP853, capi.bovy(), _disc(64, 1), t_end=np.full(64, 1.0), nt=3, rtol=1e-11,
                            atol=1e-11, precision=capi.FMA, schedule=schedule)
    return cuda_device


def test_small_requests_finish_while_a_large_pageable_request_runs(warm):
    n = 60_000
    y0 = _disc(n, 1)
    t_end = np.full(n, 1500.0)
    out = np.empty((101, n, 6))  # pageable: numpy memory, not drift_host_alloc
    with Server(streams=4, memory_fraction=0.5) as srv:
        large = srv.submit(capi.DOP853, capi.bovy(), y0, t_end=t_end, nt=101, rtol=1e-11, atol=1e-11,
                           precision=capi.FMA, out=out)
        smalls = []
        for i in range(8):
            kw = _small(100 + i)
            smalls.append((kw, srv.submit(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"],
                                          atol=kw["atol"])))
        small_lat = []
        for kw, h in smalls:
            res = h.wait(timeout=WAIT_S)
            small_lat.append(res["latency_s"])
            ref = capi.integrate_host(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"],
                                      atol=kw["atol"], schedule=capi.PLAIN)
            np.testing.assert_array_equal(res["out"], ref["out"])
        big = large.wait(timeout=WAIT_S)
    assert (big["status"] == 0).all()
    assert np.isfinite(out).all()
    # the small requests ran while the large one held its stream
    assert max(small_lat) < 0.25 * big["latency_s"], (small_lat, big["latency_s"])


def test_cancel_a_queued_request_and_keep_serving(cuda_device):
    # one stream: the second request waits behind the first and is cancelled
    # before any of its particles is admitted
    n = 20_000
    with Server(streams=1, memory_fraction=0.5) as srv:
        first = srv.submit(capi.DOP853, capi.bovy(), _disc(n, 2), t_end=np.full(n, 400.0), nt=11,
                           rtol=1e-10, atol=1e-10, precision=capi.FMA)
        second = srv.submit(capi.DOP853, capi.plummer(1.0, 1.0), _disc(n, 3, 0.5),
                            ts=np.linspace(0.0, 50.0, 11), rtol=1e-10, atol=1e-10)
        second.cancel()
        with pytest.raises(RequestCancelled):
            second.wait(timeout=WAIT_S)
        res = first.wait(timeout=WAIT_S)
        assert (res["status"] == 0).all()
        # cancelling a finished request changes nothing; the server still serves
        kw = _small(7)
        h = srv.submit(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"], atol=kw["atol"])
        h.wait(timeout=WAIT_S)
        st = srv.stats()
    assert st["requests_pending"] == 0 and st["batches_in_flight"] == 0


def test_cancel_a_request_running_in_chunks(cuda_device):
    # particle chunks of 2,048 on one stream: cancelling stops the chunks not
    # yet admitted, the one on the GPU finishes, and the wait ends
    n = 65_536
    with Server(streams=1, memory_fraction=0.5, max_batch_particles=2048) as srv:
        h = srv.submit(capi.DOP853, capi.bovy(), _disc(n, 4), t_end=np.full(n, 300.0), nt=11,
                       rtol=1e-10, atol=1e-10, precision=capi.FMA)
        import time

        time.sleep(0.05)
        h.cancel()
        with pytest.raises(RequestCancelled):
            h.wait(timeout=WAIT_S)
        st = srv.stats()
        assert st["particles_completed"] < n
        assert st["requests_pending"] == 0 and st["batches_in_flight"] == 0
        kw = _small(8)
        res = srv.submit(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"],
                         atol=kw["atol"]).wait(timeout=WAIT_S)
        assert (res["status"] == 0).all()


def test_host_path_runs_while_a_server_batch_is_in_flight(cuda_device):
    n = 40_000
    with Server(streams=2, memory_fraction=0.3) as srv:
        h = srv.submit(capi.DOP853, capi.bovy(), _disc(n, 5), t_end=np.full(n, 800.0), nt=21,
                       rtol=1e-10, atol=1e-10, precision=capi.FMA)
        # growing host-path requests: each reallocates (frees and allocates)
        # the context's device buffers while the batch runs
        for m in (1_000, 20_000, 200_000):
            y0 = _disc(m, 10 + m, 0.5)
            res = capi.integrate_host(capi.DOP853, capi.plummer(1.0, 1.0), y0, ts=np.linspace(0.0, 5.0, 6),
                                      rtol=1e-9, atol=1e-9)
            assert (res["status"] == 0).all()
        out = h.wait(timeout=WAIT_S)
    assert (out["status"] == 0).all()


def test_wait_any_retires_requests_in_completion_order(warm):
    n = 60_000
    with Server(streams=4, memory_fraction=0.5) as srv:
        large = srv.submit(capi.DOP853, capi.bovy(), _disc(n, 7), t_end=np.full(n, 1500.0), nt=101,
                           rtol=1e-11, atol=1e-11, precision=capi.FMA)
        pending, inputs = [large], {}
        for i in range(8):
            kw = _small(200 + i)
            h = srv.submit(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"], atol=kw["atol"])
            pending.append(h)
            inputs[h.ticket] = kw
        retired = []
        while pending:
            i, res = srv.wait_any(pending, timeout=WAIT_S)
            h = pending.pop(i)
            retired.append(h)
            if h is large:
                assert (res["status"] == 0).all()
                continue
            kw = inputs[h.ticket]
            ref = capi.integrate_host(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"],
                                      atol=kw["atol"], schedule=capi.PLAIN)
            np.testing.assert_array_equal(res["out"], ref["out"])
        # the small requests submitted after the large one are retired before it
        assert retired[-1] is large
        # a retired ticket is released: waiting for it again is an error
        with pytest.raises(RuntimeError, match="unknown ticket"):
            srv.wait_any([large], timeout=1.0)


def _one_stream_with_a_queued_request():
    """A server whose only stream runs a long Bovy request, with a small
    request queued behind it."""
    srv = Server(streams=1, memory_fraction=0.3)
    n = 20_000
    srv.submit(capi.DOP853, capi.bovy(), _disc(n, 3), t_end=np.full(n, 400.0), nt=11, rtol=1e-10, atol=1e-10,
               precision=capi.FMA)
    kw = _small(300)
    queued = srv.submit(kw["method"], kw["pot"], kw["y0"], ts=kw["ts"], rtol=kw["rtol"], atol=kw["atol"])
    return srv, queued


def test_destroy_lets_a_thread_inside_a_wait_return_first(warm):
    srv, queued = _one_stream_with_a_queued_request()
    ptr, lib = srv._ptr, serving._lib()
    got = {}

    def raw_wait():
        result, latency = ctypes.c_int(-1), ctypes.c_double(0.0)
        got["rc"] = lib.drift_server_wait(ptr, queued.ticket, WAIT_S, ctypes.byref(result), ctypes.byref(latency))
        got["result"] = result.value

    t = threading.Thread(target=raw_wait)
    t.start()
    time.sleep(0.3)  # the thread is blocked inside drift_server_wait
    assert lib.drift_server_destroy(ptr) == 0
    t.join(timeout=WAIT_S)
    assert not t.is_alive()
    srv._ptr = ctypes.c_void_p()  # destroyed above, not through the handle
    assert got["rc"] == 0
    assert got["result"] in (0, 7)  # finished, or DRIFT_ERROR_CANCELLED while queued


def test_close_cancels_what_other_threads_wait_for(warm):
    srv, queued = _one_stream_with_a_queued_request()
    outcome = {}

    def waiter():
        try:
            outcome["res"] = queued.wait(timeout=WAIT_S)
        except RequestCancelled:
            outcome["cancelled"] = True
        except Exception as e:  # noqa: BLE001 - reported below
            outcome["error"] = repr(e)

    t = threading.Thread(target=waiter)
    t.start()
    deadline = time.monotonic() + 10.0
    while srv._calls == 0 and time.monotonic() < deadline:
        time.sleep(0.001)  # until the waiter's call is in progress
    srv.close()
    t.join(timeout=WAIT_S)
    assert not t.is_alive()
    assert "error" not in outcome, outcome
    assert outcome.get("cancelled") or (outcome["res"]["status"] == 0).all()
    with pytest.raises(RuntimeError, match="closed"):
        srv.stats()
