"""The request server: continuous batching gives every request the result it
gets alone.

A heterogeneous mix (both methods, three potentials, 1 to 40,000 particles,
shared and per-particle grids, three tolerances, ordered and persistent
batches) is submitted from several
threads into a server whose memory budget forces large requests into
particle chunks and whose streams run several batches at once.  Exact
arithmetic makes each particle's integration independent of which launch,
chunk or thread ran it, so every result must equal drift_integrate_host's for
the same request bit for bit.
"""

from __future__ import annotations

import threading

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.serving import Server

pytestmark = pytest.mark.gpu


def _mix(seed=0, count=24):
    rng = np.random.default_rng(seed)
    pots = [capi.kepler(1.0), capi.plummer(1.0, 1.0), capi.bovy()]
    reqs = []
    for i in range(count):
        n = int(2 ** rng.uniform(0, 15.3))
        r = rng.uniform(0.5, 2.0, n)
        u = rng.normal(size=(n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        u[:, 2] *= 0.3  # keep away from the z axis (galpy Kepler force is singular there)
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        v = np.cross(u, rng.normal(size=(n, 3)))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        y0 = np.hstack([u * r[:, None], v * (0.8 / np.sqrt(r))[:, None]])
        nt = int(np.exp(rng.uniform(np.log(2), np.log(120))))
        kw = dict(method=[capi.DOPR54, capi.DOP853][i % 2], pot=pots[(i // 2) % 3], y0=y0,
                  rtol=[1e-8, 1e-10, 1e-12][i % 3])
        kw["atol"] = kw["rtol"]
        if i % 5 == 0:
            kw["schedule"] = capi.PERSISTENT  # the rest use the server's default, ordered
        if i % 4 == 3:
            kw.update(t_end=rng.uniform(1.0, 6.0, n), nt=max(nt, 2))
        else:
            kw.update(ts=np.linspace(0.0, rng.uniform(1.0, 6.0), max(nt, 2)))
        reqs.append(kw)
    return reqs


def _alone(kw):
    args = {k: v for k, v in kw.items() if k not in ("method", "pot", "y0", "schedule")}
    return capi.integrate_host(kw["method"], kw["pot"], kw["y0"], schedule=capi.PLAIN, **args)


@pytest.mark.parametrize("reserve", [0, 12, 40])  # percent of the SMs left to small batches
def test_each_result_is_the_same_alone_and_in_the_mix(cuda_device, reserve):
    mix = _mix()
    with Server(memory_bytes=96 << 20, streams=3, max_batch_particles=20000,
                sm_reserve_percent=reserve) as srv:
        handles = [None] * len(mix)

        def submit(idx):
            for i in idx:
                kw = mix[i]
                args = {k: v for k, v in kw.items() if k not in ("method", "pot", "y0")}
                handles[i] = srv.submit(kw["method"], kw["pot"], kw["y0"], **args)

        threads = [threading.Thread(target=submit, args=(range(k, len(mix), 3),)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        results = [h.wait(timeout=600) for h in handles]
        stats = srv.stats()
    assert stats["requests_completed"] == len(mix)
    assert stats["pieces_launched"] > stats["batches_launched"] or stats["batches_launched"] > len(mix)
    for kw, got in zip(mix, results):
        ref = _alone(kw)
        np.testing.assert_array_equal(got["out"], ref["out"])
        np.testing.assert_array_equal(got["accepted"], ref["accepted"])
        np.testing.assert_array_equal(got["status"], ref["status"])
        assert got["latency_s"] > 0


def test_request_larger_than_the_budget_runs_in_chunks(cuda_device):
    rng = np.random.default_rng(4)
    n = 30000
    y0 = np.hstack([rng.uniform(0.5, 1.5, (n, 3)), rng.uniform(-0.3, 0.3, (n, 3))])
    ts = np.linspace(0.0, 3.0, 64)
    # 30000 x 64 x 48 B = 92 MB of trajectory against a 16 MB budget
    with Server(memory_bytes=16 << 20, streams=2) as srv:
        got = srv.submit(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10).wait(timeout=600)
        stats = srv.stats()
    ref = capi.integrate_host(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10)
    np.testing.assert_array_equal(got["out"], ref["out"])
    assert stats["batches_launched"] >= 6
    assert stats["peak_bytes_in_flight"] <= 16 << 20


def test_close_with_requests_in_flight_returns(cuda_device):
    rng = np.random.default_rng(5)
    y0 = np.hstack([rng.uniform(0.5, 1.5, (2000, 3)), rng.uniform(-0.3, 0.3, (2000, 3))])
    srv = Server(memory_bytes=64 << 20, streams=1)
    hs = [srv.submit(capi.DOP853, capi.plummer(), y0, ts=np.linspace(0, 20, 11), rtol=1e-12, atol=1e-12)
          for _ in range(6)]
    hs[0].wait(timeout=120)
    srv.close()  # batches in flight finish; requests not yet admitted are cancelled
    with pytest.raises(RuntimeError, match="closed"):
        hs[-1].wait(timeout=1)


def test_server_on_an_explicit_device_and_a_missing_one(cuda_device):
    with Server(memory_bytes=32 << 20, device=0) as srv:
        assert srv.device_index == 0
        assert srv.stats()["device"] == 0
    with pytest.raises(RuntimeError, match="no such CUDA device"):
        Server(device=1 << 20)


def test_router_sends_each_request_whole_to_the_freest_server(cuda_device):
    """Two servers on the same GPU with different budgets: the first request
    goes to the larger one, every request's result equals the one it gets
    alone, and the queued bytes the servers report match the host estimate."""
    from astrodrift_b200.serving import Router, request_bytes

    mix = _mix(seed=3, count=12)
    servers = [Server(memory_bytes=48 << 20, streams=2), Server(memory_bytes=160 << 20, streams=2)]
    with Router(servers) as rt:
        handles = []
        for kw in mix:
            args = {k: v for k, v in kw.items() if k not in ("method", "pot", "y0")}
            handles.append(rt.submit(kw["method"], kw["pot"], kw["y0"], **args))
        assert handles[0].arrays["server"] == 1
        results = [h.wait(timeout=600) for h in handles]
        assert sum(rt.routed) == len(mix)
        for st in rt.stats():
            assert st["bytes_pending"] == 0 and st["requests_pending"] == 0
    for kw, res in zip(mix, results):
        ref = _alone(kw)
        np.testing.assert_array_equal(res["out"], ref["out"])
        np.testing.assert_array_equal(res["status"], ref["status"])
        assert res["device"] == 0


def test_router_wait_any_retires_requests_of_every_server(cuda_device):
    """Router.wait_any over requests spread across two servers returns each
    exactly once, with the result it gets alone."""
    from astrodrift_b200.serving import Router

    mix = _mix(seed=4, count=10)
    servers = [Server(memory_bytes=64 << 20, streams=2), Server(memory_bytes=64 << 20, streams=2)]
    with Router(servers) as rt:
        pending, inputs = [], {}
        for k, kw in enumerate(mix):  # alternately, so that both servers hold requests
            args = {a: v for a, v in kw.items() if a not in ("method", "pot", "y0")}
            h = servers[k % 2].submit(kw["method"], kw["pot"], kw["y0"], **args)
            pending.append(h)
            inputs[id(h)] = kw
        done = 0
        while pending:
            i, res = rt.wait_any(pending, timeout=600)
            h = pending.pop(i)
            ref = _alone(inputs[id(h)])
            np.testing.assert_array_equal(res["out"], ref["out"])
            np.testing.assert_array_equal(res["status"], ref["status"])
            done += 1
    assert done == len(mix)


def test_queued_bytes_match_the_host_estimate(cuda_device):
    from astrodrift_b200.serving import request_bytes

    rng = np.random.default_rng(5)
    n_long, n_wait, nt = 60000, 3000, 9
    y_long = np.hstack([rng.uniform(0.5, 2.0, (n_long, 3)), rng.normal(0, 0.3, (n_long, 3))])
    y_wait = np.hstack([rng.uniform(0.5, 2.0, (n_wait, 3)), rng.normal(0, 0.3, (n_wait, 3))])
    ts = np.linspace(0.0, 40.0, nt)
    with Server(memory_bytes=512 << 20, streams=1) as srv:
        a = srv.submit(capi.DOP853, capi.bovy(), y_long, ts=ts, rtol=1e-12, atol=1e-12)
        # a different tolerance cannot join the first batch, so it waits for the one stream
        b = srv.submit(capi.DOP853, capi.bovy(), y_wait, ts=ts, rtol=1e-11, atol=1e-11)
        st = srv.stats()
        if st["requests_pending"] == 1 and st["batches_in_flight"] == 1:
            assert st["bytes_pending"] == request_bytes(n_wait, nt)
        a.wait(timeout=600)
        b.wait(timeout=600)
        assert srv.stats()["bytes_pending"] == 0
