"""Routing whole requests to servers by free device memory (host logic, no
GPU): the policy, the byte estimate and the Router's bookkeeping over fake
servers."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.serving import Router, request_bytes, route


def test_route_prefers_most_free_memory_then_fewest_queued_then_lowest_index():
    assert route([100, 300, 200], [0, 0, 0], 10) == 1
    assert route([300, 300, 200], [2, 1, 0], 10) == 1
    assert route([300, 300, 300], [1, 1, 1], 10) == 0
    # larger than every server: still the freest one (it runs in chunks)
    assert route([5, 7], [0, 0], 1 << 40) == 1
    with pytest.raises(ValueError):
        route([], [], 1)
    with pytest.raises(ValueError):
        route([1, 2], [0], 1)


def test_request_bytes_counts_the_admission_buffers():
    up = lambda b: (b + 255) // 256 * 256  # noqa: E731
    n, nt = 1000, 17
    base = up(n * 48) + up(n * 48) + up(n) + 3 * up(n * 4)
    assert request_bytes(n, nt) == base + up(nt * 8) + up(nt * n * 48)
    assert request_bytes(n, nt, shared_grid=False) == base + up(n * 8) + up(nt * n * 48)
    assert request_bytes(n, nt, want_out=False) == base + up(nt * 8)


class _FakeRequest:
    def __init__(self):
        self.arrays = {}


class _FakeServer:
    def __init__(self, device, budget):
        self.device_index = device
        self.budget = budget
        self.pending = []
        self.closed = False

    def stats(self):
        return dict(memory_budget=self.budget, bytes_in_flight=0, bytes_pending=sum(self.pending),
                    requests_pending=len(self.pending))

    def submit(self, method, pot, y0, *, ts=None, t_end=None, nt=None, want_out=True, **kw):
        n = np.asarray(y0).size // 6
        self.pending.append(request_bytes(n, len(ts) if ts is not None else nt,
                                          shared_grid=ts is not None, want_out=want_out))
        return _FakeRequest()

    def close(self):
        self.closed = True


def test_router_spreads_requests_by_what_each_server_has_left():
    servers = [_FakeServer(0, 4 << 20), _FakeServer(1, 6 << 20)]
    y0 = np.zeros((2000, 6))
    ts = np.linspace(0.0, 1.0, 5)
    need = request_bytes(2000, 5)
    with Router(servers) as rt:
        devices = [rt.submit(capi.DOP853, capi.plummer(), y0, ts=ts).arrays["device"] for _ in range(8)]
        # free memory decides each pick: replay the policy by hand
        free = [4 << 20, 6 << 20]
        queued = [0, 0]
        want = []
        for _ in range(8):
            i = route(free, queued, need)
            want.append(i)
            free[i] -= need
            queued[i] += 1
        assert devices == want
        assert rt.routed == [want.count(0), want.count(1)]
        assert sum(rt.routed) == 8 and min(rt.routed) > 0
    assert all(s.closed for s in servers)


def test_router_needs_a_server():
    with pytest.raises(ValueError):
        Router([])


class _PollingServer:
    """Stands in for a Server in Router.wait_any: its requests finish after
    a given number of polls."""

    def __init__(self, finish_after):
        self.finish_after = dict(finish_after)  # ticket -> polls before it is done
        self.polls = 0

    def _wait_any(self, requests, timeout, poll):
        assert poll and timeout > 0
        self.polls += 1
        for i, r in enumerate(requests):
            if self.polls >= self.finish_after[r.ticket]:
                return i, 0, 0.25
        return None

    def wait_any(self, requests, timeout=0.0):
        return 0, requests[0]._finish(0, 0.5)


class _Req:
    def __init__(self, server, ticket):
        self.server, self.ticket = server, ticket

    def _finish(self, result, latency):
        return {"ticket": self.ticket, "result": result, "latency_s": latency}


def test_router_wait_any_polls_every_server_until_one_request_finishes():
    a, b = _PollingServer({1: 5, 2: 9}), _PollingServer({3: 3})
    reqs = [_Req(a, 1), _Req(a, 2), _Req(b, 3)]
    rt = Router([a, b])
    i, res = rt.wait_any(reqs)
    assert (i, res["ticket"]) == (2, 3)  # b's request finishes on its third poll
    assert a.polls == 3 and b.polls == 3
    # requests of one server wait in that server's own call
    i, res = rt.wait_any([_Req(a, 1)])
    assert (i, res["latency_s"]) == (0, 0.5)
    with pytest.raises(ValueError):
        rt.wait_any([])


def test_router_wait_any_gives_up_at_its_timeout():
    a, b = _PollingServer({1: 10**9}), _PollingServer({2: 10**9})
    rt = Router([a, b])
    with pytest.raises(RuntimeError, match="still running"):
        rt.wait_any([_Req(a, 1), _Req(b, 2)], timeout=0.01)
