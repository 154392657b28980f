"""Server.close() with calls in progress on other threads (host logic, no
GPU).  A fake of the drift_server_* entry points stands in for the library,
so the test sees the order close() follows: cancel the tickets not yet
waited for, let the calls in progress return, destroy the server once, and
refuse every call made afterwards."""

from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from astrodrift_b200 import capi, serving
from astrodrift_b200.serving import RequestCancelled

CANCELLED = 7  # DRIFT_ERROR_CANCELLED


class FakeServerLib:
    """drift_server_* with the C entry points' meaning; requests finish
    when the test says so or when they are cancelled."""

    def __init__(self):
        self.cond = threading.Condition()
        self.next_ticket = 1
        self.results = {}   # ticket -> drift_result once the request has ended
        self.inside = 0     # threads inside drift_server_wait
        self.destroys = []  # threads inside a wait at each destroy

    def finish(self, ticket, result=0):
        with self.cond:
            self.results[ticket] = result
            self.cond.notify_all()

    def drift_server_create(self, options, out):
        out._obj.value = 0x1000
        return 0

    def drift_server_stats_get(self, server, stats):
        stats._obj.device = 0
        return 0

    def drift_server_submit(self, server, launch, ticket):
        with self.cond:
            ticket._obj.value = self.next_ticket
            self.next_ticket += 1
        return 0

    def drift_server_wait(self, server, ticket, timeout, result, latency):
        with self.cond:
            self.inside += 1
            self.cond.wait_for(lambda: ticket in self.results, timeout=10.0)
            result._obj.value = self.results.get(ticket, -1)
            latency._obj.value = 0.0
            self.inside -= 1
            self.cond.notify_all()
        return 0

    def drift_server_cancel(self, server, ticket):
        with self.cond:
            self.results.setdefault(ticket, CANCELLED)  # a finished request keeps its result
            self.cond.notify_all()
        return 0

    def drift_server_destroy(self, server):
        with self.cond:
            self.destroys.append(self.inside)
        return 0


class FakePinned:
    def __init__(self, shape, dtype=np.float64):
        self.array = np.zeros(shape, dtype)


@pytest.fixture
def fake(monkeypatch):
    lib = FakeServerLib()
    monkeypatch.setattr(serving, "_lib", lambda: lib)
    monkeypatch.setattr(serving, "PinnedArray", FakePinned)
    return lib


def _submit(srv):
    return srv.submit(capi.DOP853, capi.plummer(), np.zeros((4, 6)), ts=np.linspace(0.0, 1.0, 3))


def test_close_cancels_a_wait_in_progress_and_destroys_after_it_returns(fake):
    srv = serving.Server()
    queued, finished = _submit(srv), _submit(srv)
    fake.finish(finished.ticket)  # ended on the device, not yet waited for
    outcome = {}

    def waiter():
        try:
            outcome["res"] = queued.wait()
        except RequestCancelled:
            outcome["cancelled"] = True

    t = threading.Thread(target=waiter)
    t.start()
    deadline = time.monotonic() + 5.0
    while fake.inside == 0 and time.monotonic() < deadline:
        time.sleep(0.001)
    assert fake.inside == 1
    srv.close()
    t.join(timeout=5.0)
    assert not t.is_alive()
    assert outcome == {"cancelled": True}
    assert fake.destroys == [0]  # destroyed once, with no thread inside a wait
    assert fake.results[finished.ticket] == 0  # cancelling a finished request changed nothing
    with pytest.raises(RuntimeError, match="closed"):
        finished.wait()
    with pytest.raises(RuntimeError, match="closed"):
        srv.stats()
    with pytest.raises(RuntimeError, match="closed"):
        _submit(srv)
    srv.close()
    assert fake.destroys == [0]


def test_results_waited_before_close_are_released(fake):
    with serving.Server() as srv:
        a = _submit(srv)
        fake.finish(a.ticket)
        res = a.wait()
        assert res["latency_s"] == 0.0 and res["out"].shape == (3, 4, 6)
        assert srv._tickets == set()
    assert fake.destroys == [0]
