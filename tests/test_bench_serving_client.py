"""bench.py's serving client (host logic, no GPU): against a fake server,
a request that waits for a result buffer holds back no later request that
needs none, a freed buffer goes to the oldest waiting request, and every
request is retired once."""

from __future__ import annotations

import importlib.util
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class FakeHandle:
    def __init__(self, name, n):
        self.name, self.n = name, n


class FakeServer:
    """Requests finish in submission order, one per wait or poll."""

    def __init__(self):
        self.submitted = []
        self.finished = []

    def submit(self, method, pot, y0, *, ts, rtol, atol, precision, want_out, out):
        h = FakeHandle(method, len(y0))
        self.submitted.append((method, want_out))
        return h

    def _next(self, handles):
        i = min(range(len(handles)), key=lambda k: self.submitted.index(
            next(s for s in self.submitted if s[0] == handles[k].name)))
        self.finished.append(handles[i].name)
        return i, {"latency_s": 0.001, "accepted": np.ones(handles[i].n, np.uint32)}

    def wait_any(self, handles, timeout=0.0):
        return self._next(handles)

    def poll_any(self, handles, timeout):
        return self._next(handles)


class FakeSlots:
    def __init__(self, count):
        self.free = list(range(count))

    def view(self, slot, nt, n):
        return np.zeros((nt, n, 6))


def _req(name, n, nt):
    return {"method": name, "pot": None, "y0": np.zeros((n, 6)), "nt": nt, "t_end": 1.0, "rtol": 1e-10, "at": 0.0}


def test_a_request_waiting_for_a_buffer_holds_back_none_that_needs_no_buffer():
    bench = _bench()
    cap = 10 * 4 * 48  # trajectories up to 10 samples of 4 particles fit a buffer
    reqs = [_req("a", 4, 5), _req("b", 4, 5), _req("big", 1000, 100), _req("c", 4, 5)]
    srv, slots = FakeServer(), FakeSlots(1)
    seconds, acc, lat, capped, waits = bench._serve(srv, reqs, cap, None, False, slots)
    # "big" needs no buffer: submitted at once, not after "a" has freed the only one
    assert [name for name, _ in srv.submitted] == ["a", "big", "b", "c"]
    assert dict(srv.submitted) == {"a": True, "big": False, "b": True, "c": True}
    assert sorted(srv.finished) == ["a", "b", "big", "c"]
    assert capped == 1 and len(lat) == 4 and acc == 4 + 1000 + 4 + 4
    assert len(waits) == 3 and waits[0] == 0.0  # one per request that took a buffer
    assert slots.free == [0]  # the buffer is back once everything has retired
