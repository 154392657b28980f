"""Python handle on the request server of the C ABI (drift_server_*).

    with Server(memory_bytes=8 << 30, streams=4) as srv:
        req = srv.submit(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10)
        res = req.wait()            # dict of numpy arrays + "latency_s"

Requests keep their host buffers alive until they complete; trajectory
buffers are page-locked (allocated by the library) so the server's copies
overlap the integration of other requests.
"""

from __future__ import annotations

import contextlib
import ctypes
import threading

import numpy as np

from . import capi


class ServerOptions(ctypes.Structure):
    _fields_ = [
        ("memory_fraction", ctypes.c_double),
        ("memory_bytes", ctypes.c_size_t),
        ("streams", ctypes.c_int32),
        ("sm_reserve_percent", ctypes.c_int32),
        ("max_batch_particles", ctypes.c_int64),
        ("select_device", ctypes.c_int32),
        ("device", ctypes.c_int32),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "requests_submitted", "requests_completed", "requests_pending", "particles_completed",
        "batches_launched", "pieces_launched", "batches_in_flight", "bytes_to_device",
        "bytes_to_host", "memory_budget", "bytes_in_flight", "peak_bytes_in_flight",
        "bytes_pending")] + [("device", ctypes.c_int32), ("reserved", ctypes.c_int32)]


def _lib():
    L = capi.lib()
    if not getattr(L, "_server_bound", False):
        L.drift_server_create.argtypes = [ctypes.POINTER(ServerOptions), ctypes.POINTER(ctypes.c_void_p)]
        L.drift_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(capi.DriftLaunch),
                                          ctypes.POINTER(ctypes.c_uint64)]
        L.drift_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        L.drift_server_stats_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(ServerStats)]
        L.drift_server_wait_any.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int32,
                                            ctypes.c_double, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        L.drift_server_cancel.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.drift_server_destroy.argtypes = [ctypes.c_void_p]
        L._server_bound = True
    return L


class PinnedArray:
    """A numpy view of page-locked host memory from drift_host_alloc."""

    def __init__(self, shape, dtype=np.float64):
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = ctypes.c_void_p()
        capi.check(capi.lib().drift_host_alloc(max(self.nbytes, 1), ctypes.byref(self.ptr)),
                   "drift_host_alloc")
        buf = (ctypes.c_char * max(self.nbytes, 1)).from_address(self.ptr.value)
        buf._owner = self  # the numpy view keeps this object, hence the memory, alive
        self.array = np.frombuffer(buf, dtype=dtype, count=int(np.prod(shape))).reshape(shape)

    def free(self):
        if self.ptr:
            capi.lib().drift_host_free(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class RequestCancelled(RuntimeError):
    """The request was cancelled before all its particles ran."""


class Request:
    def __init__(self, server, ticket, keep, arrays):
        self.server, self.ticket, self._keep, self.arrays = server, ticket, keep, arrays

    def cancel(self) -> None:
        """Stop admitting this request's particles (drift_server_cancel);
        wait() then raises RequestCancelled once the particles already on the
        GPU have finished."""
        with self.server._call() as ptr:
            capi.check(_lib().drift_server_cancel(ptr, self.ticket), "drift_server_cancel")

    def wait(self, timeout: float = 0.0) -> dict:
        """Block until the request completes; ``timeout`` > 0 bounds the wait
        (RuntimeError with the library's timeout message when it runs out;
        the request stays valid and can be waited for again)."""
        result = ctypes.c_int(0)
        latency = ctypes.c_double(0.0)
        with self.server._call() as ptr:
            capi.check(_lib().drift_server_wait(ptr, self.ticket, timeout, ctypes.byref(result),
                                                ctypes.byref(latency)), "drift_server_wait")
        return self._finish(result.value, latency.value)

    def _finish(self, result: int, latency: float) -> dict:
        # the ticket has been released: results or the request's error
        self.server._released(self.ticket)
        self._keep = None
        if result == 7:  # DRIFT_ERROR_CANCELLED
            raise RequestCancelled("request cancelled")
        if result != 0:
            raise RuntimeError(f"request failed: {capi.lib().drift_result_string(result).decode()}")
        out = dict(self.arrays)
        out["latency_s"] = latency
        return out


class Server:
    def __init__(self, memory_fraction: float = 0.5, memory_bytes: int = 0, streams: int = 4,
                 max_batch_particles: int = 1 << 20, sm_reserve_percent: int = 0,
                 device: int | None = None):
        """sm_reserve_percent: share of the SMs (0 to 50) large batches leave
        to small ones, which run on the high-priority stream (default none).
        ``device``: the CUDA device index the server runs on (default: the
        current device)."""
        opts = ServerOptions(memory_fraction=memory_fraction, memory_bytes=memory_bytes,
                             streams=streams, max_batch_particles=max_batch_particles,
                             sm_reserve_percent=sm_reserve_percent,
                             select_device=int(device is not None),
                             device=int(device) if device is not None else 0)
        self._ptr = ctypes.c_void_p()
        # Calls in progress and tickets not yet waited for: close() cancels
        # the tickets and lets every call return before freeing the server.
        self._cond = threading.Condition()
        self._calls = 0
        self._closing = False
        self._tickets: set[int] = set()
        capi.check(_lib().drift_server_create(ctypes.byref(opts), ctypes.byref(self._ptr)),
                   "drift_server_create")
        self.device_index = self.stats()["device"]

    @contextlib.contextmanager
    def _call(self):
        """The server pointer for one C call, which close() waits for."""
        with self._cond:
            if not self._ptr or self._closing:
                raise RuntimeError("the server is closed")
            self._calls += 1
        try:
            yield self._ptr
        finally:
            with self._cond:
                self._calls -= 1
                self._cond.notify_all()

    def _released(self, ticket: int) -> None:
        with self._cond:
            self._tickets.discard(ticket)

    def submit(self, method, pot, y0, *, ts=None, t_end=None, nt=None, t0=0.0, rtol=1e-12,
               atol=1e-12, precision=capi.EXACT, schedule=capi.ORDERED, out=None,
               want_out=True) -> Request:
        """Queue one request.  ``schedule``: ORDERED batches rank their
        particles most expensive first; PLAIN and PERSISTENT requests share a
        persistent claim queue."""
        y0 = np.ascontiguousarray(y0, dtype=np.float64).reshape(-1, 6)
        n = y0.shape[0]
        if ts is not None:
            ts = np.ascontiguousarray(ts, dtype=np.float64)
            nt = len(ts)
        else:
            t_end = np.ascontiguousarray(t_end, dtype=np.float64)
        L = capi.make_launch(method, pot, n, nt, rtol=rtol, atol=atol, precision=precision,
                             schedule=schedule, t0=t0)
        # Page-locked so the server's copies run asynchronously.
        arrays = dict(
            y_final=PinnedArray((n, 6)).array, status=PinnedArray((n,), np.uint8).array,
            err=PinnedArray((n,), np.int32).array, accepted=PinnedArray((n,), np.uint32).array,
            rejected=PinnedArray((n,), np.uint32).array)
        pinned = None
        if want_out:
            if out is None:
                pinned = PinnedArray((nt, n, 6))
                out = pinned.array
                pinned = None  # lifetime follows the returned array
            arrays["out"] = out
        L.y0, L.ts, L.t_end = y0.ctypes.data, (ts.ctypes.data if ts is not None else None), (
            t_end.ctypes.data if t_end is not None else None)
        L.out = out.ctypes.data if want_out else None
        L.y_final = arrays["y_final"].ctypes.data
        L.status, L.err_code = arrays["status"].ctypes.data, arrays["err"].ctypes.data
        L.n_accepted, L.n_rejected = arrays["accepted"].ctypes.data, arrays["rejected"].ctypes.data
        ticket = ctypes.c_uint64(0)
        with self._call() as ptr:
            capi.check(_lib().drift_server_submit(ptr, ctypes.byref(L), ctypes.byref(ticket)),
                       "drift_server_submit")
            with self._cond:
                self._tickets.add(ticket.value)
        return Request(self, ticket.value, (y0, ts, t_end, L, pinned), arrays)

    def wait_any(self, requests, timeout: float = 0.0) -> tuple[int, dict]:
        """Block until any of ``requests`` completes (drift_server_wait_any)
        and return (its index in ``requests``, its results).  The others stay
        pending and can be waited for again.  ``timeout`` as Request.wait; a
        failed or cancelled request raises as Request.wait does."""
        requests = list(requests)
        got = self._wait_any(requests, timeout, poll=False)
        return got[0], requests[got[0]]._finish(got[1], got[2])

    def _wait_any(self, requests, timeout: float, poll: bool):
        """drift_server_wait_any over ``requests`` (all of this server):
        (index, drift_result, latency), or None when ``poll`` and the timeout
        ran out (otherwise that raises like any other error)."""
        tickets = (ctypes.c_uint64 * len(requests))(*[r.ticket for r in requests])
        index, result, latency = ctypes.c_int32(-1), ctypes.c_int(0), ctypes.c_double(0.0)
        with self._call() as ptr:
            rc = _lib().drift_server_wait_any(ptr, tickets, len(requests), timeout, ctypes.byref(index),
                                              ctypes.byref(result), ctypes.byref(latency))
        if poll and rc == 6:  # DRIFT_ERROR_TIMEOUT: nothing finished yet
            return None
        capi.check(rc, "drift_server_wait_any")
        return index.value, result.value, latency.value

    def stats(self) -> dict:
        st = ServerStats()
        with self._call() as ptr:
            capi.check(_lib().drift_server_stats_get(ptr, ctypes.byref(st)), "drift_server_stats_get")
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}

    def close(self):
        """Cancels the requests not yet waited for (drift_server_cancel: those
        with particles on the GPU finish them), lets every call in progress on
        other threads return (their waits end with the result or
        RequestCancelled), then destroys the server.  Later calls raise."""
        with self._cond:
            if not self._ptr or self._closing:
                return
            self._closing = True
            tickets = sorted(self._tickets)
            ptr = self._ptr
        for t in tickets:
            _lib().drift_server_cancel(ptr, t)  # a ticket released meanwhile only reports an error
        with self._cond:
            self._cond.wait_for(lambda: self._calls == 0)
        _lib().drift_server_destroy(ptr)
        with self._cond:
            self._ptr = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def request_bytes(n: int, nt: int, *, shared_grid: bool = True, want_out: bool = True) -> int:
    """Device bytes a whole request of ``n`` particles and ``nt`` samples
    needs on a server (the sum the server's admission reserves for it: state,
    grid, trajectory, final state and per-particle counters, each rounded to
    256 bytes)."""
    def up(b):
        return (b + 255) // 256 * 256
    b = up(n * 48) + up(nt * 8 if shared_grid else n * 8) + up(n * 48) + up(n) + 3 * up(n * 4)
    if want_out:
        b += up(nt * n * 48)
    return b


def route(free_bytes, pending_requests, need: int) -> int:
    """Index of the server a request needing ``need`` device bytes goes to.

    The server with the most free device memory (budget minus bytes in
    flight minus bytes queued) wins; ties go to the one with fewer queued
    requests, then the lower index.  A request larger than every server's
    free memory still goes to the freest one, which runs it in particle
    chunks as memory frees up."""
    if not free_bytes:
        raise ValueError("no servers")
    if len(free_bytes) != len(pending_requests):
        raise ValueError("free_bytes and pending_requests differ in length")
    del need  # the ranking does not depend on the request's size
    return min(range(len(free_bytes)), key=lambda i: (-int(free_bytes[i]), int(pending_requests[i]), i))


class Router:
    """Whole requests to one of several servers, typically one per GPU of a
    node, by free device memory.

        with Router.on_devices([0, 1, 2, 3], memory_fraction=0.5) as rt:
            req = rt.submit(capi.DOP853, capi.plummer(), y0, ts=ts)
            res = req.wait()       # res["device"] is the GPU that ran it

    A request never splits across servers: its particles stay on one GPU,
    so its results equal drift_integrate_host's on that GPU."""

    def __init__(self, servers):
        self.servers = list(servers)
        if not self.servers:
            raise ValueError("a router needs at least one server")
        self.routed = [0] * len(self.servers)

    @classmethod
    def on_devices(cls, devices=None, **server_kwargs) -> "Router":
        """One server per CUDA device index in ``devices`` (default: every
        visible device)."""
        if devices is None:
            import torch

            devices = range(torch.cuda.device_count())
        servers = []
        try:
            for d in devices:
                servers.append(Server(device=int(d), **server_kwargs))
        except Exception:
            for s in servers:
                s.close()
            raise
        return cls(servers)

    def pick(self, need: int) -> int:
        free, queued = [], []
        for s in self.servers:
            st = s.stats()
            used = st["bytes_in_flight"] + st["bytes_pending"]
            free.append(max(st["memory_budget"] - used, 0))
            queued.append(st["requests_pending"])
        return route(free, queued, need)

    def submit(self, method, pot, y0, *, ts=None, t_end=None, nt=None, want_out=True, **kwargs) -> Request:
        n = int(np.asarray(y0).size // 6)
        samples = len(ts) if ts is not None else int(nt)
        i = self.pick(request_bytes(n, samples, shared_grid=ts is not None, want_out=want_out))
        self.routed[i] += 1
        server = self.servers[i]
        req = server.submit(method, pot, y0, ts=ts, t_end=t_end, nt=nt, want_out=want_out, **kwargs)
        req.arrays["device"] = server.device_index
        req.arrays["server"] = i
        return req

    def stats(self) -> list[dict]:
        return [s.stats() for s in self.servers]

    def wait_any(self, requests, timeout: float = 0.0, poll_s: float = 1e-3) -> tuple[int, dict]:
        """Server.wait_any across servers: (index in ``requests``, results)
        of the first request to finish.  Requests of one server wait in one
        call; requests spread over several servers are polled, each server's
        wait bounded by ``poll_s``, until one finishes or ``timeout`` (> 0)
        runs out (RuntimeError)."""
        import time

        requests = list(requests)
        if not requests:
            raise ValueError("no requests to wait for")
        groups: dict[int, list[int]] = {}
        for i, r in enumerate(requests):
            groups.setdefault(id(r.server), []).append(i)
        if len(groups) == 1:
            return requests[0].server.wait_any(requests, timeout)
        deadline = time.monotonic() + timeout if timeout > 0 else None
        while True:
            for idx in groups.values():
                server = requests[idx[0]].server
                got = server._wait_any([requests[i] for i in idx], poll_s, poll=True)
                if got is not None:
                    i = idx[got[0]]
                    return i, requests[i]._finish(got[1], got[2])
            if deadline is not None and time.monotonic() > deadline:
                raise RuntimeError("drift_server_wait_any: every request still running")

    def close(self):
        for s in self.servers:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
