"""Canary padding: every buffer a launch writes sits between guard regions
filled with a sentinel, and no launch may touch them.  With the sanitizer
closed on this hardware, this is the out-of-bounds check for the kernels'
index arithmetic: ragged particle counts, both grids, all schedules, the step
tape, batched segments, the no-allocation entry point and failing particles
(whose unreached samples are filled with NaN)."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu

G = 64                      # guard elements on each side (512 B for doubles: keeps 16-byte alignment)
SENT = -1.2345678910111213e300
SENT_U8 = 0xA5


class Guarded:
    """A device buffer of `count` elements between two guard regions."""

    def __init__(self, torch, count, dtype, dev):
        self.torch, self.count = torch, count
        fill = SENT_U8 if dtype in (torch.uint8,) else (0x5A5A5A5A if dtype in (torch.int32,) else SENT)
        self.full = torch.full((count + 2 * G,), fill, dtype=dtype, device=dev)
        self.fill = fill

    def ptr(self):
        return self.full.data_ptr() + G * self.full.element_size()

    def inner(self):
        return self.full[G:G + self.count]

    def guards_intact(self):
        t = self.torch
        head, tail = self.full[:G], self.full[G + self.count:]
        return bool(t.all(head == self.fill)) and bool(t.all(tail == self.fill))


def _states(n, seed, bad=0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 2.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    u[:, 2] *= 0.3
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(u, rng.normal(size=(n, 3)))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    y = np.hstack([u * r[:, None], v * (0.8 / np.sqrt(r))[:, None]])
    y[:bad] = np.nan  # failing particles: NONFINITE, NaN-filled samples
    return y


def _guarded_launch(torch, dev, method, n, nt, schedule, per_particle, seed, tape_steps=0, bad=0):
    y0 = torch.tensor(_states(n, seed, bad), device=dev)
    rng = np.random.default_rng(seed + 1)
    grid = torch.tensor(rng.uniform(1.0, 6.0, n) if per_particle else np.linspace(0.0, 5.0, nt), device=dev)
    bufs = dict(
        out=Guarded(torch, nt * n * 6, torch.float64, dev),
        y_final=Guarded(torch, n * 6, torch.float64, dev),
        status=Guarded(torch, n, torch.uint8, dev),
        err=Guarded(torch, n, torch.int32, dev),
        acc=Guarded(torch, n, torch.int32, dev),
        rej=Guarded(torch, n, torch.int32, dev),
    )
    L = capi.make_launch(method, capi.plummer(), n, nt, rtol=1e-9, atol=1e-9, schedule=schedule)
    L.y0 = y0.data_ptr()
    if per_particle:
        L.t_end = grid.data_ptr()
    else:
        L.ts = grid.data_ptr()
    L.out, L.y_final = bufs["out"].ptr(), bufs["y_final"].ptr()
    L.status, L.err_code = bufs["status"].ptr(), bufs["err"].ptr()
    L.n_accepted, L.n_rejected = bufs["acc"].ptr(), bufs["rej"].ptr()
    if tape_steps:
        bufs["tape"] = Guarded(torch, n * capi.tape_doubles(tape_steps, 1), torch.float64, dev)
        L.tape, L.tape_steps = bufs["tape"].ptr(), tape_steps
    need = capi.query_workspace(L)
    if need:
        bufs["ws"] = Guarded(torch, need, torch.uint8, dev)
        L.workspace, L.workspace_bytes = bufs["ws"].ptr(), need
    return L, bufs, (y0, grid)


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
@pytest.mark.parametrize("schedule", [capi.PLAIN, capi.PERSISTENT, capi.ORDERED])
@pytest.mark.parametrize("per_particle", [False, True])
def test_launches_stay_inside_their_buffers(cuda_device, method, schedule, per_particle):
    import torch

    dev = torch.device("cuda:0")
    n, nt = 1237, 9  # ragged: not a multiple of any block size
    tape = 400 if method == capi.DOP853 else 0
    L, bufs, keep = _guarded_launch(torch, dev, method, n, nt, schedule, per_particle, seed=n + schedule,
                                    tape_steps=tape, bad=3)
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for name, b in bufs.items():
        assert b.guards_intact(), name
    out = bufs["out"].inner().view(nt, n, 6).cpu().numpy()
    status = bufs["status"].inner().cpu().numpy()
    assert (status[3:] == 0).all() and (status[:3] != 0).all()
    assert np.isfinite(out[:, 3:]).all() and np.isnan(out[1:, :3]).all()


def test_batched_segments_and_the_no_allocation_entry_stay_inside(cuda_device):
    import torch

    dev = torch.device("cuda:0")
    launches, all_bufs, keep = [], [], []
    for i, (n, nt, pp) in enumerate(((33, 5, False), (517, 12, True), (1, 3, False))):
        L, bufs, k = _guarded_launch(torch, dev, capi.DOP853, n, nt, capi.ORDERED, pp, seed=10 + i)
        launches.append(L)
        all_bufs.append(bufs)
        keep.append(k)
    total = 33 + 517 + 1
    probe = capi.make_launch(capi.DOP853, capi.plummer(), total, 2, rtol=1e-9, atol=1e-9,
                             schedule=capi.ORDERED)
    ws = Guarded(torch, capi.query_workspace(probe), torch.uint8, dev)
    launches[0].workspace, launches[0].workspace_bytes = ws.ptr(), ws.count
    capi.integrate_batch_device(launches, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert ws.guards_intact()
    for bufs in all_bufs:
        for name, b in bufs.items():
            if name != "ws":
                assert b.guards_intact(), name

    L, bufs, k = _guarded_launch(torch, dev, capi.DOP853, 999, 7, capi.PERSISTENT, False, seed=20)
    L.workspace, L.workspace_bytes = None, 0
    capi.integrate_device_noalloc(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for name, b in bufs.items():
        if name != "ws":
            assert b.guards_intact(), name


def test_host_path_writes_only_the_callers_trajectory_block():
    y0 = _states(70001, 30)  # chunked, ragged last chunk
    nt = 6
    big = np.full(nt * len(y0) * 6 + 2 * G, SENT)
    out = big[G:G + nt * len(y0) * 6].reshape(nt, len(y0), 6)
    capi.integrate_host(capi.DOP853, capi.plummer(), y0, ts=np.linspace(0.0, 2.0, nt), rtol=1e-9, atol=1e-9,
                        out=out)
    assert (big[:G] == SENT).all() and (big[-G:] == SENT).all()
    assert np.isfinite(out).all()


test_host_path_writes_only_the_callers_trajectory_block = pytest.mark.usefixtures("cuda_device")(
    test_host_path_writes_only_the_callers_trajectory_block)
