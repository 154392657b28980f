"""Captured launch graphs (drift_graph_*) and the launch autotuner
(drift_autotune), through the C ABI.

* A graph replays the launch bit for bit, and picks up new initial states
  written in place between replays.
* The autotuner measures all twelve candidates on a sample, prefers a
  work-stealing schedule on a workload whose particles differ in cost by two
  decades and outnumber the resident lanes, caches its answer per workload
  class, and leaves the caller's outputs alone; its choice integrates to the
  same bits (exact arithmetic makes every schedule and block size agree).
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


def _plummer_ics(n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.2, 3.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(u, rng.normal(size=(n, 3)))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    vc = np.sqrt(r * r / (r * r + 1.0) ** 1.5) * rng.uniform(0.5, 1.1, n)
    return np.hstack([u * r[:, None], v * vc[:, None]])


def _launch(torch, y0_d, ts_d, out_d, schedule=capi.ORDERED, block=0, n=None):
    n = n or y0_d.shape[0]
    L = capi.make_launch(capi.DOP853, capi.plummer(1.0, 1.0), n, ts_d.numel(), rtol=1e-10, atol=1e-10,
                         schedule=schedule, block_size=block)
    L.y0, L.ts, L.out = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr()
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=y0_d.device)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    return L, ws


def test_graph_replays_bitwise_and_follows_in_place_inputs(cuda_device):
    import torch

    dev = torch.device("cuda:0")
    s = torch.cuda.Stream()
    a, b = _plummer_ics(3000, 1), _plummer_ics(3000, 2)
    ts_d = torch.tensor(np.linspace(0.0, 8.0, 9), device=dev)
    y0_d = torch.tensor(a, device=dev)
    out_d = torch.empty((9, 3000, 6), dtype=torch.float64, device=dev)
    ref_d = torch.empty_like(out_d)
    with torch.cuda.stream(s):
        L_ref, ws_ref = _launch(torch, y0_d, ts_d, ref_d)
        capi.integrate_device(L_ref, s.cuda_stream)  # also creates the library context
        L, ws = _launch(torch, y0_d, ts_d, out_d)
        g = capi.Graph(L, s.cuda_stream)
        g.replay(s.cuda_stream)
    s.synchronize()
    np.testing.assert_array_equal(out_d.cpu().numpy(), ref_d.cpu().numpy())
    with torch.cuda.stream(s):
        y0_d.copy_(torch.tensor(b, device=dev))
        g.replay(s.cuda_stream)
        g.replay(s.cuda_stream)  # idempotent: the cursor is reset inside the graph
        capi.integrate_device(L_ref, s.cuda_stream)
    s.synchronize()
    np.testing.assert_array_equal(out_d.cpu().numpy(), ref_d.cpu().numpy())
    assert not np.array_equal(out_d[-1].cpu().numpy(), a)
    g.close()


def test_autotune_picks_work_stealing_for_uneven_workloads_and_caches(cuda_device):
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(5)
    n = 150000  # well above the ~57,000 resident lanes, so queues matter
    y0 = _plummer_ics(n, 5)
    t_end = np.exp(rng.uniform(np.log(1.0), np.log(300.0), n))  # two decades of span
    y0_d = torch.tensor(y0, device=dev)
    te_d = torch.tensor(t_end, device=dev)
    out_d = torch.full((5, n, 6), 7.0, dtype=torch.float64, device=dev)
    L = capi.make_launch(capi.DOP853, capi.plummer(1.0, 1.0), n, 5, rtol=1e-10, atol=1e-10)
    L.y0, L.t_end, L.out = y0_d.data_ptr(), te_d.data_ptr(), out_d.data_ptr()
    t = capi.autotune(L, sample=n)
    assert t.cached == 0 and t.sample == n
    cand = np.array(list(t.candidates))
    assert (cand > 0).all() and t.seconds == cand.min()
    assert t.schedule in (capi.PERSISTENT, capi.ORDERED)
    assert cand[:4].min() > 1.5 * t.seconds  # every plain launch loses clearly
    assert (out_d == 7.0).all()  # the caller's outputs are untouched
    again = capi.autotune(L, sample=n)
    assert again.cached == 1 and again.block_size == t.block_size and again.schedule == t.schedule

    # the tuned launch integrates to the same bits as the default
    ref = capi.integrate_host(capi.DOP853, capi.plummer(1.0, 1.0), y0[:2000], t_end=t_end[:2000], nt=5,
                              rtol=1e-10, atol=1e-10)
    got = capi.integrate_host(capi.DOP853, capi.plummer(1.0, 1.0), y0[:2000], t_end=t_end[:2000], nt=5,
                              rtol=1e-10, atol=1e-10, schedule=t.schedule, block_size=t.block_size)
    np.testing.assert_array_equal(got["out"], ref["out"])


def test_autotune_choice_persists_in_a_json_cache(cuda_device, tmp_path):
    import json

    import torch

    dev = torch.device("cuda:0")
    n = 4096
    y0_d = torch.tensor(_plummer_ics(n, 9), device=dev)
    ts_d = torch.tensor(np.linspace(0.0, 3.0, 7), device=dev)
    L = capi.make_launch(capi.DOPR54, capi.plummer(1.0, 1.0), n, 7, rtol=1e-9, atol=1e-9)
    L.y0, L.ts = y0_d.data_ptr(), ts_d.data_ptr()
    path = tmp_path / "tuning.json"
    first = capi.autotune(L, cache_path=str(path))
    assert first.cached in (0, 1)  # timed now, or earlier in this process
    table = json.loads(path.read_text())
    assert table[capi.tuning_key(L)]["block_size"] == first.block_size
    again = capi.autotune(L, cache_path=str(path))
    assert again.cached == 2 and (again.block_size, again.schedule) == (first.block_size, first.schedule)
