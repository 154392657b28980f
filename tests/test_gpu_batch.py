"""drift_integrate_batch: several requests in one launch give each request the
result it gets alone.

Requests of different sizes, output grids (shared and per-particle end times)
and time spans are concatenated into one launch under each schedule; in
exact arithmetic every particle's integration is independent of the launch
that runs it, so every output must equal the single-request launch's bit for
bit.  The ordered schedule ranks the particles of all requests together.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


def _requests(rng, count=5):
    reqs = []
    for i in range(count):
        n = [1, 37, 1000, 4097, 250][i % 5]
        r = rng.uniform(0.2, 3.0, n)
        u = rng.normal(size=(n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        v = np.cross(u, rng.normal(size=(n, 3)))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        vc = np.sqrt(r * r / (r * r + 1.0) ** 1.5) * rng.uniform(0.3, 1.1, n)
        y0 = np.hstack([u * r[:, None], v * vc[:, None]])
        nt = [2, 17, 9, 33, 5][i % 5]
        if i % 2:
            reqs.append(dict(y0=y0, t_end=rng.uniform(1.0, 40.0, n), nt=nt))
        else:
            reqs.append(dict(y0=y0, ts=np.linspace(0.0, rng.uniform(1.0, 40.0), nt)))
    return reqs


def _launch(torch, method, pot, req, schedule, dev):
    y0 = torch.tensor(req["y0"], device=dev)
    n = len(req["y0"])
    nt = req.get("nt") or len(req["ts"])
    grid = torch.tensor(req["ts"] if "ts" in req else req["t_end"], device=dev)
    out = torch.full((nt, n, 6), float("nan"), dtype=torch.float64, device=dev)
    acc = torch.zeros(n, dtype=torch.int32, device=dev)
    fin = torch.zeros((n, 6), dtype=torch.float64, device=dev)
    L = capi.make_launch(method, pot, n, nt, rtol=1e-10, atol=1e-10, schedule=schedule)
    L.y0, L.out, L.n_accepted, L.y_final = y0.data_ptr(), out.data_ptr(), acc.data_ptr(), fin.data_ptr()
    if "ts" in req:
        L.ts = grid.data_ptr()
    else:
        L.t_end = grid.data_ptr()
    return L, (y0, grid, out, acc, fin)


def _alone(torch, method, pot, req, dev):
    L, keep = _launch(torch, method, pot, req, capi.PLAIN, dev)
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return [t.cpu().numpy() for t in keep[2:]]


@pytest.mark.parametrize("schedule", [capi.PLAIN, capi.PERSISTENT, capi.ORDERED])
@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
def test_batch_equals_each_request_alone(cuda_device, schedule, method):
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(31 + schedule)
    pot = capi.plummer(1.0, 1.0)
    reqs = _requests(rng)
    launches, keeps = [], []
    for req in reqs:
        L, keep = _launch(torch, method, pot, req, schedule, dev)
        launches.append(L)
        keeps.append(keep)
    total = sum(len(r["y0"]) for r in reqs)
    probe = capi.make_launch(method, pot, total, 2, rtol=1e-10, atol=1e-10, schedule=schedule)
    ws = torch.zeros(max(capi.query_workspace(probe), 8), dtype=torch.uint8, device=dev)
    launches[0].workspace, launches[0].workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_batch_device(launches, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for req, keep in zip(reqs, keeps):
        got = [t.cpu().numpy() for t in keep[2:]]
        ref = _alone(torch, method, pot, req, dev)
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g, r)
        assert np.isfinite(got[0]).all()


def test_ordered_batch_rejects_a_workspace_for_one_request(cuda_device):
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(5)
    pot = capi.plummer(1.0, 1.0)
    reqs = _requests(rng, count=3)
    launches, keeps = [], []
    for req in reqs:
        L, keep = _launch(torch, capi.DOP853, pot, req, capi.ORDERED, dev)
        launches.append(L)
        keeps.append(keep)
    # sized for the first request only: too small for all three
    ws = torch.zeros(capi.query_workspace(launches[0]), dtype=torch.uint8, device=dev)
    launches[0].workspace, launches[0].workspace_bytes = ws.data_ptr(), ws.numel()
    arr = (capi.DriftLaunch * 3)(*launches)
    rc = capi.lib().drift_integrate_batch(arr, 3, ctypes.c_void_p(0))
    assert rc == 3  # DRIFT_ERROR_WORKSPACE
    assert "workspace" in capi.lib().drift_last_error().decode()


@pytest.mark.parametrize("precision", [capi.EXACT, capi.FMA])
def test_sparse_output_skip_leaves_results_unchanged(cuda_device, precision):
    """A grid of at most 8 output times lets DOP853 skip the dense-output
    stages of steps that emit nothing; alone, such a request runs that way,
    batched with a dense request it does not.  Both runs must agree bit for
    bit (Bovy force: the step with the looped extra stages)."""
    import torch

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(8)
    pot = capi.bovy()
    reqs = _requests(rng, count=2)
    reqs[0]["ts"] = np.linspace(0.0, 30.0, 3)           # sparse
    reqs[1] = dict(y0=reqs[1]["y0"], ts=np.linspace(0.0, 20.0, 40))  # dense
    outs = []
    for batched in (False, True):
        launches, keeps = [], []
        for req in (reqs if batched else reqs[:1]):
            L, keep = _launch(torch, capi.DOP853, pot, req, capi.PERSISTENT, dev)
            L.precision = precision
            launches.append(L)
            keeps.append(keep)
        total = sum(len(r["y0"]) for r in reqs)
        probe = capi.make_launch(capi.DOP853, pot, total, 2, rtol=1e-10, atol=1e-10,
                                 schedule=capi.PERSISTENT)
        ws = torch.zeros(max(capi.query_workspace(probe), 8), dtype=torch.uint8, device=dev)
        launches[0].workspace, launches[0].workspace_bytes = ws.data_ptr(), ws.numel()
        capi.integrate_batch_device(launches, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs.append([t.cpu().numpy() for t in keeps[0][2:]])
    for a, b in zip(*outs):
        np.testing.assert_array_equal(a, b)
    assert np.isfinite(outs[0][0]).all()
