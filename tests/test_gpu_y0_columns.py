"""Initial states as six columns (DRIFT_Y0_COLUMNS) give exactly the results
of the same states as (n, 6) rows: on device pointers (with a padded column
stride and the ordered schedule, whose cost ranking reads the states too),
through the chunked host path, and inside a batch that mixes both layouts.
The request server takes rows only."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


def _states(n, seed=0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 2.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(u, rng.normal(size=(n, 3)))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return np.hstack([u * r[:, None], v * (0.8 / np.sqrt(r))[:, None]])


def _device_run(torch, method, pot, y0_rows, ts, columns, pad=0):
    dev = torch.device("cuda:0")
    n = len(y0_rows)
    if columns:
        host = np.zeros((6, n + pad))
        host[:, :n] = y0_rows.T
    else:
        host = y0_rows
    y0 = torch.tensor(host, device=dev)
    ts_d = torch.tensor(ts, device=dev)
    out = torch.empty((len(ts), n, 6), dtype=torch.float64, device=dev)
    acc = torch.zeros(n, dtype=torch.int32, device=dev)
    L = capi.make_launch(method, pot, n, len(ts), rtol=1e-10, atol=1e-10, schedule=capi.ORDERED,
                         precision=capi.FMA)
    L.y0, L.ts, L.out, L.n_accepted = y0.data_ptr(), ts_d.data_ptr(), out.data_ptr(), acc.data_ptr()
    if columns:
        L.y0_layout, L.y0_stride = capi.Y0_COLUMNS, n + pad
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy(), acc.cpu().numpy()


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
def test_columns_equal_rows_on_device_pointers(cuda_device, method):
    import torch

    y0 = _states(5000, 1)
    ts = np.linspace(0.0, 6.0, 13)
    rows = _device_run(torch, method, capi.bovy(), y0, ts, columns=False)
    cols = _device_run(torch, method, capi.bovy(), y0, ts, columns=True, pad=37)
    np.testing.assert_array_equal(cols[0], rows[0])
    np.testing.assert_array_equal(cols[1], rows[1])
    assert np.isfinite(rows[0]).all()


def test_columns_equal_rows_through_the_chunked_host_path(cuda_device):
    y0 = _states(70000, 2)  # above the host path's chunking threshold
    ts = np.linspace(0.0, 4.0, 21)
    rows = capi.integrate_host(capi.DOP853, capi.plummer(), y0, ts=ts, rtol=1e-10, atol=1e-10)
    cols = capi.integrate_host(capi.DOP853, capi.plummer(), y0.T.copy(), ts=ts, rtol=1e-10, atol=1e-10,
                               columns=True)
    for k in ("out", "y_final", "accepted", "status"):
        np.testing.assert_array_equal(cols[k], rows[k])


def test_a_batch_can_mix_rows_and_columns(cuda_device):
    import torch

    dev = torch.device("cuda:0")
    ts = np.linspace(0.0, 5.0, 9)
    ts_d = torch.tensor(ts, device=dev)
    parts = [_states(300, 3), _states(700, 4)]
    keep, launches = [], []
    for i, y in enumerate(parts):
        host = y.T.copy() if i == 1 else y
        y0 = torch.tensor(host, device=dev)
        out = torch.empty((len(ts), len(y), 6), dtype=torch.float64, device=dev)
        L = capi.make_launch(capi.DOP853, capi.plummer(), len(y), len(ts), rtol=1e-10, atol=1e-10,
                             schedule=capi.PERSISTENT)
        L.y0, L.ts, L.out = y0.data_ptr(), ts_d.data_ptr(), out.data_ptr()
        if i == 1:
            L.y0_layout = capi.Y0_COLUMNS
        keep.append((y0, out))
        launches.append(L)
    probe = capi.make_launch(capi.DOP853, capi.plummer(), 1000, 2, rtol=1e-10, atol=1e-10,
                             schedule=capi.PERSISTENT)
    ws = torch.zeros(max(capi.query_workspace(probe), 8), dtype=torch.uint8, device=dev)
    launches[0].workspace, launches[0].workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_batch_device(launches, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for y, (_, out) in zip(parts, keep):
        ref = capi.integrate_host(capi.DOP853, capi.plummer(), y, ts=ts, rtol=1e-10, atol=1e-10)
        np.testing.assert_array_equal(out.cpu().numpy(), ref["out"])


def test_the_server_refuses_columns(cuda_device):
    import ctypes

    from astrodrift_b200.serving import Server, _lib

    y0 = np.ascontiguousarray(_states(10, 5).T)
    ts = np.linspace(0.0, 1.0, 3)
    L = capi.make_launch(capi.DOP853, capi.plummer(), 10, 3, rtol=1e-10, atol=1e-10)
    L.y0, L.ts = y0.ctypes.data, ts.ctypes.data
    L.y0_layout = capi.Y0_COLUMNS
    with Server(memory_bytes=16 << 20) as srv:
        ticket = ctypes.c_uint64(0)
        rc = _lib().drift_server_submit(srv._ptr, ctypes.byref(L), ctypes.byref(ticket))
        assert rc == 1
        assert "rows" in capi.lib().drift_last_error().decode()
