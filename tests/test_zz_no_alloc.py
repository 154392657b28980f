"""The no-allocation entry point, drift_integrate_noalloc, through the C ABI.

Callers that own all device memory themselves (a pre-reserved memory pool, a
real-time loop that cannot afford an allocation's synchronisation, a plugin
inside a runtime that forbids allocation) integrate through
drift_integrate_noalloc, which keeps its scratch in a fixed array inside the
library instead of a caller-provided workspace.  Its results must match
drift_integrate's, on two calls in a row (the array keeps the previous call's
contents, so the second call checks that the scratch is cleared).

This file sorts last so that a run stopping at its first failure has already
run every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a).reshape(-1, 6)
    b = np.asarray(b).reshape(-1, 6)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def _case(torch, method, pot, y0, ts, schedule):
    dev = torch.device("cuda:0")
    n, nt = len(y0), len(ts)
    y0_d = torch.tensor(y0, device=dev)
    ts_d = torch.tensor(ts, device=dev)

    def launch(out_d, acc_d):
        L = capi.make_launch(method, pot, n, nt, rtol=1e-11, atol=1e-11, schedule=schedule)
        L.y0, L.ts, L.out, L.n_accepted = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr(), acc_d.data_ptr()
        return L

    stream = torch.cuda.current_stream().cuda_stream
    # the existing entry point, with a caller-allocated workspace
    out_ref = torch.empty((nt, n, 6), dtype=torch.float64, device=dev)
    acc_ref = torch.zeros(n, dtype=torch.int32, device=dev)
    L = launch(out_ref, acc_ref)
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, stream)
    torch.cuda.synchronize()
    ref = out_ref.cpu().numpy()
    ref_acc = acc_ref.cpu().numpy()
    assert np.isfinite(ref).all()

    # the no-allocation entry point, twice in a row
    for _ in range(2):
        out = torch.full((nt, n, 6), float("nan"), dtype=torch.float64, device=dev)
        acc = torch.zeros(n, dtype=torch.int32, device=dev)
        capi.integrate_device_noalloc(launch(out, acc), stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_err(got, ref) < REL_TOL
        np.testing.assert_array_equal(acc.cpu().numpy(), ref_acc)


@pytest.mark.parametrize("schedule", [capi.PERSISTENT, capi.PLAIN])
def test_noalloc_matches_drift_integrate_dop853_plummer(cuda_device, schedule):
    import torch

    rng = np.random.default_rng(17)
    n = 3001
    r = rng.uniform(0.2, 3.0, n)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    v = np.cross(u, rng.normal(size=(n, 3)))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    vc = np.sqrt(r * r / (r * r + 1.0) ** 1.5) * rng.uniform(0.5, 1.1, n)
    y0 = np.hstack([u * r[:, None], v * vc[:, None]])
    _case(torch, capi.DOP853, capi.plummer(1.0, 1.0), y0, np.linspace(0.0, 30.0, 31), schedule)


def test_noalloc_ordered_schedule_within_and_beyond_its_scratch(cuda_device):
    import ctypes

    import torch

    rng = np.random.default_rng(23)
    n = 500  # the ordered queue of 500 particles fits the fixed scratch
    r = rng.uniform(0.3, 2.0, n)
    y0 = np.hstack([rng.normal(size=(n, 3)), rng.normal(size=(n, 3))])
    y0[:, :3] *= (r / np.linalg.norm(y0[:, :3], axis=1))[:, None]
    y0[:, 3:] *= 0.3 / np.linalg.norm(y0[:, 3:], axis=1)[:, None]
    _case(torch, capi.DOP853, capi.plummer(1.0, 1.0), y0, np.linspace(0.0, 10.0, 11), capi.ORDERED)

    # A queue too large for the fixed scratch is refused with a clear error.
    L = capi.make_launch(capi.DOP853, capi.plummer(), 100_000, 11, rtol=1e-10, atol=1e-10,
                         schedule=capi.ORDERED)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    L.y0, L.ts, L.out = dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr()
    rc = capi.lib().drift_integrate_noalloc(ctypes.byref(L), None)
    assert rc == 3  # DRIFT_ERROR_WORKSPACE
    assert "fixed scratch" in capi.lib().drift_last_error().decode()


def test_noalloc_matches_drift_integrate_dopr54_kepler(cuda_device):
    import torch

    rng = np.random.default_rng(19)
    n = 700
    r = rng.uniform(0.6, 1.8, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    vt = np.sqrt(1.0 / r) * rng.uniform(0.9, 1.1, n)
    y0 = np.stack([r * np.cos(phi), r * np.sin(phi), 0.05 * rng.normal(size=n),
                   -vt * np.sin(phi), vt * np.cos(phi), 0.02 * rng.normal(size=n)], axis=1)
    _case(torch, capi.DOPR54, capi.kepler(1.0), y0, np.linspace(0.0, 12.0, 61), capi.PERSISTENT)
