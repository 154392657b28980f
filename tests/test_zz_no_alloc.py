"""The no-allocation entry point, drift_integrate_noalloc, through the C ABI.

Callers that own all device memory themselves (a pre-reserved memory pool, a
real-time loop that cannot afford an allocation's synchronisation, a plugin
inside a runtime that forbids allocation) integrate through
drift_integrate_noalloc, which keeps its scratch in a fixed array inside the
library instead of a caller-provided workspace.  It runs the same kernel
with the same schedule as drift_integrate, so its results must equal
drift_integrate's bit for bit, on two calls in a row (the array keeps the
previous call's contents, so the second call checks that the scratch is
cleared), and a warmed-up call must leave the device's free memory as it
found it.

This file sorts last so that a run stopping at its first failure has already
run every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu

# The ordered schedule's scratch: a 256-byte cursor, 1 KiB of bucket counts
# and 5 bytes per particle (queue entry and cost key).
ORDERED_FIT = (4096 - 1280) // 5  # 563 particles


def _case(torch, method, pot, y0, ts, schedule, *, switch_device=False):
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

    # the no-allocation entry point, twice in a row, into buffers allocated
    # before the device's free memory is read
    outs = [torch.full((nt, n, 6), float("nan"), dtype=torch.float64, device=dev) for _ in range(2)]
    accs = [torch.zeros(n, dtype=torch.int32, device=dev) for _ in range(2)]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for out, acc in zip(outs, accs):
        capi.integrate_device_noalloc(launch(out, acc), stream)
        torch.cuda.synchronize()
        if switch_device:
            # cudaSetDevice between the calls (torch's own set_device skips
            # the call when the device is already current); the next call
            # looks the scratch address up again in the current context
            import ctypes

            assert ctypes.CDLL("libcudart.so.12").cudaSetDevice(0) == 0
    free_after = torch.cuda.mem_get_info(dev)[0]
    for out, acc in zip(outs, accs):
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
        np.testing.assert_array_equal(acc.cpu().numpy(), ref_acc)
    assert free_after == free_before, f"device free memory moved by {free_before - free_after} bytes"


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
    _case(torch, capi.DOP853, capi.plummer(1.0, 1.0), y0, np.linspace(0.0, 30.0, 31), schedule,
          switch_device=schedule == capi.PERSISTENT)


def _ordered_y0(n, seed):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.3, 2.0, n)
    y0 = np.hstack([rng.normal(size=(n, 3)), rng.normal(size=(n, 3))])
    y0[:, :3] *= (r / np.linalg.norm(y0[:, :3], axis=1))[:, None]
    y0[:, 3:] *= 0.3 / np.linalg.norm(y0[:, 3:], axis=1)[:, None]
    return y0


@pytest.mark.parametrize("n", [500, ORDERED_FIT])
def test_noalloc_ordered_schedule_within_its_scratch(cuda_device, n):
    import torch

    L = capi.make_launch(capi.DOP853, capi.plummer(), n, 11, rtol=1e-10, atol=1e-10,
                         schedule=capi.ORDERED)
    assert capi.query_workspace(L) <= 4096
    _case(torch, capi.DOP853, capi.plummer(1.0, 1.0), _ordered_y0(n, 23), np.linspace(0.0, 10.0, 11),
          capi.ORDERED)


@pytest.mark.parametrize("n", [ORDERED_FIT + 1, 100_000])
def test_noalloc_ordered_schedule_beyond_its_scratch_is_refused(cuda_device, n):
    import ctypes

    import torch

    # A queue too large for the fixed scratch is refused with a clear error
    # before anything is launched.
    L = capi.make_launch(capi.DOP853, capi.plummer(), n, 11, rtol=1e-10, atol=1e-10,
                         schedule=capi.ORDERED)
    assert capi.query_workspace(L) > 4096
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
