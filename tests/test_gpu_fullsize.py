"""The benchmark configuration at full size: 2^20 Plummer particles, DOP853 at
rtol = atol = 1e-12, ts = (0, 100, 201).

Full-size checks use properties that do not need the oracle to integrate
every particle: a seeded subsample against the oracle (1e-9 relative per
sample, both precisions), conservation of energy and angular momentum over
all particles, and bitwise agreement of the plain and persistent schedules.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.workloads import plummer_sphere

pytestmark = pytest.mark.gpu

N = 1 << 20
TS = np.linspace(0.0, 100.0, 201)
SUBSAMPLE = 2048


def energy(y):
    r2 = (y[..., :3] ** 2).sum(-1)
    return 0.5 * (y[..., 3:] ** 2).sum(-1) - 1.0 / np.sqrt(r2 + 1.0)


def ang_mom(y):
    return np.cross(y[..., :3], y[..., 3:])


@pytest.fixture(scope="module")
def workload():
    return plummer_sphere(N)


def _run_device(torch, y0, precision, schedule):
    dev = torch.device("cuda:0")
    n, nt = len(y0), len(TS)
    y0_d = torch.from_numpy(y0).to(dev)
    ts_d = torch.from_numpy(TS).to(dev)
    out_d = torch.empty((nt, n, 6), dtype=torch.float64, device=dev)
    acc_d = torch.zeros(n, dtype=torch.int32, device=dev)
    st_d = torch.full((n,), 255, dtype=torch.uint8, device=dev)
    L = capi.make_launch(capi.DOP853, capi.plummer(1.0, 1.0), n, nt, rtol=1e-12, atol=1e-12,
                         precision=precision, schedule=schedule)
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.y0, L.ts, L.out = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr()
    L.n_accepted, L.status = acc_d.data_ptr(), st_d.data_ptr()
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out_d, acc_d.cpu().numpy().view(np.uint32), st_d.cpu().numpy()


@pytest.mark.parametrize("precision", [capi.EXACT, capi.FMA])
def test_full_size_subsample_matches_oracle(cuda_device, oracle, workload, precision):
    import torch

    out_d, acc, status = _run_device(torch, workload, precision, capi.PERSISTENT)
    assert (status == 0).all()
    idx = np.sort(np.random.default_rng(7).choice(N, SUBSAMPLE, replace=False))
    got = out_d[:, torch.from_numpy(idx).to(out_d.device)].cpu().numpy()
    ref = oracle.integrate_batch(1, oracle.plummer(1.0, 1.0), workload[idx], ts=TS, rtol=1e-12,
                                 atol=1e-12)
    scale = np.maximum(np.abs(ref["out"]).max(axis=2), 1e-300)
    err = (np.abs(got - ref["out"]).max(axis=2) / scale).max()
    assert err < 1e-9, err
    same = (acc[idx].astype(np.int64) == ref["accepted"]).mean()
    assert same >= (0.99 if precision == capi.EXACT else 0.9), same

    # conservation over all particles, last output against the first
    first = out_d[0].cpu().numpy()
    last = out_d[-1].cpu().numpy()
    de = np.abs(energy(last) / energy(first) - 1.0)
    dl = np.linalg.norm(ang_mom(last) - ang_mom(first), axis=1) / np.maximum(
        np.linalg.norm(ang_mom(first), axis=1), 1e-12)
    print(f"precision={precision} |dE/E| median {np.median(de):.2e} p99 {np.quantile(de, 0.99):.2e} "
          f"max {de.max():.2e}; |dL|/|L| p99 {np.quantile(dl, 0.99):.2e}")
    assert np.median(de) < 1e-11 and np.quantile(de, 0.99) < 1e-9
    assert np.quantile(dl, 0.99) < 1e-9
    del out_d
    torch.cuda.empty_cache()


def test_full_size_schedules_agree_bitwise(cuda_device, workload):
    import torch

    a, acc_a, _ = _run_device(torch, workload, capi.EXACT, capi.PERSISTENT)
    final_a = a[-1].cpu().numpy()
    del a
    torch.cuda.empty_cache()
    b, acc_b, _ = _run_device(torch, workload, capi.EXACT, capi.PLAIN)
    np.testing.assert_array_equal(b[-1].cpu().numpy(), final_a)
    np.testing.assert_array_equal(acc_a, acc_b)
    del b
    torch.cuda.empty_cache()
