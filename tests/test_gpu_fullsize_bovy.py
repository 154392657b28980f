"""The uneven Bovy configuration at full size: 2^22 particles with radii
log-uniform on [0.05, 20] and per-particle end times in [10, 1000], 101
outputs each, DOP853 at rtol = atol = 1e-10 (contraction unit, ordered
schedule), as the benchmark runs it.

The oracle cannot integrate 4 million particles in a test, so the checks are
size-independent: every particle finishes, energy and L_z are conserved over
all particles at the level of the integration error, and the particles with
the shortest spans match the oracle sample for sample."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi
from astrodrift_b200.energy import angular_momentum_drift, drift_summary
from astrodrift_b200.workloads import bovy_disc

pytestmark = pytest.mark.gpu

N = 1 << 22
NT = 101


def test_full_size_uneven_bovy(cuda_device, oracle):
    import torch

    dev = torch.device("cuda:0")
    pot = capi.bovy()

    def radial_force(R):
        xyz = torch.zeros((len(R), 3), dtype=torch.float64, device=dev)
        xyz[:, 0] = torch.from_numpy(np.asarray(R, dtype=np.float64))
        acc = torch.empty_like(xyz)
        capi.force_device(pot, len(R), xyz.data_ptr(), acc.data_ptr())
        torch.cuda.synchronize()
        return acc[:, 0].cpu().numpy()

    y0, t_end = bovy_disc(N, seed=3, radial_force=radial_force)
    y0_d = torch.tensor(y0, device=dev)
    te_d = torch.tensor(t_end, device=dev)
    out = torch.empty((NT, N, 6), dtype=torch.float64, device=dev)  # 20.3 GB
    st = torch.zeros(N, dtype=torch.uint8, device=dev)
    L = capi.make_launch(capi.DOP853, pot, N, NT, rtol=1e-10, atol=1e-10, precision=capi.FMA,
                         schedule=capi.ORDERED)
    L.y0, L.t_end, L.out, L.status = y0_d.data_ptr(), te_d.data_ptr(), out.data_ptr(), st.data_ptr()
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert int((st != 0).sum()) == 0

    first, last = out[0].cpu().numpy(), out[-1].cpu().numpy()
    e = drift_summary(pot, first, last)
    lz = angular_momentum_drift(pot, first, last)
    print("energy drift", e, "L_z drift", lz)
    # measured: energy median 6.3e-10, p99 2.2e-8; L_z median 2.1e-10, p99 2.0e-7
    assert e["median"] < 5e-9 and e["p99"] < 2e-7 and e["particles"] == N
    assert lz["median"] < 5e-9 and lz["p99"] < 2e-6

    # the 64 shortest spans (t_end near 10) against the oracle, every sample
    idx = np.sort(np.argsort(t_end)[:64])
    got = out[:, torch.from_numpy(idx).to(dev)].cpu().numpy()
    del out
    torch.cuda.empty_cache()
    ref = oracle.integrate_batch(1, oracle.bovy(), y0[idx], t_end=t_end[idx], nt=NT, rtol=1e-10, atol=1e-10)
    assert (np.asarray(ref["status"]) == 0).all()
    scale = np.maximum(np.abs(ref["out"]).max(axis=2), 1e-300)
    err = (np.abs(got - ref["out"]).max(axis=2) / scale).max()
    assert err < 1e-8, err
