"""Tidal-stream generation by particle spray (astrodrift_b200.stream).

Every release group integrates from its own release time in the Bovy host
plus the progenitor's moving Plummer potential, as segments of batched
launches.  The oracle repeats each group from the same released states with
the same force model (origin table built from the same progenitor orbit):
final states agree to 1e-9.  The stream also has the expected shape: the
particles trail and lead the progenitor along its orbit.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi, stream

pytestmark = pytest.mark.gpu


def test_spray_matches_oracle_group_by_group(cuda_device, oracle):
    import torch

    host = capi.bovy()
    xyz = torch.tensor([[1.5, 0.0, 0.0]], dtype=torch.float64, device="cuda")
    acc = torch.empty_like(xyz)
    capi.force_device(host, 1, xyz.data_ptr(), acc.data_ptr())
    torch.cuda.synchronize()
    vc = float(np.sqrt(1.5 * abs(float(acc[0, 0]))))
    prog = np.array([1.5, 0.0, 0.2, 0.0, vc, 0.0])
    n_release, t_end, mass, b = 90, 20.0, 2e-5, 0.01
    out = stream.spray(prog, host, t_end=t_end, n_release=n_release, mass=mass, plummer_b=b, seed=3,
                       rtol=1e-10, precision=capi.EXACT)
    y = out["y"].cpu().numpy()
    y0 = out["initial"].cpu().numpy()
    traj = out["progenitor"].cpu().numpy()
    assert y.shape == (2 * n_release, 6) and np.isfinite(y).all()

    dt = t_end / n_release
    table = oracle.origin_table(oracle.bovy(), traj[:, None, :], 0.0, dt)
    omodel = oracle.model([oracle.bovy()], [(oracle.POT_PLUMMER, mass, b, 0, 1)], origins=table, t0=0.0, dt=dt)
    worst = 0.0
    for k in range(0, n_release, 7):
        tk = k * t_end / n_release
        ts = np.array([tk, t_end])
        ref = oracle.integrate_batch(1, omodel, y0[2 * k: 2 * k + 2], ts=ts, rtol=1e-10, atol=1e-10)["out"][-1]
        got = y[2 * k: 2 * k + 2]
        worst = max(worst, float((np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)).max()))
    assert worst < 1e-9, worst

    # shape: stream stays close to the progenitor's orbit; trailing behind, leading ahead in azimuth
    pf = traj[-1]
    phi_p = np.arctan2(pf[1], pf[0])
    phi = np.arctan2(y[:, 1], y[:, 0])
    dphi = (phi - phi_p + np.pi) % (2 * np.pi) - np.pi
    arm = out["arm"].cpu().numpy()
    old = out["release_time"].cpu().numpy() < t_end / 2
    assert np.median(dphi[(arm == 1) & old]) < 0 < np.median(dphi[(arm == -1) & old])
    R = np.hypot(y[:, 0], y[:, 1])
    assert np.abs(np.median(R) - np.hypot(pf[0], pf[1])) < 0.5
