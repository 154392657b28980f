"""drift_force (the force code the integrators inline) against the oracle's
forces, for every potential kind, over radii that cross every region of the
bulge's incomplete-gamma table (series below x = 6, Taylor pieces to 40,
constant beyond; x = r^2 / rc^2)."""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["kepler", "kepler_cartesian", "plummer", "bovy"])
def test_device_force_matches_oracle(cuda_device, oracle, kind):
    import torch

    pot = {"kepler": capi.kepler(1.0), "kepler_cartesian": capi.kepler_cartesian(1.0),
           "plummer": capi.plummer(1.3, 0.7), "bovy": capi.bovy()}[kind]
    opot = {"kepler": oracle.kepler(1.0), "kepler_cartesian": oracle.kepler(1.0),
            "plummer": oracle.plummer(1.3, 0.7), "bovy": oracle.bovy()}[kind]
    if kind == "kepler_cartesian":
        opot.kind = 3
    rng = np.random.default_rng(2)
    rc = 1.9 / 8.0
    # radii through the table regions (x from 1e-4 to 100) plus a spread out to 20
    r = np.concatenate([rc * np.sqrt(np.exp(rng.uniform(np.log(1e-4), np.log(100.0), 4000))),
                        np.exp(rng.uniform(np.log(0.01), np.log(20.0), 4000)),
                        rc * np.sqrt(np.array([6.0, 6.0 - 1e-12, 40.0, 40.0 - 1e-12, 7.0, 39.0]))])
    u = rng.normal(size=(len(r), 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    xyz = np.ascontiguousarray(u * r[:, None])
    xyz_d = torch.tensor(xyz, device="cuda")
    acc_d = torch.empty_like(xyz_d)
    capi.force_device(pot, len(xyz), xyz_d.data_ptr(), acc_d.data_ptr())
    torch.cuda.synchronize()
    got = acc_d.cpu().numpy()
    ref = np.array([oracle.force(opot, *p) for p in xyz])
    err = np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)
    assert err.max() < 1e-13, (err.max(), xyz[err.argmax()])
