"""Force models (drift_force_model): summed stationary potentials and
potentials attached to moving particle groups, on the GPU against the oracle.

* A model with one stationary part reproduces that potential's integration
  bit for bit (the sum starts at 0 and adds one term).
* Sums of several stationary parts match the oracle's model to 1e-9.
* The device origin table (quintic Hermite segments from a source trajectory)
  and the model force at arbitrary times match the oracle's.
* A two-stage system -- a satellite carrying a Plummer potential orbits the
  Bovy composite, then test particles feel both -- matches the oracle when
  both integrate the second stage from the same satellite trajectory.
Exact arithmetic throughout, like the other parity tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from astrodrift_b200 import capi

pytestmark = pytest.mark.gpu

REL = 1e-9


def rel_err(a, b):
    a = np.asarray(a).reshape(-1, 6)
    b = np.asarray(b).reshape(-1, 6)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def disc(n, seed, rmin=0.5, rmax=2.0, v=1.0):
    rng = np.random.default_rng(seed)
    r = rng.uniform(rmin, rmax, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    vt = v * rng.uniform(0.85, 1.05, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(0, 0.05, n),
                     -vt * np.sin(phi), vt * np.cos(phi), rng.normal(0, 0.03, n)], axis=1)


def oracle_statics(oracle, parts):
    out = []
    for kind, kw in parts:
        if kind == "plummer":
            out.append(oracle.plummer(kw["amp"], kw["b"]))
        elif kind == "kepler":
            out.append(oracle.kepler(kw["amp"]))
        else:
            out.append(oracle.bovy())
    return out


def capi_statics(parts):
    out = []
    for kind, kw in parts:
        if kind == "plummer":
            out.append(capi.plummer(kw["amp"], kw["b"]))
        elif kind == "kepler":
            out.append(capi.kepler(kw["amp"]))
        else:
            out.append(capi.bovy())
    return out


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
@pytest.mark.parametrize("name", ["plummer", "bovy"])
def test_single_part_model_equals_the_potential_bitwise(cuda_device, method, name):
    pot = capi.plummer(1.0, 1.0) if name == "plummer" else capi.bovy()
    y0 = disc(300, 1, v=0.5 if name == "plummer" else 1.0)
    ts = np.linspace(0.0, 12.0, 25)
    ref = capi.integrate_host(method, pot, y0, ts=ts, rtol=1e-10, atol=1e-10)
    model = capi.force_model([pot])
    got = capi.integrate_host(method, pot, y0, ts=ts, rtol=1e-10, atol=1e-10, model=model)
    np.testing.assert_array_equal(got["out"], ref["out"])
    np.testing.assert_array_equal(got["accepted"], ref["accepted"])


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
def test_summed_stationary_parts_match_oracle(cuda_device, oracle, method):
    parts = [("bovy", {}), ("plummer", {"amp": 0.3, "b": 0.5}), ("kepler", {"amp": 0.2})]
    y0 = disc(200, 2, v=1.2)
    ts = np.linspace(0.0, 10.0, 21)
    got = capi.integrate_host(method, capi.model_potential(), y0, ts=ts, rtol=1e-10, atol=1e-10,
                              model=capi.force_model(capi_statics(parts)))
    opot = oracle.model(oracle_statics(oracle, parts))
    ref = oracle.integrate_batch(method, opot, y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert (got["status"] == 0).all()
    assert rel_err(got["out"], ref["out"]) < REL


def _satellite(oracle, nt=41, t_end=8.0):
    """Stage one: a satellite in the Bovy composite (oracle trajectory)."""
    sat = np.array([[1.2, 0.0, 0.05, 0.0, 1.0, 0.02], [0.0, -1.6, 0.0, 0.95, 0.0, 0.0]])
    ts = np.linspace(0.0, t_end, nt)
    traj = oracle.integrate_batch(1, oracle.bovy(), sat, ts=ts, rtol=1e-12, atol=1e-12)["out"]
    return sat, ts, traj


def test_origin_table_and_model_force_match_oracle(cuda_device, oracle):
    import torch

    sat, ts, traj = _satellite(oracle)
    t0, dt, nt = ts[0], ts[1] - ts[0], len(ts)
    ref_table = oracle.origin_table(oracle.bovy(), traj, t0, dt)
    traj_d = torch.tensor(traj, device="cuda")
    table_d = torch.empty((nt - 1, 2, 18), dtype=torch.float64, device="cuda")
    src_model = capi.force_model([capi.bovy()])
    capi.origin_table_device(src_model, 2, nt, t0, dt, traj_d.data_ptr(), table_d.data_ptr())
    torch.cuda.synchronize()
    table = table_d.cpu().numpy()
    scale = np.abs(ref_table).max(axis=2, keepdims=True)
    assert (np.abs(table - ref_table) / scale).max() < 1e-13
    # the quintic passes through the samples
    np.testing.assert_array_equal(table[:, :, 0], traj[:-1, :, 0])

    groups = [(capi.POT_PLUMMER, 0.05, 0.02, 0, 1), (capi.POT_KEPLER_CARTESIAN, 0.01, 0.0, 1, 1)]
    model = capi.force_model([capi.bovy()], groups, origins=table_d.data_ptr(), n_sources=2,
                             n_segments=nt - 1, t0=t0, dt=dt)
    omodel = oracle.model([oracle.bovy()], [(oracle.POT_PLUMMER, 0.05, 0.02, 0, 1),
                                            (oracle.POT_KEPLER_CARTESIAN, 0.01, 0.0, 1, 1)],
                          origins=table, t0=t0, dt=dt)
    rng = np.random.default_rng(3)
    xyz = np.ascontiguousarray(rng.uniform(-2, 2, (500, 3)))
    xyz_d = torch.tensor(xyz, device="cuda")
    acc_d = torch.empty_like(xyz_d)
    for t in (0.0, 0.37, 3.9, 7.999, 8.0, 8.3, -0.2):  # inside, at the ends, and beyond both
        capi.force_model_eval_device(model, len(xyz), t, xyz_d.data_ptr(), acc_d.data_ptr())
        torch.cuda.synchronize()
        got = acc_d.cpu().numpy()
        ref = np.array([oracle.force_t(omodel, t, *p) for p in xyz])
        err = (np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)).max()
        assert err < 1e-13, (t, err)


@pytest.mark.parametrize("method", [capi.DOPR54, capi.DOP853])
def test_particles_around_a_moving_satellite_match_oracle(cuda_device, oracle, method):
    sat, ts, traj = _satellite(oracle)
    t0, dt, nt = ts[0], ts[1] - ts[0], len(ts)
    table = oracle.origin_table(oracle.bovy(), traj, t0, dt)
    # a swarm launched near the first satellite, plus disc particles
    rng = np.random.default_rng(4)
    swarm = sat[0] + np.hstack([rng.normal(0, 0.05, (64, 3)), rng.normal(0, 0.05, (64, 3))])
    y0 = np.vstack([swarm, disc(64, 5)])
    groups = [(capi.POT_PLUMMER, 0.02, 0.05, 0, 1), (capi.POT_PLUMMER, 0.01, 0.05, 1, 1)]
    model = capi.force_model([capi.bovy()], groups, origins=table.ctypes.data, n_sources=2,
                             n_segments=nt - 1, t0=t0, dt=dt)
    got = capi.integrate_host(method, capi.model_potential(), y0, ts=ts, rtol=1e-10, atol=1e-10, model=model)
    omodel = oracle.model([oracle.bovy()], [(oracle.POT_PLUMMER, 0.02, 0.05, 0, 1),
                                            (oracle.POT_PLUMMER, 0.01, 0.05, 1, 1)],
                          origins=table, t0=t0, dt=dt)
    ref = oracle.integrate_batch(method, omodel, y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert (got["status"] == 0).all()
    assert rel_err(got["out"], ref["out"]) < REL
    # the satellite's pull matters: without it the swarm ends elsewhere
    plain = capi.integrate_host(method, capi.bovy(), y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert rel_err(plain["out"][-1, :64], got["out"][-1, :64]) > 1e-4


def test_device_entry_point_with_device_origin_table(cuda_device, oracle):
    """drift_integrate (device pointers) with the table built on the device
    from the satellite's device trajectory -- the path the host dispatch uses."""
    import torch

    sat, ts, traj = _satellite(oracle)
    t0, dt, nt = ts[0], ts[1] - ts[0], len(ts)
    dev = torch.device("cuda:0")
    traj_d = torch.tensor(traj, device=dev)
    table_d = torch.empty((nt - 1, 2, 18), dtype=torch.float64, device=dev)
    capi.origin_table_device(capi.force_model([capi.bovy()]), 2, nt, t0, dt, traj_d.data_ptr(),
                             table_d.data_ptr())
    model = capi.force_model([capi.bovy()], [(capi.POT_PLUMMER, 0.02, 0.05, 0, 2)],
                             origins=table_d.data_ptr(), n_sources=2, n_segments=nt - 1, t0=t0, dt=dt)
    y0 = disc(500, 6)
    y0_d = torch.tensor(y0, device=dev)
    ts_d = torch.tensor(ts, device=dev)
    out_d = torch.empty((nt, len(y0), 6), dtype=torch.float64, device=dev)
    for schedule in (capi.PLAIN, capi.ORDERED):
        L = capi.make_launch(capi.DOP853, capi.model_potential(), len(y0), nt, rtol=1e-10, atol=1e-10,
                             schedule=schedule)
        L.force_model = ctypes.pointer(model)
        L.y0, L.ts, L.out = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr()
        ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
        L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
        capi.integrate_device(L, 0)
        torch.cuda.synchronize()
        got = out_d.cpu().numpy()
        if schedule == capi.PLAIN:
            first = got.copy()
        else:
            np.testing.assert_array_equal(got, first)
    table = table_d.cpu().numpy()
    omodel = oracle.model([oracle.bovy()], [(oracle.POT_PLUMMER, 0.02, 0.05, 0, 2)], origins=table,
                          t0=t0, dt=dt)
    ref = oracle.integrate_batch(1, omodel, y0, ts=ts, rtol=1e-10, atol=1e-10)
    assert rel_err(first, ref["out"]) < REL


def test_chunked_host_path_with_moving_sources(cuda_device, oracle):
    """drift_integrate_host splits large requests into particle chunks; every
    chunk must see the uploaded origin table."""
    import torch

    sat, ts, traj = _satellite(oracle)
    t0, dt, nt = ts[0], ts[1] - ts[0], len(ts)
    table = oracle.origin_table(oracle.bovy(), traj, t0, dt)
    y0 = disc(70001, 8)
    model = capi.force_model([capi.bovy()], [(capi.POT_PLUMMER, 0.02, 0.05, 0, 2)], origins=table.ctypes.data,
                             n_sources=2, n_segments=nt - 1, t0=t0, dt=dt)
    got = capi.integrate_host(capi.DOP853, capi.model_potential(), y0, ts=ts, rtol=1e-10, atol=1e-10,
                              model=model)
    # the device entry point on a device copy of the same table
    dev = torch.device("cuda:0")
    table_d = torch.tensor(table, device=dev)
    model_d = capi.force_model([capi.bovy()], [(capi.POT_PLUMMER, 0.02, 0.05, 0, 2)],
                               origins=table_d.data_ptr(), n_sources=2, n_segments=nt - 1, t0=t0, dt=dt)
    y0_d = torch.tensor(y0, device=dev)
    ts_d = torch.tensor(ts, device=dev)
    out_d = torch.empty((nt, len(y0), 6), dtype=torch.float64, device=dev)
    L = capi.make_launch(capi.DOP853, capi.model_potential(), len(y0), nt, rtol=1e-10, atol=1e-10,
                         schedule=capi.ORDERED)
    L.force_model = ctypes.pointer(model_d)
    L.y0, L.ts, L.out = y0_d.data_ptr(), ts_d.data_ptr(), out_d.data_ptr()
    ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
    L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
    capi.integrate_device(L, 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got["out"], out_d.cpu().numpy())
