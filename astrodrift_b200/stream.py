"""Tidal streams by particle spray around a moving progenitor.

    out = spray(progenitor_state, capi.bovy(), t_end=50.0, n_release=400, mass=2e-5)
    out["y"]            # (2 * n_release, 6) stream particles at t_end (torch, CUDA)

The progenitor's orbit is integrated on the GPU on the release grid
t_k = k t_end / n_release.  At every release time two particles leave it,
one through each Lagrange point, following Fardal, Huang & Weinberg (2015,
MNRAS 452, 301): with the tidal radius r_t = (G m / (Omega^2 - d2Phi/dr2))^(1/3)
and the orbital angular speed Omega,
    offset along r_hat       = +-k_r r_t,          k_r  ~ N(2.0, 0.5)
    offset along the normal  =   k_z r_t,          k_z  ~ N(0.0, 0.5)
    velocity along t_hat     = +-k_vt Omega r_t,   k_vt ~ N(0.3, 0.4)
    velocity along the normal=   k_vz Omega r_t,   k_vz ~ N(0.0, 0.5)
(+ for the trailing arm at the outer point, - for the leading arm).  Each
release group is then integrated from its release time to t_end in the host
potential plus, by default, the progenitor's own Plummer potential moving
along its orbit (a force model with a one-source origin table).  Release
groups are the segments of batched launches (up to 64 per launch) under the
ordered schedule, so early releases -- which travel longest -- start first.
Everything runs on the GPU; the host only draws the offsets.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import capi


def _tidal_radius(torch, host: capi.DriftPotential, x, v, mass: float):
    """r_t, Omega and the unit vectors at progenitor states x, v (k, 3)."""
    dev = x.device
    r = torch.linalg.norm(x, dim=1)
    rhat = x / r[:, None]
    Lvec = torch.linalg.cross(x, v, dim=1)
    Lmag = torch.linalg.norm(Lvec, dim=1)
    nhat = Lvec / Lmag[:, None]
    that = torch.linalg.cross(nhat, rhat, dim=1)
    omega = Lmag / (r * r)
    # d^2 Phi / dr^2 = -dF_r/dr by central differences of the device force
    eps = 1e-4
    pts = torch.cat([x * (1 + eps), x * (1 - eps)], dim=0).contiguous()
    acc = torch.empty_like(pts)
    capi.force_device(host, pts.shape[0], pts.data_ptr(), acc.data_ptr(),
                      torch.cuda.current_stream(dev).cuda_stream)
    k = x.shape[0]
    fr_plus = (acc[:k] * rhat).sum(1)
    fr_minus = (acc[k:] * rhat).sum(1)
    d2phi = -(fr_plus - fr_minus) / (2 * eps * r)
    rt = (mass / torch.clamp(omega * omega - d2phi, min=1e-300)) ** (1.0 / 3.0)
    return rt, omega, rhat, that, nhat


def spray(progenitor, host: capi.DriftPotential, *, t_end: float, n_release: int = 200, mass: float = 1e-4,
          plummer_b: float | None = None, seed: int = 0, rtol: float = 1e-10, method: int = capi.DOP853,
          precision: int = capi.FMA, progenitor_force: bool = True, outputs: int = 2) -> dict:
    """Stream particles at t_end.  Returns a dict of CUDA tensors:
    y (2 n_release, 6) final states; release_time (2 n_release,); arm (+1
    trailing, -1 leading); progenitor (n_release + 1, 6) orbit on the release
    grid; and, with outputs > 2, trajectories: a list per release group of
    (outputs, 2, 6) samples from release to t_end."""
    import torch

    if host.kind == capi.POT_MODEL:
        raise ValueError("the host must be a single potential")
    if n_release < 1 or outputs < 2:
        raise ValueError("n_release >= 1 and outputs >= 2 are required")
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev).cuda_stream
    f64 = torch.float64
    nt = n_release + 1
    ts = np.linspace(0.0, t_end, nt)

    # 1. the progenitor's orbit on the release grid
    prog_d = torch.tensor(np.asarray(progenitor, dtype=np.float64).reshape(1, 6), device=dev)
    ts_d = torch.tensor(ts, device=dev)
    traj_d = torch.empty((nt, 1, 6), dtype=f64, device=dev)
    L = capi.make_launch(capi.DOP853, host, 1, nt, rtol=rtol, atol=rtol, precision=precision,
                         schedule=capi.PLAIN)
    L.y0, L.ts, L.out = prog_d.data_ptr(), ts_d.data_ptr(), traj_d.data_ptr()
    capi.integrate_device(L, stream)

    # 2. release states (Fardal et al. 2015)
    x = traj_d[:n_release, 0, :3]
    v = traj_d[:n_release, 0, 3:]
    rt, omega, rhat, that, nhat = _tidal_radius(torch, host, x, v, mass)
    rng = np.random.default_rng(seed)
    draw = lambda mu, sd: torch.tensor(rng.normal(mu, sd, (n_release, 2)), device=dev)  # noqa: E731
    k_r, k_z, k_vt, k_vz = draw(2.0, 0.5), draw(0.0, 0.5), draw(0.3, 0.4), draw(0.0, 0.5)
    sign = torch.tensor([1.0, -1.0], dtype=f64, device=dev)  # trailing (outer), leading (inner)
    rt2, om2 = rt[:, None], omega[:, None]
    pos = (x[:, None, :] + (sign * k_r * rt2)[..., None] * rhat[:, None, :]
           + (k_z * rt2)[..., None] * nhat[:, None, :])
    vel = (v[:, None, :] + (sign * k_vt * om2 * rt2)[..., None] * that[:, None, :]
           + (k_vz * om2 * rt2)[..., None] * nhat[:, None, :])
    y0 = torch.cat([pos, vel], dim=2).reshape(2 * n_release, 6).contiguous()

    # 3. the stream's force: host + the progenitor moving along its orbit
    keep = []
    if progenitor_force:
        table = torch.empty((n_release, 1, 18), dtype=f64, device=dev)
        capi.origin_table_device(capi.force_model([host]), 1, nt, 0.0, t_end / n_release,
                                 traj_d.data_ptr(), table.data_ptr(), stream)
        b = plummer_b if plummer_b is not None else float(rt.mean()) * 0.5
        model = capi.force_model([host], [(capi.POT_PLUMMER, mass, b, 0, 1)], origins=table.data_ptr(),
                                 n_sources=1, n_segments=n_release, t0=0.0, dt=t_end / n_release)
        keep += [table]
    else:
        model = capi.force_model([host])
    model_ptr = ctypes.pointer(model)

    # 4. release groups as segments of batched, ordered launches
    t_end_d = torch.full((2 * n_release,), float(t_end), dtype=f64, device=dev)
    y_fin = torch.empty((2 * n_release, 6), dtype=f64, device=dev)
    status = torch.zeros(2 * n_release, dtype=torch.uint8, device=dev)
    trajs = []
    for g0 in range(0, n_release, capi.MAX_BATCH):
        groups = range(g0, min(g0 + capi.MAX_BATCH, n_release))
        launches = []
        for k in groups:
            Lk = capi.make_launch(method, capi.model_potential(), 2, outputs, rtol=rtol, atol=rtol,
                                  precision=precision, schedule=capi.ORDERED, t0=float(ts[k]))
            Lk.force_model = model_ptr
            Lk.y0 = y0.data_ptr() + k * 2 * 48
            Lk.t_end = t_end_d.data_ptr() + k * 2 * 8
            Lk.y_final = y_fin.data_ptr() + k * 2 * 48
            Lk.status = status.data_ptr() + k * 2
            if outputs > 2:
                o = torch.empty((outputs, 2, 6), dtype=f64, device=dev)
                trajs.append(o)
                Lk.out = o.data_ptr()
            launches.append(Lk)
        probe = capi.make_launch(method, capi.model_potential(), 2 * len(launches), outputs, rtol=rtol,
                                 atol=rtol, schedule=capi.ORDERED)
        ws = torch.empty(capi.query_workspace(probe), dtype=torch.uint8, device=dev)
        launches[0].workspace, launches[0].workspace_bytes = ws.data_ptr(), ws.numel()
        capi.integrate_batch_device(launches, stream)
        keep.append(ws)
    torch.cuda.current_stream(dev).synchronize()
    st = status.cpu().numpy()
    if (st != capi.PARTICLE_OK).any():
        raise RuntimeError(f"{int((st != 0).sum())} stream particles did not finish (status {np.unique(st)})")
    release = torch.tensor(np.repeat(ts[:n_release], 2), device=dev)
    arm = torch.tensor(np.tile([1, -1], n_release), device=dev)
    out = {"y": y_fin, "release_time": release, "arm": arm, "progenitor": traj_d[:, 0, :],
           "initial": y0, "tidal_radius": rt}
    if outputs > 2:
        out["trajectories"] = trajs
    return out
