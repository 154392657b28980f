"""Seeded synthetic initial conditions for the benchmark configurations.

No public dataset is involved: every workload is drawn from a fixed-seed
numpy generator with the distributions the configurations specify.
"""

from __future__ import annotations

import numpy as np

# The Bovy-style composite of the benchmark configurations in natural units
# (R0 = 1, v_c(1) = 1): power-law bulge with exponential cutoff (alpha, rc)
# normalised to F_r(1) = -bulge_force, Miyamoto-Nagai disk and NFW halo with
# the reference's fraction-normalised amplitudes (shared/src/potential.rs:103-112).
BOVY_PARAMS = dict(alpha=1.8, rc=1.9 / 8.0, bulge_force=0.05, mn_amp=0.7574802019,
                   mn_a=3.0 / 8.0, mn_b=0.28 / 8.0, nfw_amp=4.852230533528, nfw_a=16.0 / 8.0)


def bovy_radial_force(R) -> np.ndarray:
    """F_R(R, z = 0) of the composite with BOVY_PARAMS, in float64 on the host.

    bulge  -k gamma(s, r^2 / rc^2) / r^2 with s = 3/2 - alpha/2 and k set so
           that the bulge's F_r(1) = -bulge_force (gamma: scipy's regularised
           lower incomplete gamma times Gamma(s));
    disk   -amp R / (R^2 + (a + b)^2)^(3/2) in the plane;
    halo   -amp (ln(1 + r/a) - r/(a + r)) / r^2.
    The benchmark's initial conditions use it in every arm, so they are the
    same whichever implementation integrates them.
    """
    from scipy.special import gamma, gammainc

    p = BOVY_PARAMS
    R = np.asarray(R, dtype=np.float64)
    s = 1.5 - 0.5 * p["alpha"]
    rc2 = p["rc"] ** 2
    lower = lambda x: gammainc(s, x) * gamma(s)  # noqa: E731
    k = p["bulge_force"] / lower(1.0 / rc2)
    bulge = -k * lower(R * R / rc2) / (R * R)
    disk = -p["mn_amp"] * R / (R * R + (p["mn_a"] + p["mn_b"]) ** 2) ** 1.5
    a = p["nfw_a"]
    halo = -p["nfw_amp"] * (np.log1p(R / a) - R / (a + R)) / (R * R)
    return bulge + disk + halo


def _isotropic(rng, n):
    u = rng.normal(size=(n, 3))
    return u / np.linalg.norm(u, axis=1, keepdims=True)


def plummer_sphere(n: int, seed: int = 2, amp: float = 1.0, b: float = 1.0,
                   u_cap: float = 0.999) -> np.ndarray:
    """Isotropic Plummer distribution function (G = 1).

    Radius by inverse CDF, r = b / sqrt(u^(-2/3) - 1) with u ~ U(0, u_cap];
    speed q * v_esc with q drawn by rejection from g(q) = q^2 (1 - q^2)^(7/2)
    under the bound 0.1 (Aarseth, Henon & Wielen 1974); isotropic directions.
    """
    rng = np.random.default_rng(seed)
    u = rng.uniform(0.0, u_cap, n)
    u = np.where(u == 0.0, u_cap, u)
    r = b / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
    q = np.empty(n)
    filled = 0
    while filled < n:
        m = 2 * (n - filled) + 64
        x = rng.uniform(0.0, 1.0, m)
        y = rng.uniform(0.0, 0.1, m)
        acc = x[y < x * x * (1.0 - x * x) ** 3.5]
        take = min(len(acc), n - filled)
        q[filled:filled + take] = acc[:take]
        filled += take
    v_esc = np.sqrt(2.0 * amp / np.sqrt(r * r + b * b))
    pos = _isotropic(rng, n) * r[:, None]
    vel = _isotropic(rng, n) * (q * v_esc)[:, None]
    return np.ascontiguousarray(np.hstack([pos, vel]))


def kepler_disc(n: int, seed: int = 1) -> np.ndarray:
    """Configuration 1: r ~ U[0.5, 2], isotropic orbital plane, tangential
    speed sqrt(1/r) U[0.9, 1.1], radial speed N(0, 0.05 sqrt(1/r)); draws with
    cylindrical radius < 1e-3 are redrawn (the galpy Kepler force is singular
    on the z axis)."""
    rng = np.random.default_rng(seed)
    out = np.empty((n, 6))
    filled = 0
    while filled < n:
        m = n - filled
        r = rng.uniform(0.5, 2.0, m)
        normal = _isotropic(rng, m)
        a = _isotropic(rng, m)
        rhat = np.cross(normal, a)
        rhat /= np.linalg.norm(rhat, axis=1, keepdims=True)
        that = np.cross(normal, rhat)
        vt = np.sqrt(1.0 / r) * rng.uniform(0.9, 1.1, m)
        vr = rng.normal(0.0, 0.05 * np.sqrt(1.0 / r))
        pos = rhat * r[:, None]
        vel = that * vt[:, None] + rhat * vr[:, None]
        ok = np.hypot(pos[:, 0], pos[:, 1]) >= 1e-3
        k = int(ok.sum())
        out[filled:filled + k] = np.hstack([pos, vel])[ok]
        filled += k
    return out


def bovy_disc(n: int, seed: int = 3, radial_force=None) -> tuple[np.ndarray, np.ndarray]:
    """Configuration 3: R log-uniform on [0.05, 20], phi ~ U[0, 2 pi),
    z ~ N(0, 0.1 R); v_c(R) = sqrt(R |F_R(R, 0)|); v_T = v_c (1 + 0.1 N(0,1)),
    v_R, v_z ~ N(0, 0.1 v_c); per-particle end times t_end ~ U[10, 1000].
    `radial_force(R)` returns F_R(R, 0) of the composite (default:
    bovy_radial_force, on the host)."""
    if radial_force is None:
        radial_force = bovy_radial_force
    rng = np.random.default_rng(seed)
    R = np.exp(rng.uniform(np.log(0.05), np.log(20.0), n))
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    z = rng.normal(0.0, 1.0, n) * 0.1 * R
    vc = np.sqrt(R * np.abs(radial_force(R)))
    vT = vc * (1.0 + 0.1 * rng.normal(size=n))
    vR = 0.1 * vc * rng.normal(size=n)
    vz = 0.1 * vc * rng.normal(size=n)
    c, s = np.cos(phi), np.sin(phi)
    y0 = np.stack([R * c, R * s, z, vR * c - vT * s, vR * s + vT * c, vz], axis=1)
    t_end = rng.uniform(10.0, 1000.0, n)
    return np.ascontiguousarray(y0), t_end


def stream_progenitor(n: int, vc: float, seed: int = 5) -> tuple[np.ndarray, np.ndarray]:
    """Configuration 5: a progenitor at R = 1.5, z = 0.2, phi = 0 moving with
    v = (0, v_c(1.5), 0), and n particles offset from it by N(0, 0.002) in
    position and N(0, 0.005) in velocity.  `vc` is the composite's circular
    speed at R = 1.5.  Returns (progenitor (6,), particles (n, 6))."""
    rng = np.random.default_rng(seed)
    prog = np.array([1.5, 0.0, 0.2, 0.0, vc, 0.0])
    y0 = prog[None, :] + np.hstack([rng.normal(0.0, 0.002, (n, 3)), rng.normal(0.0, 0.005, (n, 3))])
    return prog, np.ascontiguousarray(y0)
