"""The seeded synthetic workloads the benchmark integrates: their samples
follow the distributions their docstrings state (host-only, no GPU)."""

from __future__ import annotations

import numpy as np

from astrodrift_b200.workloads import bovy_disc, kepler_disc, plummer_sphere, stream_progenitor


def test_plummer_sphere_is_the_equilibrium_distribution():
    n = 400_000
    y = plummer_sphere(n, seed=11)
    r2 = (y[:, :3] ** 2).sum(1)
    v2 = (y[:, 3:] ** 2).sum(1)
    # mass profile: M(<1) / M = 2^-3/2 (with u drawn on (0, 0.999])
    assert abs((r2 < 1.0).mean() - 2.0 ** -1.5 / 0.999) < 0.004
    # every particle is bound: E = v^2 / 2 - (r^2 + 1)^-1/2 < 0
    assert (0.5 * v2 - 1.0 / np.sqrt(r2 + 1.0) < 0.0).all()
    # virial equilibrium in the fixed potential: <v^2> = <r . grad Phi> = <r^2 (r^2 + 1)^-3/2>
    lhs, rhs = v2.mean(), (r2 / (r2 + 1.0) ** 1.5).mean()
    assert abs(lhs / rhs - 1.0) < 0.01
    # isotropy of positions and velocities
    assert np.abs(y.mean(axis=0)).max() < 0.02 * np.sqrt(max(r2.mean(), v2.mean()))
    # reproducible from the seed
    np.testing.assert_array_equal(plummer_sphere(1000, seed=11), plummer_sphere(1000, seed=11))


def test_kepler_disc_follows_its_recipe():
    y = kepler_disc(20_000, seed=4)
    r = np.linalg.norm(y[:, :3], axis=1)
    assert r.min() >= 0.5 and r.max() <= 2.0
    assert np.hypot(y[:, 0], y[:, 1]).min() >= 1e-3  # off the z axis
    rhat = y[:, :3] / r[:, None]
    vr = (y[:, 3:] * rhat).sum(1)
    vt = np.linalg.norm(y[:, 3:] - vr[:, None] * rhat, axis=1)
    ratio = vt * np.sqrt(r)  # tangential speed over the circular speed sqrt(1/r)
    assert ratio.min() >= 0.9 - 1e-12 and ratio.max() <= 1.1 + 1e-12
    assert abs(np.std(vr * np.sqrt(r)) - 0.05) < 0.002


def test_bovy_disc_and_stream_progenitor_follow_their_recipes():
    def radial_force(R):
        return -1.0 / R  # any force: the recipe only scales speeds by it

    y0, t_end = bovy_disc(50_000, seed=5, radial_force=radial_force)
    R = np.hypot(y0[:, 0], y0[:, 1])
    assert R.min() >= 0.05 and R.max() <= 20.0
    assert abs(np.log(R).mean() - 0.5 * (np.log(0.05) + np.log(20.0))) < 0.03  # log-uniform
    assert t_end.min() >= 10.0 and t_end.max() <= 1000.0
    assert abs(np.std(y0[:, 2] / R) - 0.1) < 0.003  # z ~ N(0, 0.1 R)

    prog, y = stream_progenitor(40_000, vc=0.8, seed=6)
    np.testing.assert_array_equal(prog, [1.5, 0.0, 0.2, 0.0, 0.8, 0.0])
    d = y - prog
    assert abs(d[:, :3].std() - 0.002) < 1e-4 and abs(d[:, 3:].std() - 0.005) < 2e-4


def test_bovy_radial_force_is_the_composites():
    """The host-side F_R(R, 0) the benchmark's initial conditions use: the
    composite's circular speed is 1 at R = 1 (natural units), and it agrees
    with the oracle's force of the same composite."""
    import sys
    from pathlib import Path

    from astrodrift_b200.workloads import bovy_radial_force

    assert abs(float(bovy_radial_force(np.array([1.0]))[0]) + 1.0) < 1e-10
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
    try:
        import oracle
    finally:
        sys.path.pop(0)
    oracle.build()
    R = np.exp(np.linspace(np.log(0.05), np.log(20.0), 64))
    ref = np.array([oracle.force(oracle.bovy(), r, 0.0, 0.0)[0] for r in R])
    np.testing.assert_allclose(bovy_radial_force(R), ref, rtol=1e-11)
