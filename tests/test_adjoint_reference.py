"""The PyTorch restatement of the taped DOP853 map (tests/adjoint_reference.py)
against the CPU oracle, and its own derivatives against finite differences.

These run on the CPU.  They establish that ``replay`` of an oracle step tape
reproduces the oracle's trajectory (so it is the map the adjoint kernel
differentiates) and that its reverse- and forward-mode derivatives agree with
central differences, so the GPU tests can use it as the gradient reference.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from tests import adjoint_reference as ar


def ics(kind, n, seed):
    """Bound orbits for potential kind (0/3 Kepler, 1 Plummer, 2 Bovy)."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.6, 1.6, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    if kind == 2:
        v = rng.uniform(0.8, 1.1, n)  # the composite's circular speed is ~1 at these radii
    elif kind == 1:
        v = np.sqrt(r * r / (r * r + 1.0) ** 1.5) * rng.uniform(0.8, 1.1, n)
    else:
        v = np.sqrt(1.0 / r) * rng.uniform(0.8, 1.1, n)
    return np.stack([r * np.cos(phi), r * np.sin(phi), rng.normal(0, 0.1, n),
                     -v * np.sin(phi), v * np.cos(phi), rng.normal(0, 0.05, n)], axis=1)


def oracle_pot(oracle, kind):
    return {0: oracle.kepler(1.0), 1: oracle.plummer(1.0, 1.0), 2: oracle.bovy(), 3: oracle.kepler(1.0)}[kind]


def oracle_tapes(oracle, kind, y0, ts, tol=1e-10):
    opot = oracle_pot(oracle, kind)
    tapes, refs = [], []
    for i in range(len(y0)):
        res, status, st, tape = oracle.dop853_tape(opot, y0[i], ts, np.log(tol), np.log(tol))
        assert status == 0 and st.accepted == len(tape)
        tapes.append(tape)
        refs.append(res)
    tape, nacc = ar.pad_tapes(tapes)
    return opot, tape, nacc, np.stack(refs, axis=1)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_replay_of_oracle_tape_reproduces_oracle_trajectory(oracle, kind):
    y0 = ics(kind, 4, 10 + kind)
    ts = np.linspace(0.0, 6.0, 13)
    opot, tape, nacc, ref = oracle_tapes(oracle, kind, y0, ts)
    assert min(nacc) > 5
    np.testing.assert_array_equal(tape[:, 0, 2:].numpy(), y0)
    out = ar.replay(kind, ar.params_tensor(opot), ar.potential_constants(opot), torch.tensor(y0), tape, nacc,
                    torch.tensor(np.tile(ts, (len(y0), 1))))
    assert np.abs(out.numpy() - ref).max() / np.abs(ref).max() < 1e-10


def test_replay_backward_time_and_per_particle_grids(oracle):
    kind = 1
    y0 = ics(kind, 3, 4)
    opot = oracle_pot(oracle, kind)
    grids = [np.linspace(0.0, -5.0, 7), np.linspace(0.0, 3.0, 7), np.linspace(0.0, 9.0, 7)]
    tapes, refs = [], []
    for i in range(3):
        res, status, st, tape = oracle.dop853_tape(opot, y0[i], grids[i], np.log(1e-10), np.log(1e-10))
        tapes.append(tape)
        refs.append(res)
    tape, nacc = ar.pad_tapes(tapes)
    out = ar.replay(kind, ar.params_tensor(opot), ar.potential_constants(opot), torch.tensor(y0), tape, nacc,
                    torch.tensor(np.stack(grids)))
    ref = np.stack(refs, axis=1)
    assert np.abs(out.numpy() - ref).max() / np.abs(ref).max() < 1e-10


def _small_case(oracle, kind, n=3, t_end=4.0, nt=9):
    y0 = ics(kind, n, 20 + kind)
    ts = np.linspace(0.0, t_end, nt)
    opot, tape, nacc, _ = oracle_tapes(oracle, kind, y0, ts, tol=1e-9)
    return opot, y0, ts, tape, nacc


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_replay_reverse_mode_matches_central_differences(oracle, kind):
    pot, y0, ts, tape, nacc = _small_case(oracle, kind)
    const = ar.potential_constants(pot)
    tgrid = torch.tensor(np.tile(ts, (len(y0), 1)))
    rng = np.random.default_rng(3)
    w = torch.tensor(rng.normal(size=(len(ts), len(y0), 6)))

    def loss(y, p):
        return (w * ar.replay(kind, p, const, y, tape, nacc, tgrid)).sum()

    y = torch.tensor(y0, requires_grad=True)
    p = ar.params_tensor(pot).requires_grad_(True)
    loss(y, p).backward()
    eps = 1e-6
    for idx in [(0, 0), (1, 4), (2, 2)]:
        e = torch.zeros_like(y)
        e[idx] = eps
        with torch.no_grad():
            fd = (loss(y + e, p) - loss(y - e, p)) / (2 * eps)
        assert abs(fd - y.grad[idx]) <= 1e-6 * max(1.0, abs(fd)), idx
    for j in range(p.numel()):
        e = torch.zeros_like(p)
        e[j] = eps * max(1.0, abs(float(p.detach()[j])))
        with torch.no_grad():
            fd = (loss(y, p + e) - loss(y, p - e)) / (2 * e[j])
        assert abs(fd - p.grad[j]) <= 1e-6 * max(1.0, abs(fd)), ar.PARAM_NAMES[kind][j]


def test_replay_forward_mode_matches_reverse_mode(oracle):
    kind = 2
    pot, y0, ts, tape, nacc = _small_case(oracle, kind, n=2, t_end=3.0, nt=5)
    const = ar.potential_constants(pot)
    tgrid = torch.tensor(np.tile(ts, (len(y0), 1)))
    rng = np.random.default_rng(5)
    w = torch.tensor(rng.normal(size=(len(ts), len(y0), 6)))
    v_y = torch.tensor(rng.normal(size=y0.shape))
    p0 = ar.params_tensor(pot)
    v_p = torch.tensor(rng.normal(size=p0.shape))

    def loss(y, p):
        return (w * ar.replay(kind, p, const, y, tape, nacc, tgrid)).sum()

    _, jv = torch.func.jvp(loss, (torch.tensor(y0), p0), (v_y, v_p))
    y = torch.tensor(y0, requires_grad=True)
    p = p0.clone().requires_grad_(True)
    loss(y, p).backward()
    vjp = (y.grad * v_y).sum() + (p.grad * v_p).sum()
    assert abs(float(jv) - float(vjp)) <= 1e-10 * max(1.0, abs(float(jv)))
