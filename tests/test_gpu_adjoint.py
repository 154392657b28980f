"""The discrete-adjoint kernel (drift_integrate_adjoint) and its
torch.autograd.Function.

The forward launch records each particle's accepted steps; the reference
for the gradients is tests/adjoint_reference.replay run on that same tape
(the same discrete map, in plain PyTorch float64 on the CPU):
  * reverse mode: torch autograd of replay, elementwise;
  * forward mode: torch.func.jvp of replay, as a dot-product test
    <g, J v> = <J^T g, v>;
  * central finite differences of replay (frozen step sequence);
  * central finite differences of the production integrator, whose step
    sizes adapt to the perturbed orbit (loose: the step-size controller is
    not differentiated).
Tolerances: 1e-8 relative between the kernel and autograd (both exact
derivatives of the same map; they differ by rounding only), 1e-6 against
frozen-step differences, 1e-4 against free-adaptive differences.
"""

from __future__ import annotations

import numpy as np
import pytest

from astrodrift_b200 import adjoint, capi
from tests import adjoint_reference as ar
from tests.test_adjoint_reference import ics

pytestmark = pytest.mark.gpu

KINDS = {"kepler": (0, capi.kepler(1.0)), "plummer": (1, capi.plummer(1.0, 1.0)), "bovy": (2, None)}


def _pot(name):
    kind, pot = KINDS[name]
    return kind, (capi.bovy() if name == "bovy" else pot)


def taped(torch, pot, y0, *, ts=None, t_end=None, nt=None, rtol=1e-10, max_steps=0, tape_steps=None,
          stride=1):
    """Forward launch with a tape, through the C ABI.  Returns device tensors."""
    dev = torch.device("cuda:0")
    n = len(y0)
    nt = len(ts) if ts is not None else nt
    y0_d = torch.tensor(y0, device=dev)
    grid = torch.tensor(ts if ts is not None else t_end, device=dev)
    acc = torch.zeros(n, dtype=torch.int32, device=dev)
    st = torch.zeros(n, dtype=torch.uint8, device=dev)
    out = torch.empty((nt, n, 6), dtype=torch.float64, device=dev)

    def launch(tape=None, steps=0):
        L = capi.make_launch(capi.DOP853, pot, n, nt, rtol=rtol, atol=rtol, precision=capi.FMA,
                             schedule=capi.ORDERED, max_steps=max_steps)
        L.y0, L.out, L.n_accepted, L.status = y0_d.data_ptr(), out.data_ptr(), acc.data_ptr(), st.data_ptr()
        if ts is not None:
            L.ts = grid.data_ptr()
        else:
            L.t_end = grid.data_ptr()
        if tape is not None:
            L.tape, L.tape_steps, L.tape_stride = tape.data_ptr(), steps, stride
        ws = torch.zeros(max(capi.query_workspace(L), 8), dtype=torch.uint8, device=dev)
        L.workspace, L.workspace_bytes = ws.data_ptr(), ws.numel()
        capi.integrate_device(L, 0)
        torch.cuda.synchronize()

    if tape_steps is None:
        launch()
        tape_steps = max(int(acc.max()), 1)
    tape = torch.empty((n, capi.tape_doubles(tape_steps, stride)), dtype=torch.float64, device=dev)
    launch(tape, tape_steps)
    return dict(y0=y0_d, grid=grid, out=out, acc=acc, status=st, tape=tape, steps=tape_steps, nt=nt,
                shared=ts is not None, stride=stride)


def adjoint_kernel(torch, pot, f, grad_out):
    n = f["y0"].shape[0]
    dev = f["y0"].device
    gy = torch.empty((n, 6), dtype=torch.float64, device=dev)
    gp = torch.empty((n, capi.ADJOINT_MAX_PARAMS), dtype=torch.float64, device=dev)
    g = torch.as_tensor(grad_out, dtype=torch.float64).to(dev).contiguous()
    A = capi.DriftAdjointLaunch(method=capi.DOP853, potential=pot, n=n, nt=f["nt"])
    if f["shared"]:
        A.ts = f["grid"].data_ptr()
    else:
        A.t_end = f["grid"].data_ptr()
    A.tape, A.tape_steps, A.tape_stride = f["tape"].data_ptr(), f["steps"], f["stride"]
    A.n_accepted, A.status = f["acc"].data_ptr(), f["status"].data_ptr()
    A.grad_out, A.grad_y0, A.grad_params = g.data_ptr(), gy.data_ptr(), gp.data_ptr()
    capi.integrate_adjoint_device(A, 0)
    torch.cuda.synchronize()
    return gy.cpu().numpy(), gp.cpu().numpy()


def replay_inputs(torch, f, ts=None, t_end=None):
    tape = f["tape"].cpu().reshape(f["tape"].shape[0], -1, 8)
    nacc = f["acc"].cpu().numpy().astype(np.int64)
    n, nt = tape.shape[0], f["nt"]
    if ts is not None:
        tgrid = torch.tensor(np.tile(ts, (n, 1)))
    else:
        tgrid = torch.tensor(np.stack([[capi_grid(0.0, te, nt, k) for k in range(nt)] for te in t_end]))
    return tape, list(nacc), tgrid


def capi_grid(start, end, steps, k):
    # OutputGrid::sample (shared/src/config.rs:57-66)
    return end if k == steps - 1 else start + (end - start) * k / (steps - 1)


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.mark.parametrize("name", ["kepler", "plummer", "bovy"])
def test_adjoint_matches_reverse_mode_of_the_replayed_map(cuda_device, name):
    import torch

    kind, pot = _pot(name)
    y0 = ics(kind, 24, 40 + kind)
    ts = np.linspace(0.0, 8.0, 9)
    f = taped(torch, pot, y0, ts=ts)
    assert (f["status"].cpu().numpy() == 0).all()
    rng = np.random.default_rng(1)
    w = rng.normal(size=(len(ts), len(y0), 6))
    gy, gp = adjoint_kernel(torch, pot, f, w)

    tape, nacc, tgrid = replay_inputs(torch, f, ts=ts)
    y = torch.tensor(y0, requires_grad=True)
    p = ar.params_tensor(pot).requires_grad_(True)
    out = ar.replay(kind, p, ar.potential_constants(pot), y, tape, nacc, tgrid)
    # the replayed map is the device trajectory
    assert rel(out.detach().numpy(), f["out"].cpu().numpy()) < 1e-11
    (torch.tensor(w) * out).sum().backward()
    assert rel(gy, y.grad.numpy()) < 1e-8
    P = len(adjoint.PARAM_NAMES[pot.kind])
    assert rel(gp[:, :P].sum(0), p.grad.numpy()) < 1e-8


def test_adjoint_dot_product_with_forward_mode(cuda_device):
    import torch

    kind, pot = _pot("bovy")
    y0 = ics(kind, 8, 7)
    ts = np.linspace(0.0, 5.0, 6)
    f = taped(torch, pot, y0, ts=ts)
    rng = np.random.default_rng(2)
    w = torch.tensor(rng.normal(size=(len(ts), len(y0), 6)))
    gy, gp = adjoint_kernel(torch, pot, f, w.numpy())
    tape, nacc, tgrid = replay_inputs(torch, f, ts=ts)
    p0 = ar.params_tensor(pot)
    v_y = torch.tensor(rng.normal(size=y0.shape))
    v_p = torch.tensor(rng.normal(size=p0.shape))
    const = ar.potential_constants(pot)
    _, jv = torch.func.jvp(lambda y, p: (w * ar.replay(kind, p, const, y, tape, nacc, tgrid)).sum(),
                           (torch.tensor(y0), p0), (v_y, v_p))
    vjp = float((gy * v_y.numpy()).sum() + (gp[:, : len(p0)].sum(0) * v_p.numpy()).sum())
    assert abs(float(jv) - vjp) <= 1e-9 * max(1.0, abs(float(jv)))


def test_adjoint_matches_frozen_step_central_differences(cuda_device):
    import torch

    kind, pot = _pot("plummer")
    y0 = ics(kind, 4, 3)
    ts = np.linspace(0.0, 6.0, 7)
    f = taped(torch, pot, y0, ts=ts)
    rng = np.random.default_rng(4)
    w = rng.normal(size=(len(ts), len(y0), 6))
    gy, gp = adjoint_kernel(torch, pot, f, w)
    tape, nacc, tgrid = replay_inputs(torch, f, ts=ts)
    const = ar.potential_constants(pot)
    p0 = ar.params_tensor(pot)

    def loss(y, p):
        return float((torch.tensor(w) * ar.replay(kind, p, const, torch.tensor(y), tape, nacc, tgrid)).sum())

    eps = 1e-6
    for i, c in [(0, 0), (1, 3), (2, 5), (3, 1)]:
        e = np.zeros_like(y0)
        e[i, c] = eps
        fd = (loss(y0 + e, p0) - loss(y0 - e, p0)) / (2 * eps)
        assert abs(fd - gy[i, c]) <= 1e-6 * max(1.0, abs(fd))
    for j in range(2):
        e = torch.zeros(2, dtype=torch.float64)
        e[j] = eps
        fd = (loss(y0, p0 + e) - loss(y0, p0 - e)) / (2 * eps)
        assert abs(fd - gp[:, j].sum()) <= 1e-6 * max(1.0, abs(fd))


def test_autograd_function_matches_free_adaptive_differences(cuda_device):
    import torch

    kind, pot = _pot("bovy")
    y0 = ics(kind, 16, 11)
    ts = np.linspace(0.0, 10.0, 3)
    rng = np.random.default_rng(6)
    target = torch.tensor(rng.normal(size=(len(y0), 3)) * 0.1, device="cuda")
    pvals = adjoint.params_of(pot)

    def loss_of(y, p):
        out = adjoint.trajectory(y, pot, params=p, ts=ts, rtol=1e-11, atol=1e-11)
        return ((out[-1, :, :3] - target) ** 2).sum()

    y = torch.tensor(y0, device="cuda", requires_grad=True)
    p = torch.tensor(pvals, dtype=torch.float64, requires_grad=True)
    loss_of(y, p).backward()
    eps = 1e-6
    with torch.no_grad():
        for i, c in [(0, 0), (5, 4), (9, 2)]:
            e = torch.zeros_like(y)
            e[i, c] = eps
            fd = (float(loss_of(y + e, p)) - float(loss_of(y - e, p))) / (2 * eps)
            assert abs(fd - float(y.grad[i, c])) <= 1e-4 * max(1.0, abs(fd))
        for j, name in enumerate(adjoint.PARAM_NAMES[pot.kind]):
            if name not in ("mn_amp", "mn_a", "nfw_a"):
                continue
            e = torch.zeros_like(p)
            e[j] = eps
            fd = (float(loss_of(y, p + e)) - float(loss_of(y, p - e))) / (2 * eps)
            assert abs(fd - float(p.grad[j])) <= 1e-4 * max(1.0, abs(fd)), name


def test_per_particle_grids_and_backward_time(cuda_device):
    import torch

    kind, pot = _pot("plummer")
    y0 = ics(kind, 6, 9)
    t_end = np.array([3.0, -4.0, 7.5, -1.0, 2.0, 5.0])
    nt = 5
    f = taped(torch, pot, y0, t_end=t_end, nt=nt)
    assert (f["status"].cpu().numpy() == 0).all()
    rng = np.random.default_rng(8)
    w = rng.normal(size=(nt, len(y0), 6))
    gy, gp = adjoint_kernel(torch, pot, f, w)
    tape, nacc, tgrid = replay_inputs(torch, f, t_end=t_end)
    y = torch.tensor(y0, requires_grad=True)
    p = ar.params_tensor(pot).requires_grad_(True)
    out = ar.replay(kind, p, ar.potential_constants(pot), y, tape, nacc, tgrid)
    assert rel(out.detach().numpy(), f["out"].cpu().numpy()) < 1e-11
    (torch.tensor(w) * out).sum().backward()
    assert rel(gy, y.grad.numpy()) < 1e-8
    assert rel(gp[:, :2].sum(0), p.grad.numpy()) < 1e-8


def test_failed_particles_get_nan_gradients_and_a_full_tape_is_reported(cuda_device):
    import torch

    kind, pot = _pot("plummer")
    y0 = ics(kind, 4, 12)
    ts = np.linspace(0.0, 20.0, 5)
    f = taped(torch, pot, y0, ts=ts, max_steps=6, tape_steps=64)
    st = f["status"].cpu().numpy()
    assert (st == capi.PARTICLE_MAX_STEPS).all()
    gy, gp = adjoint_kernel(torch, pot, f, np.ones((len(ts), 4, 6)))
    assert np.isnan(gy).all() and np.isnan(gp).all()

    f = taped(torch, pot, y0, ts=ts, tape_steps=3)
    assert (f["status"].cpu().numpy() == capi.PARTICLE_TAPE_FULL).all()
    with pytest.raises(RuntimeError, match="tape"):
        adjoint.trajectory(torch.tensor(y0, device="cuda"), pot, ts=ts, tape_steps=3)


@pytest.mark.parametrize("stride", [2, 5, 16])
@pytest.mark.parametrize("name", ["plummer", "bovy"])
def test_checkpointed_tape_gives_the_same_gradients(cuda_device, name, stride):
    """A tape with a checkpoint every `stride` steps (every step's h kept)
    holds 8 + 64/stride bytes per step; the adjoint recomputes the states in
    between and must return the full tape's gradients."""
    import torch

    kind, pot = _pot(name)
    y0 = ics(kind, 40, 70 + kind)
    t_end = np.random.default_rng(3).uniform(2.0, 9.0, 40)  # step counts not multiples of stride
    full = taped(torch, pot, y0, t_end=t_end, nt=7)
    cp = taped(torch, pot, y0, t_end=t_end, nt=7, stride=stride, tape_steps=full["steps"])
    np.testing.assert_array_equal(cp["out"].cpu().numpy(), full["out"].cpu().numpy())
    assert cp["tape"].numel() < full["tape"].numel() * (8 + 64 / stride + 16) / 64
    w = np.random.default_rng(4).normal(size=(7, 40, 6))
    gy_full, gp_full = adjoint_kernel(torch, pot, full, w)
    gy_cp, gp_cp = adjoint_kernel(torch, pot, cp, w)
    assert rel(gy_cp, gy_full) < 1e-10
    P = len(adjoint.PARAM_NAMES[pot.kind])
    assert rel(gp_cp[:, :P], gp_full[:, :P]) < 1e-10


def test_autograd_function_with_checkpoints(cuda_device):
    import torch

    kind, pot = _pot("bovy")
    y0 = torch.tensor(ics(kind, 32, 90), device="cuda")
    ts = np.linspace(0.0, 6.0, 4)
    grads = []
    for stride in (1, 8):
        y = y0.clone().requires_grad_(True)
        p = torch.tensor(adjoint.params_of(pot), dtype=torch.float64, requires_grad=True)
        out = adjoint.trajectory(y, pot, params=p, ts=ts, checkpoint_stride=stride)
        (out[-1, :, :3] ** 2).sum().backward()
        grads.append((y.grad.cpu().numpy(), p.grad.numpy()))
    assert rel(grads[1][0], grads[0][0]) < 1e-10 and rel(grads[1][1], grads[0][1]) < 1e-10
