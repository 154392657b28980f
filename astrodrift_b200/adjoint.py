"""Differentiable DOP853 trajectories: the discrete adjoint behind
``torch.autograd.Function``.

    out = trajectory(y0, capi.bovy(), params=p, ts=ts, rtol=1e-10, atol=1e-10)
    loss = ((out[-1, :, :3] - target) ** 2).sum()
    loss.backward()          # y0.grad (N, 6), p.grad (P,)

The forward pass is drift_integrate with a step tape: every accepted step's
(t_old, h, y_old) is recorded on the device.  The backward pass is
drift_integrate_adjoint, which replays each particle's steps in reverse and
returns the exact derivative of the computed trajectory for that step
sequence (step sizes held fixed).  ``params`` are the potential's
differentiable parameters, in the order of ``PARAM_NAMES[kind]``; their
values replace the potential's fields.  Everything runs on the GPU; there is
no CPU path.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import capi

PARAM_NAMES = {
    capi.POT_KEPLER: ("amp",),
    capi.POT_KEPLER_CARTESIAN: ("amp",),
    capi.POT_PLUMMER: ("amp", "b"),
    capi.POT_BOVY: ("mn_amp", "mn_a", "mn_b", "nfw_amp", "nfw_a", "bulge_k"),
}


def params_of(pot: capi.DriftPotential) -> list[float]:
    """The differentiable parameters of a potential, in PARAM_NAMES order."""
    return [float(getattr(pot, name)) for name in PARAM_NAMES[pot.kind]]


def with_params(pot: capi.DriftPotential, values) -> capi.DriftPotential:
    """A copy of ``pot`` with its differentiable parameters replaced."""
    out = capi.DriftPotential()
    ctypes.memmove(ctypes.byref(out), ctypes.byref(pot), ctypes.sizeof(pot))
    names = PARAM_NAMES[pot.kind]
    values = [float(v) for v in values]
    if len(values) != len(names):
        raise ValueError(f"{len(names)} parameters expected ({', '.join(names)}), got {len(values)}")
    for name, v in zip(names, values):
        setattr(out, name, v)
    return out


@dataclass
class _Spec:
    pot: capi.DriftPotential
    ts: object            # device tensor (nt,) or None
    t_end: object         # device tensor (N,) or None
    t0: float
    nt: int
    rtol: float
    atol: float
    precision: int
    schedule: int
    tape_steps: int | None
    max_steps: int
    stride: int = 1


def _launch(spec: _Spec, pot, y0, n, out=None, tape=None, tape_steps=0, acc=None, status=None):
    import torch

    L = capi.make_launch(capi.DOP853, pot, n, spec.nt, rtol=spec.rtol, atol=spec.atol,
                         precision=spec.precision, schedule=spec.schedule, t0=spec.t0,
                         max_steps=spec.max_steps)
    L.y0 = y0.data_ptr()
    if spec.ts is not None:
        L.ts = spec.ts.data_ptr()
    else:
        L.t_end = spec.t_end.data_ptr()
    L.out = out.data_ptr() if out is not None else None
    L.n_accepted = acc.data_ptr() if acc is not None else None
    L.status = status.data_ptr() if status is not None else None
    if tape is not None:
        L.tape, L.tape_steps, L.tape_stride = tape.data_ptr(), tape_steps, spec.stride
    ws = None
    need = capi.query_workspace(L)
    if need:
        ws = torch.empty(need, dtype=torch.uint8, device=y0.device)
        L.workspace, L.workspace_bytes = ws.data_ptr(), need
    capi.integrate_device(L, torch.cuda.current_stream(y0.device).cuda_stream)
    return ws  # stream-ordered: freeing it after the launch is safe


class Dop853Trajectory:
    """``torch.autograd.Function`` wrapper, built lazily so importing this
    module does not import torch."""

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            import torch

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, y0, params, spec):
                    n = y0.shape[0]
                    dev = y0.device
                    pot = with_params(spec.pot, params.detach().cpu().tolist()) if params is not None \
                        else spec.pot
                    acc = torch.zeros(n, dtype=torch.int32, device=dev)
                    status = torch.zeros(n, dtype=torch.uint8, device=dev)
                    steps = spec.tape_steps
                    if steps is None:
                        # size the tape from an untaped pass (same arithmetic, same steps)
                        _launch(spec, pot, y0, n, acc=acc, status=status)
                        steps = max(int(acc.max().item()), 1)
                    tape = torch.empty((n, capi.tape_doubles(steps, spec.stride)), dtype=torch.float64,
                                       device=dev)
                    out = torch.empty((spec.nt, n, 6), dtype=torch.float64, device=dev)
                    _launch(spec, pot, y0, n, out=out, tape=tape, tape_steps=steps, acc=acc, status=status)
                    st = status.cpu().numpy()
                    if (st == capi.PARTICLE_TAPE_FULL).any():
                        raise RuntimeError(f"the step tape of {steps} rows per particle is too small for "
                                           f"{int((st == capi.PARTICLE_TAPE_FULL).sum())} particles")
                    ctx.save_for_backward(tape, acc, status)
                    ctx.spec, ctx.pot, ctx.steps = spec, pot, steps
                    ctx.has_params = params is not None
                    ctx.params_device = params.device if params is not None else None
                    return out

                @staticmethod
                def backward(ctx, grad_out):
                    tape, acc, status = ctx.saved_tensors
                    spec = ctx.spec
                    n = tape.shape[0]
                    dev = tape.device
                    g = grad_out.detach().to(dtype=torch.float64).contiguous()
                    grad_y0 = torch.empty((n, 6), dtype=torch.float64, device=dev)
                    grad_pp = torch.empty((n, capi.ADJOINT_MAX_PARAMS), dtype=torch.float64, device=dev)
                    A = capi.DriftAdjointLaunch()
                    A.method = capi.DOP853
                    A.potential = ctx.pot
                    A.n, A.nt, A.t0 = n, spec.nt, spec.t0
                    if spec.ts is not None:
                        A.ts = spec.ts.data_ptr()
                    else:
                        A.t_end = spec.t_end.data_ptr()
                    A.tape, A.tape_steps, A.tape_stride = tape.data_ptr(), ctx.steps, spec.stride
                    A.n_accepted, A.status = acc.data_ptr(), status.data_ptr()
                    A.grad_out, A.grad_y0, A.grad_params = g.data_ptr(), grad_y0.data_ptr(), grad_pp.data_ptr()
                    capi.integrate_adjoint_device(A, torch.cuda.current_stream(dev).cuda_stream)
                    grad_params = None
                    if ctx.has_params:
                        grad_params = grad_pp[:, : len(PARAM_NAMES[spec.pot.kind])].sum(0).to(
                            ctx.params_device)
                    return grad_y0, grad_params, None

            cls._fn = _Fn
        return cls._fn


def trajectory(y0, potential: capi.DriftPotential, *, params=None, ts=None, t_end=None,
               t0: float = 0.0, nt: int | None = None, rtol: float = 1e-10, atol: float = 1e-10,
               precision: int = capi.FMA, schedule: int = capi.ORDERED,
               tape_steps: int | None = None, max_steps: int = 0, checkpoint_stride: int = 1):
    """DOP853 trajectories (nt, N, 6) on the GPU, differentiable with respect
    to ``y0`` (N, 6) and ``params`` (the potential's PARAM_NAMES values).

    ``ts`` is a shared output grid; or ``t_end`` (N,) with ``nt`` gives each
    particle the grid t0..t_end[i].  ``tape_steps`` bounds the accepted steps
    recorded per particle (default: sized by an untaped pass).
    ``checkpoint_stride`` m > 1 keeps a full state every m steps and every
    step's size (about 8 + 64/m bytes per step instead of 64); the backward
    pass recomputes the states in between.  Particles
    that fail (step cap, non-finite state) have NaN samples and NaN
    gradients.
    """
    import torch

    if not isinstance(y0, torch.Tensor) or y0.device.type != "cuda":
        raise TypeError("y0 must be a CUDA tensor")
    y0c = y0.to(torch.float64).contiguous()
    if y0c.dim() != 2 or y0c.shape[1] != 6:
        raise ValueError("y0 must have shape (N, 6)")
    dev = y0c.device

    def as_dev(a):
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.asarray(a, dtype=np.float64))
        return t.to(device=dev, dtype=torch.float64).contiguous()

    if ts is not None:
        ts_t = as_dev(ts)
        spec = _Spec(potential, ts_t, None, t0, int(ts_t.numel()), rtol, atol, precision, schedule,
                     tape_steps, max_steps, checkpoint_stride)
    else:
        if t_end is None or nt is None:
            raise ValueError("give ts, or t_end and nt")
        spec = _Spec(potential, None, as_dev(t_end), t0, int(nt), rtol, atol, precision, schedule,
                     tape_steps, max_steps, checkpoint_stride)
    if not 1 <= checkpoint_stride <= capi.MAX_TAPE_STRIDE:
        raise ValueError(f"checkpoint_stride must be in [1, {capi.MAX_TAPE_STRIDE}]")
    if params is not None:
        params = torch.as_tensor(params, dtype=torch.float64)
        if params.numel() != len(PARAM_NAMES[potential.kind]):
            raise ValueError(f"params must hold {', '.join(PARAM_NAMES[potential.kind])}")
    return Dop853Trajectory.function().apply(y0c, params, spec)
