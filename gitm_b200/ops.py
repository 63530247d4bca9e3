"""The vertical step as a torch.library custom op: ``torch.ops.gitm.vertical_step``.

The reference exposes the path to Python only through its post-processing
readers; this op is the Python form of the drop-in, registered with the
dispatcher so that tracing and ``torch.compile`` see it as one node (the
fake kernel gives the output shapes; the CUDA kernel runs libgitmvert.so).

    torch.ops.gitm.vertical_step(ndensity_s, idensity_s, rho, temperature,
                                 velocity, vert_vel, ivel_up, eddy, cos_lat,
                                 sza, mlat, altitude, gravity, dalt_c, inv_r,
                                 dt, n_steps, solver)
        -> (ndensity_s, idensity_s, rho, temperature, velocity, vert_vel)

Arguments are the GitmColumnBatch arrays of one member (include/gitm_vert.h),
float64 CUDA tensors in the native layout [field, cell, column]; altitude,
gravity, dalt_c and inv_r are the member's shared grid [G].  The op is
functional: it advances copies of the six state arrays ``n_steps`` RK4 steps
of ``dt`` seconds (advance_vertical_all, advance_vertical.f90:8-39, with the
coefficient producers of calc_pressure / calc_rates / calc_timestep on the
device) and returns them; the inputs are not modified.  ``solver`` is 0
(Rusanov, vertical_solver_rusanov.f90) or 1 (AUSM, vertical_solver_ausm.f90);
the other flags take the reference defaults.  A column that meets one of the
reference's stop_gitm conditions raises ``gitm_b200.vertical.GitmStop`` (the
call synchronises to read the status words).  There is no CPU kernel: CPU
tensors are refused by the dispatcher.

Backward (Rusanov): the adjoint kernel (gitm_vert_plan_adjoint) gives the
gradients of the six state inputs and of ``eddy``; for n_steps > 1 the
intermediate states are recomputed from the saved inputs.  The other inputs
get no gradient.
"""
from __future__ import annotations

from typing import Tuple

import torch

from . import abi
from . import vertical as V

STATE = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel")
INPUTS = ("ivel_up", "eddy", "cos_lat", "sza", "mlat", "altitude", "gravity", "dalt_c", "inv_r")

_CTX: dict = {}


def _context(device: torch.device, solver: int) -> V.VerticalContext:
    key = (device.index if device.index is not None else torch.cuda.current_device(), int(solver))
    ctx = _CTX.get(key)
    if ctx is None:
        ctx = V.VerticalContext(abi.default_params(solver=int(solver)), device=key[0])
        _CTX[key] = ctx
    return ctx


def _member(state, inputs) -> V.DeviceMember:
    t = dict(zip(STATE, state))
    t.update(zip(INPUTS, inputs))
    for k, v in t.items():
        if not (v.is_cuda and v.dtype == torch.float64):
            raise V.GitmError(f"{k}: expected a float64 CUDA tensor")
    t = {k: v.contiguous() for k, v in t.items()}
    nd = t["ndensity_s"]
    if nd.dim() != 3 or nd.shape[0] != abi.NSPECIES:
        raise V.GitmError("ndensity_s: expected [6, nAlts + 4, n_cols]")
    return V.DeviceMember(int(nd.shape[1]) - 4, int(nd.shape[2]), t)


def _advance(state, inputs, dt: float, n_steps: int, solver: int):
    """Copies of the state advanced n_steps steps (device arrays, checked)."""
    new = [s.detach().clone(memory_format=torch.contiguous_format) for s in state]
    dm = _member(new, [x.detach() for x in inputs])
    ctx = _context(new[0].device, solver)
    plan = V.Plan(ctx, [dm])
    try:
        plan.advance(float(dt), int(n_steps), stream=torch.cuda.current_stream(new[0].device))
        plan.check()
    finally:
        plan.close()
    return [dm.tensors[k] for k in STATE]


@torch.library.custom_op("gitm::vertical_step", mutates_args=(), device_types="cuda")
def vertical_step(ndensity_s: torch.Tensor, idensity_s: torch.Tensor, rho: torch.Tensor,
                  temperature: torch.Tensor, velocity: torch.Tensor, vert_vel: torch.Tensor,
                  ivel_up: torch.Tensor, eddy: torch.Tensor, cos_lat: torch.Tensor, sza: torch.Tensor,
                  mlat: torch.Tensor, altitude: torch.Tensor, gravity: torch.Tensor, dalt_c: torch.Tensor,
                  inv_r: torch.Tensor, dt: float, n_steps: int, solver: int
                  ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    if n_steps < 0:
        raise V.GitmError("n_steps < 0")
    state = (ndensity_s, idensity_s, rho, temperature, velocity, vert_vel)
    inputs = (ivel_up, eddy, cos_lat, sza, mlat, altitude, gravity, dalt_c, inv_r)
    return tuple(_advance(state, inputs, dt, n_steps, solver))


@vertical_step.register_fake
def _(ndensity_s, idensity_s, rho, temperature, velocity, vert_vel, ivel_up, eddy, cos_lat, sza, mlat,
      altitude, gravity, dalt_c, inv_r, dt, n_steps, solver):
    torch._check(ndensity_s.dim() == 3 and ndensity_s.shape[0] == abi.NSPECIES)
    torch._check(idensity_s.shape[0] == abi.NIONS)
    return tuple(torch.empty_like(x, memory_format=torch.contiguous_format)
                 for x in (ndensity_s, idensity_s, rho, temperature, velocity, vert_vel))


def _setup_context(ctx, inputs, output):
    *tensors, dt, n_steps, solver = inputs
    ctx.save_for_backward(*tensors)
    ctx.dt, ctx.n_steps, ctx.solver = float(dt), int(n_steps), int(solver)


def _backward(ctx, *grads):
    saved = ctx.saved_tensors
    state, inputs = list(saved[:6]), list(saved[6:])
    if ctx.solver != abi.SOLVER_RUSANOV:
        raise V.GitmError("gitm::vertical_step backward: the adjoint covers the Rusanov solver")
    # the step inputs of every step, recomputed from the saved inputs
    steps = [[s.detach().clone() for s in state]]
    for _ in range(ctx.n_steps - 1):
        steps.append(_advance(steps[-1], inputs, ctx.dt, 1, ctx.solver))
    bars = [torch.zeros_like(s) if g is None else g.detach().clone(memory_format=torch.contiguous_format)
            for g, s in zip(grads, state)]
    eddy_bar = torch.zeros_like(inputs[1])
    vctx = _context(state[0].device, ctx.solver)
    for x in reversed(steps):
        dm = _member([s.clone() for s in x], [t.detach() for t in inputs])
        plan = V.Plan(vctx, [dm])
        try:
            b = dict(zip(STATE, bars))
            b["eddy"] = eddy_bar
            plan.adjoint([b], ctx.dt)
            plan.check()
        finally:
            plan.close()
    return (*bars, None, eddy_bar, *([None] * 7), None, None, None)


torch.library.register_autograd("gitm::vertical_step", _backward, setup_context=_setup_context)
