"""Gradients through the vertical step: the adjoint kernel
(gitm_vert_plan_adjoint) behind torch.autograd.

GITM has no adjoint; this module adds reverse-mode differentiation of the
step of advance_vertical_all (Rusanov solver, GITM-array form) for
sensitivity studies and data assimilation:

* ``StepRunner`` holds one member's device arrays and a plan; ``step`` runs
  one forward step, ``vjp`` one adjoint step.
* ``vertical_step(runner, state, eddy, heating_scale)`` is one step as a
  differentiable torch op (``torch.autograd.Function``).
* ``rollout(runner, state, n_steps, every, eddy, heating_scale)`` is an
  ``n_steps`` rollout that keeps only every ``every``-th state in memory and
  recomputes the states of a segment when its adjoint runs (checkpointing);
  the recompute saves each step's stage states (``step_saving``) and the
  adjoint kernel reads them.  The last segment keeps its stage states from
  the forward (the backward would recompute it first, into the same
  buffers), so it is not recomputed.  ``every = 0`` keeps every step's input state
  and stage states from the forward itself (no recompute: about seven
  states of memory per step, ``stage_bytes_per_step``).
* ``o_n2_objective`` is the column-weighted log(n_O / n_N2) at one altitude
  level.

The state is the GITM arrays the step reads and writes: NDensityS,
IDensityS, Rho, Temperature (normalised), Velocity, VerticalVelocity, as
[field, cell, column] float64 CUDA tensors.  All compute goes through
libgitmvert.so.
"""
from __future__ import annotations

import torch

from . import synthetic
from . import vertical as V

STATE = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel")


class StepRunner:
    """One member's arrays and a plan over them; the state arrays are
    overwritten by every call."""

    def __init__(self, ctx: V.VerticalContext, member, dt: float, autotune: bool = True):
        self.ctx = ctx
        self.dt = float(dt)
        self.dm = V.device_member(member) if isinstance(member, synthetic.Member) else member
        if self.dm.tensors.get("heating") is not None and self.dm.tensors.get("heating_scale") is None:
            self.dm.tensors["heating_scale"] = torch.ones(self.dm.n_cols, dtype=torch.float64,
                                                          device=self.dm.tensors["rho"].device)
        self.plan = V.Plan(ctx, [self.dm])
        if autotune:
            # one step per call: pick the fastest launch shape for that
            # (the state is left as it was)
            self.plan.autotune(self.dt, 1)

    @property
    def tensors(self):
        return self.dm.tensors

    def _load(self, state, eddy=None, heating_scale=None):
        for k in STATE:
            self.dm.tensors[k].copy_(state[k])
        if eddy is not None:
            self.dm.tensors["eddy"].copy_(eddy)
        if heating_scale is not None and self.dm.tensors.get("heating_scale") is not None:
            self.dm.tensors["heating_scale"].copy_(heating_scale)

    def state(self) -> dict:
        return {k: self.dm.tensors[k].clone() for k in STATE}

    def step(self, state, eddy=None, heating_scale=None) -> dict:
        """One forward step from `state`; returns the new state (copies)."""
        self._load(state, eddy, heating_scale)
        self.plan.advance(self.dt, 1)
        return self.state()

    def saved_buffer(self):
        """A device buffer for the stage states of one step."""
        return torch.empty(self.plan.saved_state_doubles(), dtype=torch.float64,
                           device=self.dm.tensors["rho"].device)

    def step_saving(self, state, saved, eddy=None, heating_scale=None, loaded=False) -> dict:
        """step() that also writes the step's stage states to `saved`.
        loaded: the runner's arrays hold `state`, eddy and heating_scale
        already (the output of the previous call), so nothing is copied in."""
        if not loaded:
            self._load(state, eddy, heating_scale)
        self.plan.advance_saving(self.dt, saved)
        return self.state()

    def stage_bytes_per_step(self) -> int:
        """Device bytes one step keeps when a rollout keeps its stages: the
        saved stage states and the step's input state."""
        n = self.plan.saved_state_doubles() + sum(self.dm.tensors[k].numel() for k in STATE)
        return 8 * n

    def vjp_into(self, state, bars, eddy_bar, hs_bar, eddy=None, heating_scale=None, saved=None):
        """vjp() in place: `bars` holds ybar for the STATE arrays on entry and
        xbar on return (contiguous float64 CUDA tensors); eddy_bar / hs_bar
        (may be None) accumulate."""
        self._load(state, eddy, heating_scale)
        b = dict(bars)
        b["eddy"] = eddy_bar
        b["heating_scale"] = hs_bar if self.dm.tensors.get("heating_scale") is not None else None
        self.plan.adjoint([b], self.dt, saved=saved)

    def vjp(self, state, ybar, eddy=None, heating_scale=None, saved=None):
        """Adjoint of one step taken from `state`: returns (xbar, eddy_bar,
        heating_scale_bar).  ybar: dict of output adjoints (None = zero);
        saved: the buffer step_saving filled for this step, or None (the
        adjoint kernel then recomputes the stage states)."""
        self._load(state, eddy, heating_scale)
        bars = {}
        for k in STATE:
            y = ybar.get(k)
            bars[k] = torch.zeros_like(self.dm.tensors[k]) if y is None else y.detach().clone().contiguous()
        for k in ("log_ns", "ndensity"):
            if ybar.get(k) is not None:
                bars[k] = ybar[k].detach().contiguous()
        bars["eddy"] = torch.zeros_like(self.dm.tensors["eddy"])
        hs = self.dm.tensors.get("heating_scale")
        bars["heating_scale"] = None if hs is None else torch.zeros_like(hs)
        self.plan.adjoint([bars], self.dt, saved=saved)
        return {k: bars[k] for k in STATE}, bars["eddy"], bars["heating_scale"]

    def check(self):
        self.plan.check()

    def close(self):
        self.plan.close()


class _Step(torch.autograd.Function):
    @staticmethod
    def forward(ctx, runner, eddy, heating_scale, *state):
        out = runner.step(dict(zip(STATE, state)), eddy, heating_scale)
        ctx.runner = runner
        ctx.save_for_backward(eddy, heating_scale, *state)
        return tuple(out[k] for k in STATE)

    @staticmethod
    def backward(ctx, *ybar):
        eddy, hs, *state = ctx.saved_tensors
        xbar, eb, hb = ctx.runner.vjp(dict(zip(STATE, state)), dict(zip(STATE, ybar)), eddy, hs)
        return (None, eb, hb, *[xbar[k] for k in STATE])


def vertical_step(runner: StepRunner, state: dict, eddy=None, heating_scale=None) -> dict:
    """One step as a differentiable op; eddy / heating_scale default to the
    runner's arrays (then not differentiated)."""
    if eddy is None:
        eddy = runner.tensors["eddy"].clone()
    if heating_scale is None:
        hs = runner.tensors.get("heating_scale")
        heating_scale = torch.ones(1, device=eddy.device, dtype=eddy.dtype) if hs is None else hs.clone()
    out = _Step.apply(runner, eddy, heating_scale, *[state[k] for k in STATE])
    return dict(zip(STATE, out))


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, runner, n_steps, every, eddy, heating_scale, *state):
        s = dict(zip(STATE, (t.detach() for t in state)))
        ckpts, stages = [], []
        if every == 0:
            need = n_steps * runner.stage_bytes_per_step()
            dev = runner.tensors["rho"].device
            free = torch.cuda.mem_get_info(dev)[0] if dev.type == "cuda" else float("inf")
            if need > 0.9 * free:
                raise V.GitmError(f"rollout with every = 0 keeps {need / 1e9:.1f} GB of stage states, "
                                  f"{free / 1e9:.1f} GB free: use checkpoints (every > 0)")
            s = {k: v.clone() for k, v in s.items()}
        # with checkpoints, the last segment keeps its stage states from the
        # forward (its recompute would be the first thing the backward does)
        t_tail = 0 if every == 0 else ((n_steps - 1) // every) * every if n_steps > 0 else 0
        for t in range(n_steps):
            if t >= t_tail:
                # keep the step's input and its stage states
                buf = runner.saved_buffer()
                stages.append((s, buf))
                s = runner.step_saving(s, buf, eddy, heating_scale)
                continue
            if t % every == 0:
                ckpts.append({k: v.clone() for k, v in s.items()})
            s = runner.step(s, eddy, heating_scale)
        ctx.runner, ctx.n_steps, ctx.every, ctx.ckpts, ctx.stages = runner, n_steps, every, ckpts, stages
        ctx.save_for_backward(eddy, heating_scale)
        return tuple(s[k] for k in STATE)

    @staticmethod
    def backward(ctx, *ybar):
        eddy, hs = ctx.saved_tensors
        runner = ctx.runner
        # the running adjoint, updated in place step by step
        y = {k: (torch.zeros_like(runner.tensors[k]) if g is None else g.detach().clone().contiguous())
             for k, g in zip(STATE, ybar)}
        eb = torch.zeros_like(runner.tensors["eddy"])
        hrun = runner.tensors.get("heating_scale")
        hb = None if hrun is None else torch.zeros_like(hrun)
        n, k = ctx.n_steps, ctx.every
        # the steps whose stages the forward kept (all of them with k = 0,
        # else the last segment), then the checkpointed segments
        saved = []  # one stage-state buffer per step of a segment, reused
        for j in reversed(range(len(ctx.stages))):
            st, buf = ctx.stages[j]
            runner.vjp_into(st, y, eb, hb, eddy, hs, saved=buf)
            ctx.stages[j] = None
            if k > 0:
                saved.insert(0, buf)
        if k > 0:
            for seg in reversed(range(len(ctx.ckpts))):
                t0 = seg * k
                t1 = min(t0 + k, n)
                # recompute the segment's step inputs, saving each step's stages
                states = [ctx.ckpts[seg]]
                while len(saved) < t1 - t0:
                    saved.append(runner.saved_buffer())
                for j in range(t1 - t0):
                    # from the second step on, the runner's arrays hold the
                    # step's input (the previous step's output) already
                    nxt = runner.step_saving(states[-1], saved[j], eddy, hs, loaded=j > 0)
                    if j < t1 - t0 - 1:
                        states.append(nxt)
                for j in reversed(range(t1 - t0)):
                    runner.vjp_into(states[j], y, eb, hb, eddy, hs, saved=saved[j])
                ctx.ckpts[seg] = None
        eb = eb.reshape(eddy.shape)
        if hb is None or hb.shape != hs.shape:
            hb = torch.zeros_like(hs)
        return (None, None, None, eb, hb, *[y[k2] for k2 in STATE])


def rollout(runner: StepRunner, state: dict, n_steps: int, every: int = 10, eddy=None,
            heating_scale=None) -> dict:
    """n_steps steps with checkpoints every `every` steps, or with every
    step's stage states kept when every = 0 (see module doc)."""
    if eddy is None:
        eddy = runner.tensors["eddy"].clone()
    if heating_scale is None:
        hs = runner.tensors.get("heating_scale")
        heating_scale = torch.ones(1, device=eddy.device, dtype=eddy.dtype) if hs is None else hs.clone()
    out = _Rollout.apply(runner, int(n_steps), max(0, int(every)), eddy, heating_scale,
                         *[state[k] for k in STATE])
    return dict(zip(STATE, out))


def o_n2_objective(ndensity_s, weights, level: int):
    """sum_c w_c log(n_O / n_N2) at cell index `level` (0 = cell -1)."""
    return (weights * (torch.log(ndensity_s[0, level]) - torch.log(ndensity_s[2, level]))).sum()


def level_of(altitude, alt_m: float) -> int:
    """Cell index (0 = cell -1) whose altitude is closest to alt_m."""
    a = torch.as_tensor(altitude).reshape(-1)
    return int(torch.argmin((a - alt_m).abs()))
