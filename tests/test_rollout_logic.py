"""The rollout's bookkeeping (checkpoints, kept stages, the adjoint state
updated in place, the accumulated KappaEddyDiffusion and heating-factor
adjoints) on the CPU, with a linear stand-in for the step: the gradients
of every rollout mode must equal torch autograd through the same map."""
import torch

from gitm_b200 import adjoint as AD

SHAPES = {"ndensity_s": (6, 8, 5), "idensity_s": (10, 8, 5), "rho": (1, 8, 5), "temperature": (1, 8, 5),
          "velocity": (3, 8, 5), "vert_vel": (6, 8, 5)}
A, B, C = 0.9, 0.01, 0.02


def step_map(state, eddy, hs):
    """new_k = A x_k + B mean(eddy) + C sum(hs) * x_k[..., :1] (differentiable)."""
    e = eddy.mean()
    h = hs.sum()
    return {k: A * v + B * e + C * h * v[..., :1] for k, v in state.items()}


class LinearRunner:
    """StepRunner's interface over step_map, state in self.tensors."""

    def __init__(self):
        g = torch.Generator().manual_seed(3)
        self.tensors = {k: torch.rand(s, dtype=torch.float64, generator=g) + 0.5 for k, s in SHAPES.items()}
        self.tensors["eddy"] = torch.rand(1, 8, 5, dtype=torch.float64, generator=g)
        self.tensors["heating_scale"] = torch.rand(5, dtype=torch.float64, generator=g)
        self.saved_calls = 0
        self.recomputes = 0

    def _load(self, state, eddy, hs):
        for k in AD.STATE:
            self.tensors[k].copy_(state[k])
        if eddy is not None:
            self.tensors["eddy"].copy_(eddy)
        if hs is not None:
            self.tensors["heating_scale"].copy_(hs)

    def state(self):
        return {k: self.tensors[k].clone() for k in AD.STATE}

    def step(self, state, eddy=None, heating_scale=None):
        self._load(state, eddy, heating_scale)
        new = step_map(self.state(), self.tensors["eddy"], self.tensors["heating_scale"])
        for k in AD.STATE:
            self.tensors[k].copy_(new[k])
        return self.state()

    def saved_buffer(self):
        return torch.zeros(1, dtype=torch.float64)

    def step_saving(self, state, saved, eddy=None, heating_scale=None, loaded=False):
        self.saved_calls += 1
        saved.fill_(1.0)  # marks the buffer as written by a saving step
        if loaded:
            # the caller says the arrays hold the step's input already
            for k in AD.STATE:
                assert torch.equal(self.tensors[k], state[k]), k
            state, eddy, heating_scale = self.state(), None, None
        return self.step(state, eddy, heating_scale)

    def stage_bytes_per_step(self):
        return 8

    def vjp_into(self, state, bars, eddy_bar, hs_bar, eddy=None, heating_scale=None, saved=None):
        assert saved is not None and float(saved[0]) == 1.0  # the adjoint reads a saving step's buffer
        self._load(state, eddy, heating_scale)
        x = self.state()
        e, hs = self.tensors["eddy"], self.tensors["heating_scale"]
        h = hs.sum()
        yb_total = 0.0
        hb = 0.0
        for k in AD.STATE:
            y = bars[k]
            yb_total = yb_total + float(y.sum())
            hb = hb + float((y.sum(dim=-1, keepdim=True) * x[k][..., :1]).sum()) * C
            xb = A * y
            xb[..., :1] += C * h * y.sum(dim=-1, keepdim=True)
            bars[k].copy_(xb)
        eddy_bar += B * yb_total / e.numel()
        hs_bar += hb


def _objective(out):
    return (out["ndensity_s"] ** 2).sum() + out["temperature"].sum() * 0.5


def _reference_grads(run, n):
    s0 = {k: run.tensors[k].clone().requires_grad_(True) for k in AD.STATE}
    e = run.tensors["eddy"].clone().requires_grad_(True)
    h = run.tensors["heating_scale"].clone().requires_grad_(True)
    s = s0
    for _ in range(n):
        s = step_map(s, e, h)
    wrt = [s0[k] for k in AD.STATE] + [e, h]
    g = torch.autograd.grad(_objective(s), wrt, allow_unused=True)
    return [torch.zeros_like(t) if gg is None else gg for gg, t in zip(g, wrt)]


def test_rollout_modes_match_autograd():
    for n, every in [(7, 0), (7, 1), (7, 3), (6, 3), (5, 10), (10, 5), (1, 3)]:
        run = LinearRunner()
        want = _reference_grads(run, n)
        s0 = {k: run.tensors[k].clone().requires_grad_(True) for k in AD.STATE}
        e = run.tensors["eddy"].clone().requires_grad_(True)
        h = run.tensors["heating_scale"].clone().requires_grad_(True)
        out = AD.rollout(run, s0, n, every, e, h)
        got = torch.autograd.grad(_objective(out), [s0[k] for k in AD.STATE] + [e, h])
        for name, g, w in zip(list(AD.STATE) + ["eddy", "heating_scale"], got, want):
            assert torch.allclose(g, w, rtol=1e-12, atol=1e-14), (n, every, name)
        # kept stages: one saving step per step in the forward, none after;
        # checkpoints: one saving step per step, the last segment's in the
        # forward, the others' in the backward
        assert run.saved_calls == n, (n, every, run.saved_calls)
