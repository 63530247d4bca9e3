"""The adjoint kernel (gitm_vert_plan_adjoint) against torch autograd through
the FP64 PyTorch transcription of the step (tests/torch_step.py), the
checkpointed rollout against step-by-step composition, and rollout gradients
against central finite differences of the GPU forward."""
import numpy as np
import pytest
import torch

from gitm_b200 import abi, synthetic
from tests import torch_step as TS

pytestmark = pytest.mark.gpu

OUT_KEYS = {"ndensity_s": "nd", "idensity_s": "ion", "rho": "rho", "temperature": "temp", "velocity": "vel",
            "vert_vel": "ww"}


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda")


def _ybar(m, gen, dev):
    """Random output adjoints with the output shapes (unit scale per field)."""
    y = {}
    for k in OUT_KEYS:
        a = getattr(m, k)
        y[k] = torch.randn(a.shape, generator=gen, dtype=torch.float64).to(dev)
    y["log_ns"] = torch.randn(m.ndensity_s.shape, generator=gen, dtype=torch.float64).to(dev)
    y["ndensity"] = torch.randn(m.rho.shape, generator=gen, dtype=torch.float64).to(dev)
    return y


def _torch_vjp(m, p, dt, y, dev):
    st, inp = TS.from_member(m, device=dev, requires_grad=True)
    eddy = inp["eddy"].clone().requires_grad_(True)
    inp["eddy"] = eddy
    hs = None
    if inp["heating"] is not None:
        hs = inp["heating_scale"].clone().requires_grad_(True)
        inp["heating_scale"] = hs
    out = TS.step(st, inp, p, dt)
    loss = 0.0
    for k, tk in OUT_KEYS.items():
        o = out[tk]
        yy = y[k]
        if tk in ("rho", "temp"):
            yy = yy[0]
        loss = loss + (o * yy).sum()
    loss = loss + (out["log_ns"] * y["log_ns"]).sum() + (out["ndensity"] * y["ndensity"][0]).sum()
    names = ["nd", "ion", "rho", "temp", "vel", "ww"]
    wrt = [st[n] for n in names] + [eddy] + ([hs] if hs is not None else [])
    g = torch.autograd.grad(loss, wrt, allow_unused=True)
    res = {}
    for (k, tk), gg in zip(OUT_KEYS.items(), g[:6]):
        gg = torch.zeros_like(st[tk]) if gg is None else gg
        res[k] = gg[None] if tk in ("rho", "temp") else gg
    res["eddy"] = torch.zeros_like(eddy)[None] if g[6] is None else g[6][None]
    if hs is not None:
        res["heating_scale"] = g[7]
    return res


def _gpu_vjp(m, p, dt, y):
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(p)
    run = AD.StepRunner(ctx, m, dt)
    st = run.state()
    xbar, eb, hb = run.vjp(st, dict(y), run.tensors["eddy"], run.tensors.get("heating_scale"))
    status = run.plan.status()
    res = dict(xbar)
    res["eddy"] = eb
    if hb is not None:
        res["heating_scale"] = hb
    run.close()
    ctx.close()
    return res, status


VARIANTS = {
    "default": (dict(), dict()),
    "no_friction": (dict(use_neutral_friction=0), dict()),
    "log_ions": (dict(use_improved_ion_advection=0), dict()),
    "msis_damping_no_coriolis": (dict(use_msis_bcs=1, use_damping=1, use_coriolis=0), dict(with_lbc=True)),
    "heating": (dict(), dict(with_heating=True)),
}


def _rel(a, b):
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-300))


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_adjoint_matches_autograd(cuda, variant):
    over, mk = VARIANTS[variant]
    p = abi.default_params(**over)
    m = synthetic.make_member(24, 50, seed=71, **mk)
    gen = torch.Generator().manual_seed(5)
    y = _ybar(m, gen, cuda)
    want = _torch_vjp(m, p, 2.0, y, cuda)
    got, status = _gpu_vjp(m, p, 2.0, y)
    assert status == (0, 0)
    for k, w in want.items():
        g = got[k]
        if k == "idensity_s":  # the electron slot is not an input
            assert float(g[9].abs().max()) == 0.0
            g, w = g[:9], w[:9]
        assert _rel(g, w) < 1e-9, (k, _rel(g, w))


@pytest.mark.parametrize("n_alts", [8, 30, 75, 128])
def test_adjoint_other_altitude_counts(cuda, n_alts):
    """The adjoint kernel built for any nAlts: several columns per CTA
    (8, 30), one (75, 128), warp boundaries inside a column at different
    cells, against autograd through the transcription."""
    p = abi.default_params()
    m = synthetic.make_member(12, n_alts, seed=80 + n_alts, with_heating=True)
    gen = torch.Generator().manual_seed(6)
    y = _ybar(m, gen, cuda)
    want = _torch_vjp(m, p, 2.0, y, cuda)
    got, status = _gpu_vjp(m, p, 2.0, y)
    assert status == (0, 0)
    for k, w in want.items():
        g = got[k]
        if k == "idensity_s":
            g, w = g[:9], w[:9]
        assert _rel(g, w) < 1e-9, (n_alts, k, _rel(g, w))


@pytest.mark.parametrize("case", range(6))
def test_adjoint_random_parameter_combinations(cuda, case):
    """Seeded draws over the switches the adjoint differentiates through
    (friction, ion advection and its form, the MSIS lower boundary, damping,
    Coriolis, the nighttime ion boundary, the limiter's beta, the heating
    line) and over nAlts, against autograd through the transcription."""
    rng = np.random.default_rng(3000 + case)
    flags = {k: int(rng.integers(0, 2)) for k in ("use_neutral_friction", "use_ion_advection",
                                                   "use_improved_ion_advection", "use_msis_bcs",
                                                   "use_damping", "use_coriolis", "use_nighttime_ion_bcs")}
    p = abi.default_params(beta_limiter=float(rng.choice([1.0, 2.0])), **flags)
    n_alts = int(rng.choice([20, 50]))
    m = synthetic.make_member(16, n_alts, seed=4000 + case, with_lbc=bool(flags["use_msis_bcs"]),
                              with_heating=bool(rng.integers(0, 2)))
    gen = torch.Generator().manual_seed(9 + case)
    y = _ybar(m, gen, cuda)
    want = _torch_vjp(m, p, 2.0, y, cuda)
    got, status = _gpu_vjp(m, p, 2.0, y)
    assert status == (0, 0)
    for k, w in want.items():
        g = got[k]
        if k == "idensity_s":
            g, w = g[:9], w[:9]
        assert _rel(g, w) < 1e-9, (flags, k, _rel(g, w))


def test_adjoint_is_reproducible(cuda):
    """Every sum of the adjoint kernel has a fixed order (no atomics of
    floating-point values): two runs give the same bits."""
    p = abi.default_params()
    m = synthetic.make_member(40, 50, seed=79, with_heating=True)
    gen = torch.Generator().manual_seed(8)
    y = _ybar(m, gen, cuda)
    a, _ = _gpu_vjp(m, p, 2.0, y)
    b, _ = _gpu_vjp(m, p, 2.0, y)
    for k in a:
        assert torch.equal(a[k], b[k]), k


@pytest.mark.parametrize("every", [2, 0])
def test_rollout_equals_stepwise_composition(cuda, every):
    """Checkpoints every 2 steps, and every step's stages kept (every = 0)."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(32, 50, seed=72, with_heating=True)
    ctx = V.VerticalContext(p)
    run = AD.StepRunner(ctx, m, 2.0)
    s0 = {k: v.clone().requires_grad_(True) for k, v in run.state().items()}
    eddy = run.tensors["eddy"].clone().requires_grad_(True)
    hs = run.tensors["heating_scale"].clone().requires_grad_(True)
    w = torch.rand(32, dtype=torch.float64, device=cuda, generator=torch.Generator(cuda).manual_seed(1))
    lvl = AD.level_of(m.altitude, 400e3)
    out = AD.rollout(run, s0, 6, every, eddy, hs)
    g1 = torch.autograd.grad(AD.o_n2_objective(out["ndensity_s"], w, lvl), [s0["ndensity_s"], s0["temperature"],
                                                                                 s0["velocity"], eddy, hs])
    s = s0
    for _ in range(6):
        s = AD.vertical_step(run, s, eddy, hs)
    g2 = torch.autograd.grad(AD.o_n2_objective(s["ndensity_s"], w, lvl), [s0["ndensity_s"], s0["temperature"],
                                                                               s0["velocity"], eddy, hs])
    for a, b in zip(g1, g2):
        assert _rel(a, b) < 1e-12
    run.close()


def test_kept_stages_refused_when_they_do_not_fit(cuda):
    """every = 0 with more steps than device memory holds stage states for
    raises before the first step."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    m = synthetic.make_member(32, 50, seed=73)
    ctx = V.VerticalContext(abi.default_params())
    run = AD.StepRunner(ctx, m, 2.0, autotune=False)
    free = torch.cuda.mem_get_info(cuda)[0]
    n = int(free // run.stage_bytes_per_step()) + 1
    with pytest.raises(V.GitmError, match="every > 0"):
        AD.rollout(run, run.state(), n, 0)
    run.close()
    ctx.close()


def test_rollout_matches_transcription_autograd(cuda):
    """A 20-step rollout: the adjoint's gradient against torch autograd
    through 20 steps of the transcription (the exact linearisation of the
    same branch path)."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    p = abi.default_params()
    n_cols, n_steps = 4, 20
    m = synthetic.make_member(n_cols, 50, seed=74, with_heating=True)
    lvl = AD.level_of(m.altitude, 400e3)
    w = torch.rand(n_cols, dtype=torch.float64, generator=torch.Generator().manual_seed(2)).to(cuda)
    ctx = V.VerticalContext(p)
    run = AD.StepRunner(ctx, m, 2.0)
    s0 = {k: v.clone().requires_grad_(True) for k, v in run.state().items()}
    eddy = run.tensors["eddy"].clone().requires_grad_(True)
    hs = run.tensors["heating_scale"].clone().requires_grad_(True)
    out = AD.rollout(run, s0, n_steps, 5, eddy, hs)
    names = ("ndensity_s", "temperature", "velocity", "vert_vel", "rho")
    got = torch.autograd.grad(AD.o_n2_objective(out["ndensity_s"], w, lvl), [s0[k] for k in names] + [eddy, hs])
    run.close()
    st, inp = TS.from_member(m, device=cuda, requires_grad=True)
    ed = inp["eddy"].clone().requires_grad_(True)
    h = inp["heating_scale"].clone().requires_grad_(True)
    inp["eddy"], inp["heating_scale"] = ed, h
    s = st
    for _ in range(n_steps):
        o = TS.step(s, inp, p, 2.0)
        s = {k: o[k] for k in ("nd", "ion", "rho", "temp", "vel", "ww")}
    J = (w * (torch.log(s["nd"][0, lvl]) - torch.log(s["nd"][2, lvl]))).sum()
    tn = ("nd", "temp", "vel", "ww", "rho")
    want = torch.autograd.grad(J, [st[k] for k in tn] + [ed, h])
    for k, g, wt in zip(names + ("eddy", "heating_scale"), got, want):
        g = g.reshape(wt.shape) if g.numel() == wt.numel() else g
        assert _rel(g, wt) < 1e-8, (k, _rel(g, wt))


def test_rollout_gradient_matches_finite_differences(cuda):
    """Two steps; directions on one column each; eps = 5e-8 relative.  The
    limiter makes the step piecewise smooth with kinks dense enough that a
    perturbation of this size often crosses one, so only directions whose
    +-eps runs take every branch the base run takes (branch signatures of
    the transcription) are compared; they must agree to 1e-6 above the
    difference's rounding floor (a few ulps of the column's J)."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    p = abi.default_params()
    n_cols, n_steps = 8, 2
    m = synthetic.make_member(n_cols, 50, seed=73, with_heating=True)
    ctx = V.VerticalContext(p)
    run = AD.StepRunner(ctx, m, 2.0)
    base = run.state()
    eddy0 = run.tensors["eddy"].clone()
    hs0 = run.tensors["heating_scale"].clone()
    lvl = AD.level_of(m.altitude, 400e3)
    gen = torch.Generator().manual_seed(3)
    w = torch.rand(n_cols, dtype=torch.float64, generator=gen).to(cuda)
    s0 = {k: v.clone().requires_grad_(True) for k, v in base.items()}
    eddy = eddy0.clone().requires_grad_(True)
    hs = hs0.clone().requires_grad_(True)
    out = AD.rollout(run, s0, n_steps, 1, eddy, hs)
    names = ("ndensity_s", "temperature", "velocity", "vert_vel", "rho")
    grads = torch.autograd.grad(AD.o_n2_objective(out["ndensity_s"], w, lvl),
                                [s0[k] for k in names] + [eddy, hs])
    tst, tinp = TS.from_member(m)

    def ts_roll(state, ed, h):
        i2 = dict(tinp)
        i2["eddy"], i2["heating_scale"] = ed, h
        s = state
        for _ in range(n_steps):
            o = TS.step(s, i2, p, 2.0)
            s = {k: o[k] for k in ("nd", "ion", "rho", "temp", "vel", "ww")}
        return s

    def per_column_J(state, ed, h):
        s = {k: v.clone() for k, v in state.items()}
        for _ in range(n_steps):
            s = run.step(s, ed, h)
        nd = s["ndensity_s"]
        return w * (torch.log(nd[0, lvl]) - torch.log(nd[2, lvl]))

    eps = 5e-8
    sig0 = TS.branch_signature(ts_roll, tst, tinp["eddy"], tinp["heating_scale"])
    checked, errs = 0, []
    for trial in range(32):
        col = trial % n_cols
        dirs = {}
        for k in names:
            d = torch.zeros_like(base[k])
            d[..., col] = torch.randn(d[..., col].shape, generator=gen, dtype=torch.float64).to(cuda)
            dirs[k] = d
        de = torch.zeros_like(eddy0)
        de[..., col] = torch.randn(de[..., col].shape, generator=gen, dtype=torch.float64).to(cuda)
        dh = torch.zeros_like(hs0)
        dh[col] = 1.0
        steps = {k: base[k].abs() * eps for k in names}
        se, sh = eddy0.abs() * eps, hs0.abs() * eps

        def point(sign):
            st = {k: base[k] + sign * dirs[k] * steps[k] if k in dirs else base[k] for k in base}
            return st, eddy0 + sign * de * se, hs0 + sign * dh * sh

        def ts_point(sign):
            st, ed, h = point(sign)
            s2 = {"nd": st["ndensity_s"].cpu(), "ion": tst["ion"], "rho": st["rho"][0].cpu(),
                  "temp": st["temperature"][0].cpu(), "vel": st["velocity"].cpu(), "ww": st["vert_vel"].cpu()}
            return s2, ed[0].cpu(), h.cpu()
        if not all(TS.same_branches(sig0, TS.branch_signature(ts_roll, *ts_point(sg))) for sg in (1.0, -1.0)):
            continue
        jp = per_column_J(*point(1.0))[col]
        jm = per_column_J(*point(-1.0))[col]
        fd = float(jp - jm) / 2.0
        ana = sum(float((g * dirs[k] * steps[k]).sum()) for g, k in zip(grads[:5], names))
        ana += float((grads[5] * de * se).sum()) + float((grads[6] * dh * sh).sum())
        floor = 8 * 2.2e-16 * abs(float(jp))
        errs.append(max(abs(fd - ana) - floor, 0.0) / max(abs(fd), abs(ana), 1e-300))
        checked += 1
    assert checked >= 4, checked
    assert max(errs) < 1e-6, errs
    run.close()


def test_saved_states_match_recompute(cuda):
    """The saving step gives the plain step's outputs, and the adjoint that
    reads its saved stage states equals the one that recomputes them."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(40, 50, seed=75, with_heating=True)
    ctx = V.VerticalContext(p)
    run = AD.StepRunner(ctx, m, 2.0)
    s0 = run.state()
    plain = run.step(s0)
    buf = run.saved_buffer()
    saving = run.step_saving(s0, buf)
    for k in plain:
        assert _rel(saving[k], plain[k]) < 1e-13, k
    gen = torch.Generator().manual_seed(8)
    y = _ybar(m, gen, cuda)
    a = run.vjp(s0, dict(y), run.tensors["eddy"], run.tensors["heating_scale"])
    b = run.vjp(s0, dict(y), run.tensors["eddy"], run.tensors["heating_scale"], saved=buf)
    for k in a[0]:
        assert _rel(b[0][k], a[0][k]) < 1e-12, k
    assert _rel(b[1], a[1]) < 1e-12 and _rel(b[2], a[2]) < 1e-12
    run.close()
