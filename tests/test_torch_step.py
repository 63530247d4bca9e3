"""The FP64 PyTorch transcription (tests/torch_step.py) against the oracle,
and its autograd gradient against central finite differences (CPU)."""
import numpy as np
import pytest
import torch

from gitm_b200 import abi, synthetic
from tests import torch_step as TS

VARIANTS = {
    "default": (dict(), dict()),
    "no_friction": (dict(use_neutral_friction=0), dict()),
    "log_ions": (dict(use_improved_ion_advection=0), dict()),
    "msis_damping_no_coriolis": (dict(use_msis_bcs=1, use_damping=1, use_coriolis=0), dict(with_lbc=True)),
    "heating": (dict(), dict(with_heating=True)),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_transcription_matches_oracle(oracle_lib, variant):
    over, mk = VARIANTS[variant]
    p = abi.default_params(**over)
    m = synthetic.make_member(12, 50, seed=5, **mk)
    r = m.copy()
    oracle_lib.advance(r, p, 2.0, 1)
    st, inp = TS.from_member(m)
    got = TS.to_member_arrays(TS.step(st, inp, p, 2.0))
    ref = dict(r.arrays())
    for k, a in got.items():
        b = ref[k]
        den = np.abs(b).max(axis=tuple(range(a.ndim - 1)), keepdims=True)
        assert (np.abs(a - b) / den).max() < 1e-11, k


def _objective(out, w):
    # weighted log(n_O / n_N2) at one cell: the form of the rollout objective
    return (w * (torch.log(out["nd"][0, 14]) - torch.log(out["nd"][2, 14]))).sum()


def test_transcription_gradient_matches_finite_differences():
    """Two steps, J of the rollout form; directions whose +-eps runs take a
    different branch anywhere (a limiter kink, a clamp, a boundary switch)
    are skipped.  FD noise floor: a few ulps of J over the perturbation."""
    p = abi.default_params()
    m = synthetic.make_member(4, 20, seed=6, with_heating=True)
    st, inp = TS.from_member(m, requires_grad=True)
    hs = inp["heating_scale"].clone().requires_grad_(True)
    names = ("nd", "temp", "vel", "ww", "rho")
    w = torch.rand(4, dtype=torch.float64, generator=torch.Generator().manual_seed(0))

    def J(state, scale):
        i2 = dict(inp)
        i2["heating_scale"] = scale
        out = TS.step(state, i2, p, 2.0)
        out = TS.step({k: out[k] for k in ("nd", "ion", "rho", "temp", "vel", "ww")}, i2, p, 2.0)
        return _objective(out, w)

    j = J(st, hs)
    grads = torch.autograd.grad(j, [st[n] for n in names] + [hs])
    base = [st[n].detach() for n in names] + [hs.detach()]
    rng = np.random.default_rng(1)
    checked = 0
    for trial in range(12):
        dirs = [torch.from_numpy(rng.normal(size=t.shape)) for t in base]
        eps = 1e-7
        steps = [b.abs() * eps for b in base]

        def point(sign):
            vals = [b + sign * d * s for b, d, s in zip(base, dirs, steps)]
            s2 = {k: v.detach() for k, v in st.items()}
            for n, v in zip(names, vals):
                s2[n] = v
            return s2, vals[-1]
        sp, sm = point(1.0), point(-1.0)
        sig0 = TS.branch_signature(J, {k: v.detach() for k, v in st.items()}, hs.detach())
        if not (TS.same_branches(sig0, TS.branch_signature(J, *sp)) and
                TS.same_branches(sig0, TS.branch_signature(J, *sm))):
            continue
        with torch.no_grad():
            fd = (float(J(*sp)) - float(J(*sm))) / 2.0
        ana = sum(float((g * d * s).sum()) for g, d, s in zip(grads, dirs, steps))
        noise = 1e-14 * abs(float(j))
        assert abs(fd - ana) <= 1e-6 * max(abs(fd), abs(ana)) + noise, (trial, fd, ana)
        checked += 1
    assert checked >= 4


def test_rollout_finite_differences_track_branch_flips():
    """A six-step rollout of the objective's form, central differences for
    eps from 1e-6 to 1e-9 (relative) in random directions.  The MC limiter
    makes the step piecewise smooth: a perturbation can flip a limiter case
    (or a clamp, a boundary switch) somewhere in the rollout, and then the
    difference quotient mixes two pieces.  Checked: wherever the +-eps runs
    take exactly the base run's branches (the transcription's recorder), the
    difference agrees with the autograd gradient to 1e-6 (beyond a rounding
    floor of the difference of two J); every disagreement beyond 1e-6 comes
    with flipped branches; some directions flip branches at the larger eps."""
    p = abi.default_params()
    m = synthetic.make_member(4, 20, seed=7, with_heating=True)
    st, inp = TS.from_member(m, requires_grad=True)
    names = ("nd", "temp", "vel", "ww", "rho")
    w = torch.rand(4, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    n_steps = 6

    def J(state):
        s = state
        for _ in range(n_steps):
            out = TS.step(s, inp, p, 2.0)
            s = {k: out[k] for k in ("nd", "ion", "rho", "temp", "vel", "ww")}
        return _objective(out, w)

    def J_and_branches(state):
        box = {}

        def run():
            box["j"] = float(J(state))
        sig = TS.branch_signature(run)
        return box["j"], sig

    j = J(st)
    grads = torch.autograd.grad(j, [st[n] for n in names])
    base = {k: v.detach() for k, v in st.items()}
    j0, sig0 = J_and_branches(base)
    rng = np.random.default_rng(2)
    dirs = [[torch.from_numpy(rng.normal(size=base[n].shape)) for n in names] for _ in range(6)]
    checked = flipped = 0
    for eps in (1e-6, 1e-7, 1e-8, 1e-9):
        for d in dirs:
            steps = [base[n].abs() * eps for n in names]

            def point(sign):
                s2 = dict(base)
                for n, dd, ss in zip(names, d, steps):
                    s2[n] = base[n] + sign * dd * ss
                return s2
            jp, sp = J_and_branches(point(1.0))
            jm, sm = J_and_branches(point(-1.0))
            fd = (jp - jm) / 2.0
            ana = sum(float((g * dd * ss).sum()) for g, dd, ss in zip(grads, d, steps))
            err = abs(fd - ana)
            tol = 1e-6 * max(abs(fd), abs(ana)) + 3e-14 * abs(j0)
            same = TS.same_branches(sig0, sp) and TS.same_branches(sig0, sm)
            if same:
                assert err <= tol, (eps, fd, ana)
                checked += 1
            else:
                flipped += 1
            # a disagreement beyond the tolerance only with flipped branches
            assert err <= tol or not same, (eps, fd, ana)
    assert checked >= 6
    assert flipped >= 1
