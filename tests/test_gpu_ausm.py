"""The AUSM solver (UseAUSMSolver, vertical_solver_ausm.f90) on the GPU vs
the CPU oracle, through libgitmvert.so.

Same tolerance as the Rusanov parity tests (tests/parity.py); multi-step
runs compound the FP64 rounding differences and use 1e-9.
"""
import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import assert_state_close
from tests.test_gpu_parity import STATE, gpu_advance, ref_advance

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def ausm(**over):
    return abi.default_params(solver=abi.SOLVER_AUSM, **over)


VARIANTS = {
    "default": dict(),
    "no_friction": dict(use_neutral_friction=0),
    "log_ions": dict(use_improved_ion_advection=0),
    "damping_no_coriolis": dict(use_damping=1, use_coriolis=0),
    "given_coefficients": dict(compute_coefficients=0),
    "beta1": dict(beta_limiter=1.0),
}


# 384 threads: the shape with Orig in global scratch, built for nAlts = 50
@pytest.mark.parametrize("threads", [128, 256, 384])
@pytest.mark.parametrize("variant", list(VARIANTS))
def test_ausm_step_matches_oracle(torch_cuda, oracle_lib, variant, threads):
    p = ausm(**VARIANTS[variant])
    m = synthetic.make_member(96, 50, seed=41)
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0, config=dict(threads=threads))
    assert_state_close(out, ref, STATE)
    np.testing.assert_array_equal(st, st_ref)


def test_ausm_msis_lower_boundary(torch_cuda, oracle_lib):
    p = ausm(use_msis_bcs=1)
    m = synthetic.make_member(64, 50, seed=42, with_lbc=True)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    out, _ = gpu_advance(m, p, 2.0)
    assert_state_close(out, ref, STATE)


@pytest.mark.parametrize("n_alts", [8, 20, 100, 128])
def test_ausm_other_altitude_counts(torch_cuda, oracle_lib, n_alts):
    p = ausm()
    m = synthetic.make_member(30, n_alts, seed=43 + n_alts)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    out, _ = gpu_advance(m, p, 2.0)
    assert_state_close(out, ref, STATE)


@pytest.mark.parametrize("threads", [256, 384])
def test_ausm_multistep_resident(torch_cuda, oracle_lib, threads):
    p = ausm()
    m = synthetic.make_member(48, 50, seed=44)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0, n_steps=5)
    out, _ = gpu_advance(m, p, 2.0, n_steps=5, config=dict(threads=threads, steps_per_launch=5))
    assert_state_close(out, ref, STATE, rtol=1e-9)
    out1, _ = gpu_advance(m, p, 2.0, n_steps=5, config=dict(threads=threads, steps_per_launch=1))
    assert_state_close(out, out1, STATE, rtol=1e-12)


def test_ausm_ragged_batch(torch_cuda, oracle_lib):
    from gitm_b200 import vertical as V
    p = ausm()
    ms = [synthetic.make_member(n, na, seed=45 + i) for i, (n, na) in enumerate([(17, 50), (9, 75), (5, 30)])]
    refs = [ref_advance(oracle_lib, m, p, 2.0)[0] for m in ms]
    ctx = V.VerticalContext(p)
    dms = [V.device_member(m) for m in ms]
    plan = V.Plan(ctx, dms)
    plan.advance(2.0, 1)
    plan.check()
    for dm, ref in zip(dms, refs):
        assert_state_close(dm.to_numpy(), ref, STATE)


def test_ausm_modvertical_form(torch_cuda, oracle_lib):
    import torch
    from gitm_b200 import vertical as V
    p = ausm()
    m = synthetic.make_member(32, 50, seed=48)
    d = synthetic.to_modvertical(m, p)
    ref = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    oracle_lib.advance_1d(ref, p, 2.0)
    td = {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    ctx = V.VerticalContext(p)
    V.advance_vertical_1d(ctx, td, 2.0)
    keys = ("log_rho", "temp", "vel_gd", "log_ns", "vert_vel")
    got = {k: td[k].cpu().numpy() for k in keys}
    got["log_ins"] = td["log_ins"].cpu().numpy()[:9]
    want = {k: ref[k] for k in keys}
    want["log_ins"] = ref["log_ins"][:9]
    assert_state_close(got, want, list(got))


def test_ausm_host_pointer_path(torch_cuda):
    from gitm_b200 import vertical as V
    p = ausm()
    m = synthetic.make_member(700, 50, seed=49)
    # the launch shape of the host-pointer form (each shape is compiled on its own)
    dev_out, _ = gpu_advance(m, p, 2.0, config=dict(threads=128, steps_per_launch=1))
    h = m.copy()
    ctx = V.VerticalContext(p)
    V.advance_vertical_all_host(ctx, [h], 2.0)
    for k in STATE:
        np.testing.assert_array_equal(getattr(h, k), dev_out[k], err_msg=k)


def test_plan_keeps_its_solver(torch_cuda):
    """A plan made under one solver refuses to run after the context switches."""
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(abi.default_params())
    dm = V.device_member(synthetic.make_member(8, 50, seed=50))
    plan = V.Plan(ctx, [dm])
    ctx.set_params(ausm())
    with pytest.raises(V.GitmError):
        plan.advance(2.0, 1)
    np.testing.assert_array_equal(dm.tensors["rho"].cpu().numpy(), synthetic.make_member(8, 50, seed=50).rho)


def test_ausm_autotune(torch_cuda):
    from gitm_b200 import vertical as V
    m = synthetic.make_member(600, 50, seed=51)
    ctx = V.VerticalContext(ausm())
    dm = V.device_member(m)
    plan = V.Plan(ctx, [dm])
    cfg = plan.autotune(2.0, 2)
    assert cfg.threads in (128, 256, 384)
    np.testing.assert_array_equal(dm.tensors["ndensity_s"].cpu().numpy(), m.ndensity_s)


def test_unbuilt_shape_is_refused_and_plan_keeps_working(torch_cuda, oracle_lib):
    """The AUSM 384-thread shape is compiled for nAlts = 50 only: a plan of
    another nAlts refuses it with an error, keeps its launch shape and still
    steps like the oracle."""
    from gitm_b200 import vertical as V
    p = ausm()
    m = synthetic.make_member(40, 30, seed=52)
    ctx = V.VerticalContext(p)
    dm = V.device_member(m)
    plan = V.Plan(ctx, [dm])
    before = plan.config
    with pytest.raises(V.GitmError, match="not built"):
        plan.set_config(threads=384)
    after = plan.config
    assert (after.threads, after.steps_per_launch) == (before.threads, before.steps_per_launch)
    np.testing.assert_array_equal(dm.tensors["ndensity_s"].cpu().numpy(), m.ndensity_s)
    plan.advance(2.0, 1)
    plan.check()
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    assert_state_close(dm.to_numpy(), ref, STATE)
    plan.close()
    ctx.close()


def test_ausm_autotune_ragged(torch_cuda, oracle_lib):
    """The autotuner over members of nAlts 50, 75 and 30 picks one of the
    shapes built for such a plan, leaves the state as it was, and the chosen
    shape steps like the oracle over two steps."""
    from gitm_b200 import vertical as V
    p = ausm()
    ms = [synthetic.make_member(n, na, seed=53 + i) for i, (n, na) in enumerate([(200, 50), (90, 75), (150, 30)])]
    ctx = V.VerticalContext(p)
    dms = [V.device_member(m) for m in ms]
    plan = V.Plan(ctx, dms)
    cfg = plan.autotune(2.0, 2)
    assert cfg.threads in (128, 256)
    for dm, m in zip(dms, ms):
        np.testing.assert_array_equal(dm.tensors["ndensity_s"].cpu().numpy(), m.ndensity_s)
    plan.advance(2.0, 2)
    plan.check()
    for dm, m in zip(dms, ms):
        ref, _ = ref_advance(oracle_lib, m, p, 2.0, n_steps=2)
        assert_state_close(dm.to_numpy(), ref, STATE, rtol=1e-9)
    plan.close()
    ctx.close()
