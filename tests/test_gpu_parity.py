"""CUDA path vs the CPU oracle on identical seeded inputs (run on a B200).

Every call goes through libgitmvert.so (the C ABI); see tests/parity.py for
the tolerance.
"""
import glob
import os

import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import RTOL, assert_state_close

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
STATE = synthetic.Member.STATE + ("log_ns", "ndensity")


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def gpu_advance(m, params, dt, n_steps=1, config=None):
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(params)
    dm = V.device_member(m)
    plan = V.Plan(ctx, [dm])
    if config:
        plan.set_config(**config)
    plan.advance(dt, n_steps)
    words = plan.status_words()
    out = dm.to_numpy()
    plan.close()
    ctx.close()
    return out, words


def ref_advance(oracle_lib, m, params, dt, n_steps=1):
    r = m.copy()
    st = oracle_lib.advance(r, params, dt, n_steps)
    return {k: v for k, v in r.arrays()}, st


VARIANTS = {
    "default": dict(),
    "no_friction": dict(use_neutral_friction=0),
    "no_coriolis_damping": dict(use_coriolis=0, use_damping=1),
    "log_ions": dict(use_improved_ion_advection=0),
    "no_ion_advection": dict(use_ion_advection=0),
    "beta1": dict(beta_limiter=1.0),
    "given_coefficients": dict(compute_coefficients=0),
    "no_nighttime_bcs": dict(use_nighttime_ion_bcs=0),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_step_matches_oracle(torch_cuda, oracle_lib, variant):
    p = abi.default_params(**VARIANTS[variant])
    m = synthetic.make_member(96, 50, seed=21)
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0)
    assert_state_close(out, ref, STATE)
    np.testing.assert_array_equal(st, st_ref)


@pytest.mark.parametrize("case", range(12))
def test_random_parameter_combinations(torch_cuda, oracle_lib, case):
    """Seeded draws over the switches of the path taken together (solver,
    friction, ion advection and its form, the MSIS lower boundary, damping,
    Coriolis, the nighttime ion boundary, producers on the device or given,
    the limiter's beta, thermal diffusion, a low wind clamp, the heating
    line) and over nAlts, two steps, against the oracle."""
    rng = np.random.default_rng(1000 + case)
    flags = {k: int(rng.integers(0, 2)) for k in ("use_neutral_friction", "use_ion_advection",
                                                   "use_improved_ion_advection", "use_msis_bcs",
                                                   "use_damping", "use_coriolis", "use_nighttime_ion_bcs",
                                                   "compute_coefficients")}
    solver = abi.SOLVER_AUSM if rng.random() < 0.35 else abi.SOLVER_RUSANOV
    over = dict(flags, solver=solver, beta_limiter=float(rng.choice([1.0, 1.5, 2.0])),
                max_vertical_velocity=float(rng.choice([1000.0, 5.0])))
    if rng.random() < 0.5:
        over["thermal_diff_coef"] = [0.0, 0.0, 0.0, 0.0, -0.2, -0.38]
    p = abi.default_params(**over)
    n_alts = int(rng.choice([20, 50, 64]))
    m = synthetic.make_member(40, n_alts, seed=2000 + case, with_lbc=bool(flags["use_msis_bcs"]),
                              with_heating=bool(rng.integers(0, 2)))
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0, n_steps=2)
    out, st = gpu_advance(m, p, 2.0, n_steps=2, config=dict(steps_per_launch=1))
    assert_state_close(out, ref, STATE)
    np.testing.assert_array_equal(st, st_ref)


@pytest.mark.parametrize("n_steps", [1, 4])
def test_heating_update(torch_cuda, oracle_lib, n_steps):
    """The add_sources temperature line after each step, resident steps included."""
    p = abi.default_params()
    m = synthetic.make_member(64, 50, seed=34, with_heating=True)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0, n_steps=n_steps)
    out, _ = gpu_advance(m, p, 2.0, n_steps=n_steps, config=dict(steps_per_launch=n_steps))
    assert_state_close(out, ref, STATE, rtol=1e-10 if n_steps == 1 else 1e-9)


@pytest.mark.parametrize("solver", [abi.SOLVER_RUSANOV, abi.SOLVER_AUSM])
@pytest.mark.parametrize("n_steps,spl", [(1, 1), (4, 4), (4, 1)])
def test_eddy_producer(torch_cuda, oracle_lib, solver, n_steps, spl):
    """compute_eddy: KappaEddyDiffusion(1:nAlts) recomputed after every step
    from the pressure the step started from (calc_sources), read by the next
    step, resident steps included; with the heating line on."""
    p = abi.default_params(compute_eddy=1, solver=solver)
    m = synthetic.make_member(64, 50, seed=35, with_heating=True)
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0, n_steps=n_steps)
    out, st = gpu_advance(m, p, 2.0, n_steps=n_steps, config=dict(steps_per_launch=spl))
    assert_state_close(out, ref, STATE + ("eddy",), rtol=1e-10 if n_steps == 1 else 1e-9)
    np.testing.assert_array_equal(st, st_ref)
    # the produced profile is not the one passed in
    assert np.abs(out["eddy"] - m.eddy).max() > 0.0


def test_eddy_producer_host_path(torch_cuda, oracle_lib):
    """The host-pointer form copies the produced coefficient back."""
    from gitm_b200 import vertical as V
    p = abi.default_params(compute_eddy=1)
    m = synthetic.make_member(700, 50, seed=36)
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0, n_steps=2)
    h = m.copy()
    ctx = V.VerticalContext(p)
    V.advance_vertical_all_host(ctx, [h], 2.0, n_steps=2)
    ctx.close()
    assert (st_ref == 0).all()
    assert_state_close(dict(h.arrays()), ref, synthetic.Member.STATE + ("eddy",), rtol=1e-9)


def test_eddy_producer_refused_by_adjoint(torch_cuda):
    """The adjoint differentiates a step with the eddy coefficient as an input."""
    from gitm_b200 import adjoint as AD
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(abi.default_params(compute_eddy=1))
    run = AD.StepRunner(ctx, synthetic.make_member(8, 50, seed=37), 2.0, autotune=False)
    st = run.state()
    with pytest.raises(V.GitmError):
        run.vjp(st, {})
    run.close()
    ctx.close()


def test_msis_lower_boundary(torch_cuda, oracle_lib):
    p = abi.default_params(use_msis_bcs=1)
    m = synthetic.make_member(64, 50, seed=22, with_lbc=True)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    out, _ = gpu_advance(m, p, 2.0)
    assert_state_close(out, ref, STATE)


@pytest.mark.parametrize("n_alts", [8, 20, 75, 100, 128])
def test_other_altitude_counts(torch_cuda, oracle_lib, n_alts):
    p = abi.default_params()
    m = synthetic.make_member(40, n_alts, seed=23 + n_alts)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    out, _ = gpu_advance(m, p, 2.0)
    assert_state_close(out, ref, STATE)


@pytest.mark.parametrize("threads", [256, 320, 384, 512])
def test_launch_shapes_agree(torch_cuda, oracle_lib, threads):
    p = abi.default_params()
    m = synthetic.make_member(50, 50, seed=24)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0)
    out, _ = gpu_advance(m, p, 2.0, config=dict(threads=threads, ctas_per_sm=1))
    assert_state_close(out, ref, STATE)


def test_multistep_resident_matches_stepwise(torch_cuda, oracle_lib):
    """steps_per_launch > 1 keeps columns in shared memory across steps."""
    p = abi.default_params()
    m = synthetic.make_member(64, 50, seed=25)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0, n_steps=6)
    out, _ = gpu_advance(m, p, 2.0, n_steps=6, config=dict(steps_per_launch=6))
    assert_state_close(out, ref, STATE, rtol=1e-9)
    out1, _ = gpu_advance(m, p, 2.0, n_steps=6, config=dict(steps_per_launch=1))
    assert_state_close(out, out1, STATE, rtol=1e-12)


GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_golden_fixtures(torch_cuda, path):
    from tests.test_oracle import load_golden
    p, m, out_ref, n_steps, dt, status = load_golden(path)
    out, st = gpu_advance(m, p, dt, n_steps)
    assert_state_close(out, out_ref, STATE, rtol=RTOL * 10 if n_steps > 1 else RTOL)
    np.testing.assert_array_equal(st, status)


def test_ragged_batch(torch_cuda, oracle_lib):
    """Members of different nAlts and sizes advance in one launch."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    ms = [synthetic.make_member(n, na, seed=30 + i) for i, (n, na) in
          enumerate([(37, 50), (20, 75), (13, 100), (5, 30)])]
    refs = [ref_advance(oracle_lib, m, p, 2.0)[0] for m in ms]
    ctx = V.VerticalContext(p)
    dms = [V.device_member(m) for m in ms]
    plan = V.Plan(ctx, dms)
    plan.advance(2.0, 1)
    plan.check()
    for dm, ref in zip(dms, refs):
        assert_state_close(dm.to_numpy(), ref, STATE)


@pytest.mark.parametrize("case", range(6))
def test_random_ragged_plans(torch_cuda, oracle_lib, case):
    """Seeded ragged plans (3 to 5 members of nAlts 8 to 100 and 3 to 40
    columns) under a random launch configuration of the plan API (a built
    thread count, columns per CTA, steps per launch, CTAs per SM), three
    steps, every member against the oracle."""
    from gitm_b200 import vertical as V
    rng = np.random.default_rng(5000 + case)
    solver = abi.SOLVER_AUSM if case % 3 == 2 else abi.SOLVER_RUSANOV
    p = abi.default_params(solver=solver)
    n_m = int(rng.integers(3, 6))
    ms = [synthetic.make_member(int(rng.integers(3, 41)), int(rng.choice([8, 20, 50, 64, 100])),
                                seed=6000 + 10 * case + i, with_heating=bool(rng.integers(0, 2)))
          for i in range(n_m)]
    refs = [ref_advance(oracle_lib, m, p, 2.0, n_steps=3)[0] for m in ms]
    ctx = V.VerticalContext(p)
    dms = [V.device_member(m) for m in ms]
    plan = V.Plan(ctx, dms)
    threads = [128, 256] if solver == abi.SOLVER_AUSM else [128, 160, 192, 256, 320, 384, 512]
    cfg = dict(threads=int(rng.choice(threads)), cols_per_cta=int(rng.choice([0, 1, 2])),
               steps_per_launch=int(rng.choice([1, 2, 3])), ctas_per_sm=int(rng.choice([0, 1, 2])))
    plan.set_config(**cfg)
    plan.advance(2.0, 3)
    plan.check()
    for dm, ref in zip(dms, refs):
        assert_state_close(dm.to_numpy(), ref, STATE, rtol=1e-9)
    plan.close()
    ctx.close()


def test_neg_density_status(torch_cuda, oracle_lib):
    p = abi.default_params()
    m = synthetic.make_member(12, 50, seed=26)
    m.ndensity_s[4, 20, 7] = -1.0
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0)
    assert st[7] & abi.ST_NEG_DENSITY and st_ref[7] & abi.ST_NEG_DENSITY
    assert (st[np.arange(12) != 7] == 0).all()
    assert_state_close(out, ref, synthetic.Member.STATE)


def test_one_shot_raises_gitmstop(torch_cuda):
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(8, 50, seed=27)
    m.ndensity_s[0, 5, 3] = 0.0
    ctx = V.VerticalContext(p)
    with pytest.raises(V.GitmStop):
        V.advance_vertical_all(ctx, [V.device_member(m)], 2.0)


def test_host_pointer_path_matches_oracle(torch_cuda, oracle_lib):
    """gitm_vert_advance_native_host (host arrays, chunked copies overlapped
    with the steps) against the oracle, and bit for bit against the device
    form with the launch shape the host form uses (128 threads, one step per
    launch: each launch shape is compiled on its own and may round
    differently)."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(5000, 50, seed=28)
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    h = m.copy()
    ctx = V.VerticalContext(p)
    V.advance_vertical_all_host(ctx, [h], 2.0)
    ctx.close()
    assert (st_ref == 0).all()
    assert_state_close(dict(h.arrays()), ref, STATE)
    dev_out, _ = gpu_advance(m, p, 2.0, config=dict(threads=128, steps_per_launch=1))
    for k in STATE:
        np.testing.assert_array_equal(getattr(h, k), dev_out[k], err_msg=k)


def test_host_pointer_path_floors_passive_ions(torch_cuda, oracle_lib):
    """With UseImprovedIonAdvection the step floors every ion density of the
    interior cells at 1, the passive ions' too: the host form must bring
    those interior values back as well (against the oracle)."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(300, 50, seed=29)
    rng = np.random.default_rng(3)
    for q in range(abi.NIONS_ADVECT, abi.NIONS - 1):
        cols = rng.choice(m.n_cols, 20, replace=False)
        cells = rng.integers(4, 40, 20)  # interior cells away from the boundary rows
        m.idensity_s[q, cells + 1, cols] = 0.5
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    h = m.copy()
    ctx = V.VerticalContext(p)
    V.advance_vertical_all_host(ctx, [h], 2.0)
    ctx.close()
    assert (st_ref == 0).all()
    assert (ref["idensity_s"][abi.NIONS_ADVECT:abi.NIONS - 1, 2:51] >= 1.0).all()
    assert_state_close(dict(h.arrays()), ref, STATE)


def test_globe5deg_100_steps_each_against_the_oracle(torch_cuda, oracle_lib):
    """The 5 deg globe (36 x 72 = 2,592 columns, GITM's 4 x 8 blocks of 9 x 9),
    nAlts = 50, 100 RK4 steps of dt = 2 s through the plain per-call drop-in
    (gitm_vert_advance_native, one call per step).  After every step the GPU
    result is compared with one oracle step taken from the GPU's own previous
    state, at the per-step tolerance of 1e-10, so rounding differences do not
    accumulate across the comparison."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.globe_member(5.0, 5.0, n_alts=50, seed=1)
    assert m.n_cols == 2592
    ctx = V.VerticalContext(p)
    dm = V.device_member(m)
    cur = m.copy()
    worst = 0.0
    for step in range(100):
        V.advance_vertical_all(ctx, [dm], 2.0)
        out = dm.to_numpy()
        ref, st_ref = ref_advance(oracle_lib, cur, p, 2.0)
        assert (st_ref == 0).all(), f"step {step}: oracle status"
        rep = assert_state_close(out, ref, STATE)
        worst = max(worst, max(rep.values()))
        for k in synthetic.Member.STATE + synthetic.Member.COEFFS:
            setattr(cur, k, out[k].copy())
    ctx.close()
    print(f"100 steps of 2592 columns: worst per-step normwise rel err {worst:.3e}")


@pytest.mark.parametrize("variant,n_alts", [("default", 50), ("default", 20), ("no_friction", 64),
                                            ("log_ions", 50), ("given_coefficients", 30), ("beta1", 100)])
def test_modvertical_form(torch_cuda, oracle_lib, variant, n_alts):
    """The advance_vertical_1d_rusanov argument form (ModVertical arrays)
    against the oracle over parameter variants and nAlts."""
    import torch
    from gitm_b200 import vertical as V
    p = abi.default_params(**VARIANTS[variant])
    m = synthetic.make_member(48, n_alts, seed=29 + n_alts)
    d = synthetic.to_modvertical(m, p)
    ref = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    oracle_lib.advance_1d(ref, p, 2.0)
    td = {k: (torch.from_numpy(v).cuda() if isinstance(v, np.ndarray) else v) for k, v in d.items()}
    ctx = V.VerticalContext(p)
    V.advance_vertical_1d(ctx, td, 2.0)
    got = {k: td[k].cpu().numpy() for k in ("log_rho", "temp", "vel_gd", "log_ns", "vert_vel")}
    got["log_ins"] = td["log_ins"].cpu().numpy()[:9]
    want = {k: ref[k] for k in ("log_rho", "temp", "vel_gd", "log_ns", "vert_vel")}
    want["log_ins"] = ref["log_ins"][:9]
    assert_state_close(got, want, list(got))


def test_cfl_timestep(torch_cuda, oracle_lib):
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(300, 50, seed=31)
    want = oracle_lib.cfl_dt(m, p, 0.75)
    ctx = V.VerticalContext(p)
    dm = V.device_member(m)
    got = V.calc_timestep_vertical(ctx, [dm], cfl=0.75, dt=1e32, dt_end=1e32)
    assert got == pytest.approx(want, rel=1e-14)
    assert V.calc_timestep_vertical(ctx, [dm], cfl=0.75, dt=0.5) == 0.5


def test_cfl_timestep_ragged_members(torch_cuda, oracle_lib):
    """calc_timestep_vertical over members of different nAlts and sizes:
    the minimum over all their columns (the reference's MPI_Allreduce MIN
    over blocks), and dt_end when it is smaller."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    ms = [synthetic.make_member(n, na, seed=90 + i) for i, (n, na) in enumerate([(77, 20), (500, 50), (33, 100)])]
    want = min(oracle_lib.cfl_dt(m, p, 0.6) for m in ms)
    ctx = V.VerticalContext(p)
    dms = [V.device_member(m) for m in ms]
    assert V.calc_timestep_vertical(ctx, dms, cfl=0.6) == pytest.approx(want, rel=1e-14)
    assert V.calc_timestep_vertical(ctx, dms, cfl=0.6, dt_end=0.5 * want) == 0.5 * want


def test_graph_capture_replays(torch_cuda, oracle_lib):
    import torch
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(200, 50, seed=32)
    ref, _ = ref_advance(oracle_lib, m, p, 2.0, n_steps=3)
    ctx = V.VerticalContext(p)
    dm = V.device_member(m)
    plan = V.Plan(ctx, [dm])
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            plan.advance(2.0, 1, stream=s)
    torch.cuda.synchronize()
    # capture does not execute: the state is still the input
    np.testing.assert_array_equal(dm.tensors["rho"].cpu().numpy(), m.rho)
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    plan.check()
    assert_state_close(dm.to_numpy(), ref, STATE, rtol=1e-9)


def test_autotune_leaves_state(torch_cuda):
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(3000, 50, seed=33)
    ctx = V.VerticalContext(p)
    dm = V.device_member(m)
    plan = V.Plan(ctx, [dm])
    cfg = plan.autotune(2.0, 2)
    assert cfg.threads in (128, 160, 192, 256, 320, 384, 512)
    np.testing.assert_array_equal(dm.tensors["ndensity_s"].cpu().numpy(), m.ndensity_s)
    assert plan.status() == (0, 0)
