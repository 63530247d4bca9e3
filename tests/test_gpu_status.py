"""Per-column status words for the reference's stop_gitm triggers (run on a B200).

Each test plants the failing input on the host, runs one step through the C
ABI and through the oracle on the same columns, and checks that the status
words are equal, that the failing column carries the expected bit, and that
every other column is unaffected (no bit, state within the parity tolerance).
Nothing here faults or traps the GPU: the kernels record the condition and
carry on.
"""
import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import assert_state_close
from tests.test_gpu_parity import STATE, gpu_advance, ref_advance

pytestmark = pytest.mark.gpu

N_COLS, N_ALTS, BAD = 24, 50, 9


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _others(d: dict, bad: int) -> dict:
    keep = np.arange(N_COLS) != bad
    return {k: v[..., keep] for k, v in d.items() if isinstance(v, np.ndarray) and v.shape[-1] == N_COLS}


def _check(out, st, ref, st_ref, bit):
    np.testing.assert_array_equal(st, st_ref)
    assert st[BAD] & bit, f"column {BAD}: status {st[BAD]:#x} lacks {bit:#x}"
    assert (st[np.arange(N_COLS) != BAD] == 0).all()
    assert_state_close(_others(out, BAD), _others(ref, BAD), STATE)


@pytest.mark.parametrize("ion", [0, 5], ids=["advected_ion", "passive_ion"])
def test_negative_ion_next_to_top(torch_cuda, oracle_lib, ion):
    """set_vertical_bcs.Earth.f90:608-620: an ion density below zero within
    five cells of the top with a negative value six cells below the ghost cell
    stops the reference (GITM_ST_NEG_ION_TOP)."""
    p = abi.default_params()
    m = synthetic.make_member(N_COLS, N_ALTS, seed=71)
    for i_alt in (N_ALTS - 5, N_ALTS - 4):  # Fortran cells; native cell g = iAlt + 1
        m.idensity_s[ion, i_alt + 1, BAD] = -1.0e3
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0)
    _check(out, st, ref, st_ref, abi.ST_NEG_ION_TOP)


def test_negative_ion_repaired_without_stop(torch_cuda, oracle_lib):
    """A negative ion density within five cells of the top with a positive value
    six cells below is repaired in place (set_vertical_bcs.Earth.f90:622-645)
    and sets no bit; the repaired column matches the oracle."""
    p = abi.default_params()
    m = synthetic.make_member(N_COLS, N_ALTS, seed=72)
    m.idensity_s[0, N_ALTS - 2 + 1, BAD] = -5.0
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0)
    np.testing.assert_array_equal(st, st_ref)
    assert (st == 0).all()
    assert_state_close(out, ref, STATE)


@pytest.mark.parametrize("friction", [1, 0], ids=["friction", "no_friction"])
def test_nonfinite_temperature(torch_cuda, oracle_lib, friction):
    """A NaN temperature in one interior cell.  With neutral friction the row
    of that cell's friction matrix is all NaN, which ludcmp treats as a zero
    row and stops on ('singular matrix in ludcmp', ludcmp.f:9-17:
    GITM_ST_LU_SINGULAR); with or without it the step's result is not finite
    (check_for_nans.f90: GITM_ST_NONFINITE)."""
    p = abi.default_params(use_neutral_friction=friction)
    m = synthetic.make_member(N_COLS, N_ALTS, seed=73)
    m.temperature[0, 26, BAD] = np.nan
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0)
    out, st = gpu_advance(m, p, 2.0)
    _check(out, st, ref, st_ref, abi.ST_NONFINITE)
    if friction:
        assert st[BAD] & abi.ST_LU_SINGULAR
    else:
        assert not st[BAD] & abi.ST_LU_SINGULAR



def test_host_watchdog_times_out_and_recovers(torch_cuda):
    """gitm_vert_plan_wait returns GITM_ERR_TIMEOUT while a long launch is
    still running (a zero timeout right after issuing 8 resident steps of
    64,800 columns, about 40 ms of work) and GITM_OK once it has finished;
    the context and the plan stay usable and the state is the same as
    without the watchdog.  Nothing on the device waits."""
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.globe_member(1.0, 1.0, n_alts=50, seed=5)
    ctx = V.VerticalContext(p)
    a, b = V.device_member(m), V.device_member(m)
    pa, pb = V.Plan(ctx, [a]), V.Plan(ctx, [b])
    for plan in (pa, pb):
        plan.set_config(threads=384, steps_per_launch=8)
    torch_cuda.cuda.synchronize()
    pa.advance(2.0, 8)
    assert pa.wait(0.0) is False
    assert pa.wait(60.0) is True
    pa.check()
    pb.advance(2.0, 8)
    torch_cuda.cuda.synchronize()
    pb.check()
    for k in synthetic.Member.STATE:
        assert torch_cuda.equal(a.tensors[k], b.tensors[k]), k
    pa.close()
    pb.close()
    ctx.close()
