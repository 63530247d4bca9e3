"""The allocation-free step, gitm_vert_advance_native_noalloc, through the C ABI.

It serves callers that cannot allocate device memory while they run (a host
whose GPU memory belongs to its own pool, per-step loops that must not
synchronise on an allocation); its scratch is a fixed file-scope device
array.  Checked against the existing plan entry point and against the oracle
on two calls in a row, with the parity tolerance of the other GPU tests.
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import assert_state_close

pytestmark = pytest.mark.gpu
STATE = synthetic.Member.STATE + ("log_ns", "ndensity")


@pytest.mark.parametrize("n_steps,n_alts", [(1, 50), (4, 50), (1, 100)],
                         ids=["1step_nalts50", "4steps_nalts50", "1step_nalts100"])
def test_noalloc_matches_existing_entry_point_and_oracle_on_two_calls(oracle_lib, n_steps, n_alts):
    """Two calls in a row: each against gitm_vert_advance_native (the existing
    entry point) on the same state, and against the oracle; n_steps > 1 runs
    the resident multi-step loop through the shared scratch, nAlts = 100 the
    one-column-per-CTA shape."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(3000 if n_alts == 50 else 900, n_alts, seed=61)
    ctx = V.VerticalContext(p)
    ref = V.device_member(m)
    new = V.device_member(m)
    cpu = m.copy()
    status = torch.full((m.n_cols,), 7, dtype=torch.int32, device="cuda")
    for call in range(2):
        V.advance_vertical_all(ctx, [ref], 2.0, n_steps)  # the existing entry point
        b = new.batch()
        rc = _lib.lib().gitm_vert_advance_native_noalloc(ctx.handle, C.byref(b), 2.0, n_steps,
                                                          C.c_void_p(status.data_ptr()), None)
        assert rc == abi.OK, ctx.last_error()
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0, f"call {call}: status words set"
        got = new.to_numpy()
        assert_state_close(got, ref.to_numpy(), STATE, rtol=1e-10 if n_steps == 1 else 1e-9)
        st_ref = oracle_lib.advance(cpu, p, 2.0, n_steps)
        assert (st_ref == 0).all()
        assert_state_close(got, dict(cpu.arrays()), STATE, rtol=1e-10 if n_steps == 1 else 1e-9)
        # the next oracle call starts from this call's GPU result
        for k in synthetic.Member.STATE + synthetic.Member.COEFFS:
            setattr(cpu, k, got[k].copy())
    ctx.close()


def test_noalloc_rejects_host_arrays():
    """Every pointer the kernels read must be device memory."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(abi.default_params())
    m = synthetic.make_member(4, 50, seed=64)
    dm = V.device_member(m)
    b = dm.batch()
    host_alt = np.ascontiguousarray(m.altitude)
    b.altitude = abi.dptr(host_alt.ctypes.data)  # a host grid: refused before any launch
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _lib.lib().gitm_vert_advance_native_noalloc(ctx.handle, C.byref(b), 2.0, 1,
                                                      C.c_void_p(status.data_ptr()), None)
    assert rc == abi.ERR_ARG
    assert "device pointers" in ctx.last_error()
    ctx.close()


def test_noalloc_rejects_oversized_member():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(abi.default_params())
    m = V.device_member(synthetic.make_member(4, 50, seed=62))
    b = m.batch()
    b.n_cols = 262145  # one more than the stated limit; rejected before any access
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _lib.lib().gitm_vert_advance_native_noalloc(ctx.handle, C.byref(b), 2.0, 1,
                                                      C.c_void_p(status.data_ptr()), None)
    assert rc == abi.ERR_ARG
    assert "262144" in ctx.last_error()


def test_noalloc_rejects_ausm():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    ctx = V.VerticalContext(abi.default_params(solver=abi.SOLVER_AUSM))
    m = V.device_member(synthetic.make_member(4, 50, seed=63))
    b = m.batch()
    status = torch.zeros(4, dtype=torch.int32, device="cuda")
    rc = _lib.lib().gitm_vert_advance_native_noalloc(ctx.handle, C.byref(b), 2.0, 1,
                                                      C.c_void_p(status.data_ptr()), None)
    assert rc == abi.ERR_UNSUPPORTED
