"""The allocation-free step, gitm_vert_advance_native_noalloc, through the C ABI.

It serves callers that cannot allocate device memory while they run (a host
whose GPU memory belongs to its own pool, work issued during stream capture,
per-step loops that must not synchronise on an allocation); its scratch is a
fixed file-scope device array.  Checked against the existing plan entry point
on two calls in a row, with the parity tolerance of the other GPU tests.
"""
import ctypes as C

import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import assert_state_close

pytestmark = pytest.mark.gpu
STATE = synthetic.Member.STATE + ("log_ns", "ndensity")


def test_noalloc_matches_existing_entry_point_on_two_calls():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    p = abi.default_params()
    m = synthetic.make_member(3000, 50, seed=61)
    ctx = V.VerticalContext(p)
    ref = V.device_member(m)
    new = V.device_member(m)
    status = torch.full((m.n_cols,), 7, dtype=torch.int32, device="cuda")
    for call in range(2):
        V.advance_vertical_all(ctx, [ref], 2.0)  # the existing entry point
        b = new.batch()
        rc = _lib.lib().gitm_vert_advance_native_noalloc(ctx.handle, C.byref(b), 2.0, 1,
                                                          C.c_void_p(status.data_ptr()), None)
        assert rc == abi.OK, ctx.last_error()
        torch.cuda.synchronize()
        assert int(status.abs().max()) == 0, f"call {call}: status words set"
        assert_state_close(new.to_numpy(), ref.to_numpy(), STATE)


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
