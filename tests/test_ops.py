"""torch.ops.gitm.vertical_step, the vertical step registered with torch.library.

CPU: the registration, the schema, the fake kernel on meta and fake tensors
(torch.library.opcheck), and that CPU tensors are refused (there is no CPU
kernel).  GPU: the op against the oracle, its gradient against autograd
through the FP64 PyTorch transcription of the step, and opcheck on CUDA
tensors.
"""
import numpy as np
import pytest
import torch

from gitm_b200 import abi, ops, synthetic
from tests.parity import assert_state_close

ARGNAMES = ops.STATE + ops.INPUTS


def _args(m, device, dt=2.0, n_steps=1, solver=0):
    return [torch.from_numpy(np.ascontiguousarray(getattr(m, k))).to(device) for k in ARGNAMES] + [dt, n_steps, solver]


def test_op_is_registered_with_its_schema():
    op = torch.ops.gitm.vertical_step.default
    names = [a.name for a in op._schema.arguments]
    assert names == list(ARGNAMES) + ["dt", "n_steps", "solver"]
    assert len(op._schema.returns) == 6


@pytest.mark.parametrize("test", ["test_schema", "test_autograd_registration", "test_faketensor"])
def test_opcheck_on_meta_tensors(test):
    m = synthetic.make_member(5, 20, seed=81)
    torch.library.opcheck(torch.ops.gitm.vertical_step.default, tuple(_args(m, "meta")), test_utils=[test])


def test_fake_kernel_gives_the_state_shapes():
    from torch._subclasses.fake_tensor import FakeTensorMode
    m = synthetic.make_member(7, 30, seed=82)
    with FakeTensorMode() as fm:
        a = [fm.from_tensor(t) if isinstance(t, torch.Tensor) else t for t in _args(m, "cpu")]
        out = torch.ops.gitm.vertical_step(*a)
    assert [tuple(o.shape) for o in out] == [getattr(m, k).shape for k in ops.STATE]


def test_cpu_tensors_have_no_kernel():
    m = synthetic.make_member(3, 20, seed=83)
    with pytest.raises(NotImplementedError):
        torch.ops.gitm.vertical_step(*_args(m, "cpu"))


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("n_steps,solver", [(1, 0), (3, 0), (1, 1)], ids=["rusanov_1", "rusanov_3", "ausm_1"])
def test_op_matches_oracle(cuda, oracle_lib, n_steps, solver):
    p = abi.default_params(solver=solver)
    m = synthetic.make_member(64, 50, seed=84)
    args = _args(m, cuda, 2.0, n_steps, solver)
    before = [a.clone() for a in args[:6]]
    out = torch.ops.gitm.vertical_step(*args)
    for a, b in zip(args[:6], before):
        assert torch.equal(a, b), "the op modified an input"
    ref = m.copy()
    st = oracle_lib.advance(ref, p, 2.0, n_steps)
    assert (st == 0).all()
    got = {k: o.cpu().numpy() for k, o in zip(ops.STATE, out)}
    assert_state_close(got, dict(ref.arrays()), ops.STATE, rtol=1e-10 if n_steps == 1 else 1e-9)


@pytest.mark.gpu
def test_op_gradient_matches_autograd_through_transcription(cuda):
    from tests.test_gpu_adjoint import OUT_KEYS, _torch_vjp
    p = abi.default_params()
    m = synthetic.make_member(16, 50, seed=85)
    gen = torch.Generator().manual_seed(3)
    y = {k: torch.randn(getattr(m, k).shape, generator=gen, dtype=torch.float64).to(cuda) for k in OUT_KEYS}
    args = _args(m, cuda)
    for i in (*range(6), 7):  # the state and eddy
        args[i].requires_grad_(True)
    out = torch.ops.gitm.vertical_step(*args)
    loss = sum((o * y[k]).sum() for o, k in zip(out, ops.STATE))
    g = torch.autograd.grad(loss, [args[i] for i in (*range(6), 7)])
    yy = dict(y)
    yy["log_ns"] = torch.zeros(m.ndensity_s.shape, dtype=torch.float64, device=cuda)
    yy["ndensity"] = torch.zeros(m.rho.shape, dtype=torch.float64, device=cuda)
    want = _torch_vjp(m, p, 2.0, yy, cuda)
    for (k, gg) in zip(list(ops.STATE) + ["eddy"], g):
        w = want[k]
        err = float((gg - w).norm() / max(float(w.norm()), 1e-300))
        assert err < 1e-9, f"{k}: relative error {err:.3e}"


@pytest.mark.gpu
def test_opcheck_on_cuda_tensors(cuda):
    m = synthetic.make_member(8, 50, seed=86)
    args = _args(m, cuda)
    torch.library.opcheck(torch.ops.gitm.vertical_step.default, tuple(args),
                          test_utils=["test_schema", "test_autograd_registration", "test_faketensor"])
