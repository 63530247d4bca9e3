"""gitm_hz_advance (the horizontal advance) on the GPU vs the CPU oracle, on
the same seeded blocks, through libgitmvert.so.

Tolerance as the vertical parity tests: the normwise relative error of every
output over the interior cells of every block at most 1e-10; the electron
sum and the ghost cells are compared the same way over the whole arrays.
"""
import numpy as np
import pytest

from gitm_b200 import abi
from gitm_b200 import horizontal as H

pytestmark = pytest.mark.gpu

RTOL = 1e-10


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gitm_b200 import vertical as V
    c = V.VerticalContext(abi.default_params())
    yield c
    c.close()


def _compare(got: dict, want: dict, names=H.OUTPUTS, rtol=RTOL):
    for k in names:
        g, w = got[k], want[k]
        assert g.shape == w.shape, k
        assert np.isfinite(g).all(), k
        scale = max(float(np.abs(w).max()), 1e-300)
        err = float(np.linalg.norm((g - w).ravel())) / max(float(np.linalg.norm(w.ravel())), 1e-300)
        if k == "temp_source":  # a difference of temperatures: relative to the temperature scale
            err = float(np.abs(g - w).max()) / float(np.abs(want.get("temperature", w)).max())
        assert err <= rtol or float(np.abs(g - w).max()) <= 1e-300 * scale, f"{k}: {err:.3e}"


def _run(ctx, blocks, params, dt=2.0, steps=1):
    d = blocks.to_device()
    for _ in range(steps):
        H.advance_horizontal(ctx, d, dt, params)
    return d.to_numpy()


def _ref(oracle_lib, blocks, params, dt=2.0, steps=1):
    r = blocks.copy()
    for _ in range(steps):
        st = oracle_lib.hz_advance(r, params, dt)
        assert (st == 0).all()
    return r.arrays


VARIANTS = {
    "default": dict(),
    "no_coriolis": dict(use_coriolis=0),
    "no_improved_ions": dict(use_improved_ion_advection=0),
    "no_ion_advection": dict(use_ion_advection=0),
    "non_magnetic": dict(non_magnetic=1),
    "beta1": dict(beta_limiter=1.0),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_hz_matches_oracle(ctx, oracle_lib, variant):
    p = abi.default_hz_params(**VARIANTS[variant])
    b = H.synthetic_blocks(9, 9, 20, 4, 2, seed=11)
    got = _run(ctx, b, p)
    want = _ref(oracle_lib, b, p)
    _compare(got, want)


@pytest.mark.parametrize("shape", [(5, 7, 12, 3, 2), (16, 16, 6, 2, 2), (1, 4, 5, 4, 2), (3, 1, 5, 2, 3),
                                   (11, 11, 3, 1, 1)])
def test_hz_block_shapes(ctx, oracle_lib, shape):
    """Non-square blocks, the 256-thread shape, one-cell-wide blocks (the
    gradient's nLons > 1 / nLats > 1 branches) and a single block."""
    nl, nt, na, bl, bt = shape
    p = abi.default_hz_params()
    b = H.synthetic_blocks(nl, nt, na, bl, bt, seed=12 + nl)
    _compare(_run(ctx, b, p), _ref(oracle_lib, b, p))


def test_hz_three_steps(ctx, oracle_lib):
    p = abi.default_hz_params()
    b = H.synthetic_blocks(9, 9, 10, 4, 2, seed=13)
    _compare(_run(ctx, b, p, steps=3), _ref(oracle_lib, b, p, steps=3), rtol=1e-9)


def test_hz_uniform_state_is_steady(ctx):
    """Constant fields and no horizontal wind: every array is left bit for bit."""
    b = H.synthetic_blocks(9, 9, 10, 2, 2, seed=14)
    A = b.arrays
    for name in ("rho", "temperature", "gamma"):
        A[name][:] = A[name][:, :, 2:3, 2:3]
    for name in ("velocity", "vert_vel", "ndensity_s", "idensity_s", "ivelocity"):
        A[name][:] = A[name][:, :, :, 2:3, 2:3]
    A["cmax"][:] = A["cmax"][:, :, :, 1:2, 1:2]
    A["velocity"][:, 0:2] = 0.0
    got = _run(ctx, b, abi.default_hz_params(use_coriolis=0, use_ion_advection=0))
    for k in ("rho", "temperature", "velocity", "vert_vel", "ndensity_s", "idensity_s"):
        np.testing.assert_array_equal(got[k], A[k], err_msg=k)


def test_hz_rejects_large_blocks(ctx):
    from gitm_b200 import vertical as V
    b = H.synthetic_blocks(17, 16, 2, 1, 1, seed=15).to_device()
    with pytest.raises(V.GitmError):
        H.advance_horizontal(ctx, b, 2.0)


# ---------------------------------------------------------------- exchange
@pytest.mark.parametrize("cfg", [dict(shape=(9, 9, 10, 4, 2)), dict(shape=(5, 7, 6, 6, 3)),
                                 dict(shape=(4, 4, 5, 2, 2), use_ion_advection=False),
                                 dict(shape=(6, 5, 4, 4, 2), non_magnetic=True),
                                 dict(shape=(5, 5, 3, 4, 3), north_pole=False, south_pole=False)])
def test_exchange_matches_oracle(ctx, cfg):
    """gitm_hz_exchange against the block-by-block restatement, bit for bit
    (copies and sign changes only)."""
    from oracle import hz_exchange as X
    nl, nt, na, nbl, nbt = cfg["shape"]
    flags = {k: v for k, v in cfg.items() if k != "shape"}
    b = H.synthetic_blocks(nl, nt, na, nbl, nbt, seed=20 + nl)
    ref = b.copy()
    X.exchange(ref.arrays, nl, nt, na, nbl, nbt, **flags)
    d = b.to_device()
    H.exchange_messages(ctx, d, **flags)
    got = d.to_numpy()
    for k in ("rho", "temperature", "itemperature", "etemperature", "velocity", "vert_vel", "ndensity_s",
              "idensity_s", "ivelocity", "ivelocity_par"):
        np.testing.assert_array_equal(got[k], ref.arrays[k], err_msg=k)


def test_exchange_then_advance_then_exchange(ctx, oracle_lib):
    """advance_horizontal_all's sequence (exchange, advance, exchange) on the
    GPU against the restatements."""
    from oracle import hz_exchange as X
    nl, nt, na, nbl, nbt = 9, 9, 8, 4, 2
    b = H.synthetic_blocks(nl, nt, na, nbl, nbt, seed=30)
    p = abi.default_hz_params()
    ref = b.copy()
    X.exchange(ref.arrays, nl, nt, na, nbl, nbt)
    assert (oracle_lib.hz_advance(ref, p, 2.0) == 0).all()
    X.exchange(ref.arrays, nl, nt, na, nbl, nbt)
    d = b.to_device()
    H.exchange_messages(ctx, d)
    H.advance_horizontal(ctx, d, 2.0, p)
    H.exchange_messages(ctx, d)
    _compare(d.to_numpy(), ref.arrays)


def test_exchange_reports_low_temperature(ctx):
    from gitm_b200 import vertical as V
    b = H.synthetic_blocks(5, 5, 3, 4, 2, seed=31)
    b.arrays["temperature"][3, 2, 3, 3] = 50.0
    d = b.to_device()
    with pytest.raises(V.GitmStop):
        H.exchange_messages(ctx, d)


def test_exchange_rejects_odd_block_rows_with_poles(ctx):
    from gitm_b200 import vertical as V
    b = H.synthetic_blocks(5, 5, 3, 3, 2, seed=32).to_device()
    with pytest.raises(V.GitmError):
        H.exchange_messages(ctx, b)
