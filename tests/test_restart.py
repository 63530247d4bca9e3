"""Restart-file ingestion (gitm_b200/restart.py): the record format of
restart.f90, the block <-> column mapping, and a step on ingested columns."""
import numpy as np
import pytest

from gitm_b200 import abi
from gitm_b200 import restart as R

NL, NT, NA, NB = 3, 2, 20, 2


@pytest.fixture(scope="module")
def restart_dir(tmp_path_factory):
    d = tmp_path_factory.mktemp("rst")
    blocks = R.synthetic_blocks(NL, NT, NA, NB, seed=3)
    for b, blk in enumerate(blocks):
        R.write_block(str(d / R.block_name(b + 1)), blk)
    return str(d), blocks


def test_block_round_trip(restart_dir):
    d, blocks = restart_dir
    got = R.read_block(d + "/" + R.block_name(2), NL, NT, NA)
    for k, v in blocks[1].items():
        np.testing.assert_array_equal(got[k], v, err_msg=k)


def test_record_markers(restart_dir):
    """gfortran sequential records: each starts and ends with its byte count."""
    d, _ = restart_dir
    raw = open(d + "/" + R.block_name(1), "rb").read()
    n = int.from_bytes(raw[:4], "little")
    assert n == 8 * (NL + 4)
    assert int.from_bytes(raw[4 + n:8 + n], "little") == n


def test_member_columns_follow_blocks(restart_dir):
    d, blocks = restart_dir
    m = R.member_from_restart(d, NL, NT, NA, NB)
    assert m.n_cols == NL * NT * NB and m.n_alts == NA
    # column c = iLon + nLons * (iLat + nLats * block), interior cells only
    for c in (0, 4, NL * NT + 5):
        b, r = divmod(c, NL * NT)
        j, i = divmod(r, NL)
        np.testing.assert_array_equal(m.ndensity_s[:, :, c], blocks[b]["nd"][i + 2, j + 2, :, :6].T)
        np.testing.assert_array_equal(m.velocity[:, :, c], blocks[b]["vel"][i + 2, j + 2].T)
        np.testing.assert_array_equal(m.ivel_up[0, :, c], blocks[b]["ivel"][i + 2, j + 2, :, 2])
        tu = R.restart_temp_unit(blocks[b]["nd"][i + 2, j + 2])
        np.testing.assert_allclose(m.temperature[0, :, c] * tu, blocks[b]["t_k"][i + 2, j + 2], rtol=1e-15)
        assert m.cos_lat[c] == np.cos(blocks[b]["lat"][j + 2])


def test_member_back_to_blocks(restart_dir):
    d, blocks = restart_dir
    m = R.member_from_restart(d, NL, NT, NA, NB)
    back = R.member_to_blocks(m, blocks, NL, NT)
    for b in range(NB):
        for k in ("nd", "ion", "vel", "vv", "rho"):
            np.testing.assert_array_equal(back[b][k], blocks[b][k], err_msg=k)
        np.testing.assert_allclose(back[b]["t_k"], blocks[b]["t_k"], rtol=1e-14)


def test_oracle_steps_ingested_columns(restart_dir, oracle_lib):
    d, _ = restart_dir
    m = R.member_from_restart(d, NL, NT, NA, NB)
    st = oracle_lib.advance(m, abi.default_params(), 2.0, 2)
    assert (st == 0).all()
    assert np.isfinite(m.ndensity_s).all() and np.isfinite(m.temperature).all()


@pytest.mark.gpu
def test_gpu_step_on_ingested_columns(restart_dir, oracle_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tests.parity import assert_state_close
    from tests.test_gpu_parity import STATE, gpu_advance, ref_advance
    d, _ = restart_dir
    m = R.member_from_restart(d, NL, NT, NA, NB)
    p = abi.default_params()
    ref, st_ref = ref_advance(oracle_lib, m, p, 2.0, n_steps=3)
    out, st = gpu_advance(m, p, 2.0, n_steps=3)
    assert_state_close(out, ref, STATE, rtol=1e-9)
    np.testing.assert_array_equal(st, st_ref)
