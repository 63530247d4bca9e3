"""The horizontal advance's oracle (oracle/oracle_hz.hpp, a restatement of
advance_horizontal.f90:58-1034) and the synthetic blocks: properties the
reference's scheme has, on the CPU."""
import numpy as np
import pytest

from gitm_b200 import abi
from gitm_b200 import horizontal as H


def _uniform(blocks):
    """Every altitude's fields constant in longitude and latitude, horizontal
    winds zero: no gradient, no face jump, no flux."""
    A = blocks.arrays
    for name in ("rho", "temperature", "gamma"):
        A[name][:] = A[name][:, :, 2:3, 2:3]
    for name in ("velocity", "vert_vel", "ndensity_s", "idensity_s", "ivelocity"):
        A[name][:] = A[name][:, :, :, 2:3, 2:3]
    A["cmax"][:] = A["cmax"][:, :, :, 1:2, 1:2]
    A["velocity"][:, 0:2] = 0.0
    return blocks


def test_synthetic_blocks_shapes():
    b = H.synthetic_blocks(5, 7, 12, 3, 2, seed=3)
    A = b.arrays
    assert b.n_blocks == 6
    assert A["rho"].shape == (6, 16, 11, 9)
    assert A["ndensity_s"].shape == (6, abi.NSPECIES_TOTAL, 16, 11, 9)
    assert A["latitude"].shape == (6, 11) and A["grad_lon_m"].shape == (6, 5)
    # UAM_Gradient's coefficients (initialize.f90:271-291) differentiate a
    # linear function exactly: d Latitude / d Latitude = 1
    lat = A["latitude"]
    d = A["grad_lat_m"] * lat[:, 0:7] + A["grad_lat_0"] * lat[:, 1:8] + A["grad_lat_p"] * lat[:, 2:9]
    np.testing.assert_allclose(d, 1.0, rtol=1e-12)
    assert np.all(A["inv_dlon_dist_fb"] > 0) and np.all(A["inv_dlat_dist_fb"] > 0)


def test_oracle_uniform_state_is_steady(oracle_lib):
    b = _uniform(H.synthetic_blocks(9, 9, 10, 2, 2, seed=4))
    a = b.copy()
    p = abi.default_hz_params(use_coriolis=0, use_ion_advection=0)
    st = oracle_lib.hz_advance(a, p, 2.0)
    assert (st == 0).all()
    for k in ("rho", "temperature", "velocity", "vert_vel", "ndensity_s", "idensity_s"):
        np.testing.assert_array_equal(a.arrays[k], b.arrays[k], err_msg=k)
    assert np.abs(a.arrays["temp_source"]).max() == 0.0


def test_oracle_blocks_are_independent(oracle_lib):
    """Advancing all blocks at once equals advancing one block alone."""
    b = H.synthetic_blocks(6, 4, 8, 2, 2, seed=5)
    p = abi.default_hz_params()
    all_ = b.copy()
    oracle_lib.hz_advance(all_, p, 2.0)
    one = H.HzBlocks(b.n_lons, b.n_lats, b.n_alts, 1,
                     {k: np.ascontiguousarray(v[2:3]) for k, v in b.arrays.items()})
    oracle_lib.hz_advance(one, p, 2.0)
    for k in H.OUTPUTS:
        np.testing.assert_array_equal(one.arrays[k][0], all_.arrays[k][2], err_msg=k)


def test_oracle_touches_only_interior_cells(oracle_lib):
    """Ghost cells keep their values (the electrons aside, which the
    divergence term re-sums everywhere)."""
    b = H.synthetic_blocks(5, 5, 6, 2, 1, seed=6)
    a = b.copy()
    oracle_lib.hz_advance(a, abi.default_hz_params(), 2.0)
    for k in ("rho", "temperature", "velocity", "vert_vel", "ndensity_s"):
        x, y = a.arrays[k], b.arrays[k]
        ghost = np.ones(x.shape, dtype=bool)
        ghost[..., 2:-2, 2:-2, 2:-2] = False
        np.testing.assert_array_equal(x[ghost], y[ghost], err_msg=k)
        assert np.abs(x - y).max() > 0.0, k
    ion = a.arrays["idensity_s"]
    np.testing.assert_allclose(ion[:, -1], ion[:, :-1].sum(axis=1), rtol=1e-15)


def test_oracle_temperature_source(oracle_lib):
    """HorizontalTempSource = new Temperature - old Temperature."""
    b = H.synthetic_blocks(5, 5, 6, 2, 1, seed=7)
    a = b.copy()
    oracle_lib.hz_advance(a, abi.default_hz_params(), 2.0)
    new = a.arrays["temperature"][:, 2:-2, 2:-2, 2:-2]
    old = b.arrays["temperature"][:, 2:-2, 2:-2, 2:-2]
    np.testing.assert_array_equal(a.arrays["temp_source"], new - old)


@pytest.mark.parametrize("variant", [dict(use_coriolis=0), dict(use_improved_ion_advection=0),
                                     dict(non_magnetic=1), dict(beta_limiter=1.0)])
def test_oracle_variants_change_the_result(oracle_lib, variant):
    b = H.synthetic_blocks(5, 5, 6, 2, 1, seed=8)
    a0, a1 = b.copy(), b.copy()
    oracle_lib.hz_advance(a0, abi.default_hz_params(), 2.0)
    oracle_lib.hz_advance(a1, abi.default_hz_params(**variant), 2.0)
    diff = max(np.abs(a0.arrays[k] - a1.arrays[k]).max() for k in ("velocity", "idensity_s", "temperature"))
    assert diff > 0.0


# ---------------------------------------------------------------- exchange
def _global_source(b, i, j, nl, nt, nbl, nbt):
    """The interior cell (block, i, j) a ghost cell covers on a sphere with
    both poles connected: periodic in longitude, mirrored in latitude across a
    pole with the longitude moved by nbl / 2 blocks."""
    bx, by = b % nbl, b // nbl
    G, GJ = bx * nl + i, by * nt + j
    NLON, NLAT = nl * nbl, nt * nbt
    flip = False
    if GJ < 1:
        GJ, G, flip = 1 - GJ, G + (nbl // 2) * nl, True
    elif GJ > NLAT:
        GJ, G, flip = 2 * NLAT + 1 - GJ, G + (nbl // 2) * nl, True
    G = (G - 1) % NLON + 1
    sbx, sby = (G - 1) // nl, (GJ - 1) // nt
    return sby * nbl + sbx, G - sbx * nl, GJ - sby * nt, flip


def test_exchange_oracle_follows_the_sphere():
    """Every ghost cell of altitudes 1..nAlts holds the interior cell it
    covers; winds and ion velocities change sign across the poles."""
    from oracle import hz_exchange as X
    nl, nt, na, nbl, nbt = 5, 4, 3, 4, 3
    b0 = H.synthetic_blocks(nl, nt, na, nbl, nbt, seed=9)
    b = b0.copy()
    st = X.exchange(b.arrays, nl, nt, na, nbl, nbt)
    assert (st == 0).all()
    A, A0 = b.arrays, b0.arrays
    for blk in range(nbl * nbt):
        for j in range(-1, nt + 3):
            for i in range(-1, nl + 3):
                if 1 <= i <= nl and 1 <= j <= nt:
                    continue
                sb, si, sj, flip = _global_source(blk, i, j, nl, nt, nbl, nbt)
                for k in range(1, na + 1):
                    assert A["rho"][blk, k + 1, j + 1, i + 1] == A0["rho"][sb, k + 1, sj + 1, si + 1]
                    for d in range(3):
                        sign = -1.0 if (flip and d < 2) else 1.0
                        assert A["velocity"][blk, d, k + 1, j + 1, i + 1] == \
                            sign * A0["velocity"][sb, d, k + 1, sj + 1, si + 1]
                        assert A["ivelocity_par"][blk, d, k + 1, j + 1, i + 1] == \
                            sign * A0["ivelocity_par"][sb, d, k + 1, sj + 1, si + 1]
                    for s in range(10):
                        assert A["idensity_s"][blk, s, k + 1, j + 1, i + 1] == \
                            A0["idensity_s"][sb, s, k + 1, sj + 1, si + 1]
    # the polar ghost rows of the ghost altitudes are only negated (the
    # reference's array sections run over every altitude)
    south = A["latitude"][:, 1] < -np.pi / 2
    np.testing.assert_array_equal(A["velocity"][south][:, 0:2, 0, 0:2], -A0["velocity"][south][:, 0:2, 0, 0:2])
    # interiors and the fields the exchange does not move are untouched
    np.testing.assert_array_equal(A["rho"][:, :, 2:-2, 2:-2], A0["rho"][:, :, 2:-2, 2:-2])
    np.testing.assert_array_equal(A["gamma"], A0["gamma"])


def test_exchange_oracle_without_poles_and_ions():
    from oracle import hz_exchange as X
    nl, nt, na, nbl, nbt = 4, 4, 2, 2, 2
    b0 = H.synthetic_blocks(nl, nt, na, nbl, nbt, seed=10)
    b = b0.copy()
    X.exchange(b.arrays, nl, nt, na, nbl, nbt, north_pole=False, south_pole=False, use_ion_advection=False)
    A, A0 = b.arrays, b0.arrays
    # beyond the edges nothing moves; ions are not exchanged
    np.testing.assert_array_equal(A["rho"][0:nbl, :, 0:2], A0["rho"][0:nbl, :, 0:2])
    np.testing.assert_array_equal(A["idensity_s"], A0["idensity_s"])
    assert np.abs(A["rho"] - A0["rho"]).max() > 0.0  # the east / west rings did move
