"""The Fortran-layout drop-in (gitm_vert_advance_fortran) on ModGITM-shaped
arrays in Fortran order, against the oracle on the same columns.

The blocks are 9 x 9 columns (GITM's default grid, Config.pl -g=9,9,50,4);
the largest case is GITM's default run of 2 x 2 blocks = 324 columns at
nAlts = 50, one step of dt = 2 s."""
import ctypes as C

import numpy as np
import pytest

from gitm_b200 import abi, synthetic
from tests.parity import assert_state_close

pytestmark = pytest.mark.gpu

NLON, NLAT = 9, 9


def fortran_arrays(m, n_blk):
    """ModGITM arrays (Fortran order, halo'd) holding member m's columns,
    column c = (iBlock-1)*81 + (iLat-1)*9 + (iLon-1)."""
    n_alt = m.n_alts
    G = n_alt + 4
    H = (NLON + 4, NLAT + 4, G)
    rng = np.random.default_rng(1)

    def halo(*extra):
        return np.asfortranarray(rng.normal(size=H + extra + (n_blk,)))  # junk in halos

    f = {
        "ndensity_s": halo(11), "idensity_s": halo(10), "rho": halo(), "temperature": halo(),
        "velocity": halo(3), "ivelocity": halo(3), "vertical_velocity": halo(6), "log_ns": halo(6),
        "ndensity": halo(), "species_density": halo(20), "species_density_old": halo(20),
        "gamma": halo(), "altitude": halo(), "gravity": halo(), "dalt": halo(), "inv_r": halo(),
        "mlatitude": halo(),
        "mean_major_mass": np.asfortranarray(rng.normal(size=H + (n_blk,))),  # per block slices
        "temp_unit": np.asfortranarray(rng.normal(size=H + (n_blk,))),
        "cmax": np.asfortranarray(rng.normal(size=(NLON + 2, NLAT + 2, n_alt + 2, 3, n_blk))),
        "kappa_eddy": np.asfortranarray(rng.normal(size=(NLON, NLAT, G, n_blk))),
        "cos_latitude": np.asfortranarray(rng.normal(size=(NLAT + 4, n_blk))),
        "sza": np.asfortranarray(rng.normal(size=(NLON, NLAT, n_blk))),
    }
    for b in range(n_blk):
        for j in range(NLAT):
            for i in range(NLON):
                c = b * 81 + j * 9 + i
                li, lj = i + 2, j + 2  # Fortran index 1 -> offset 2 in a -1 based halo
                f["ndensity_s"][li, lj, :, :6, b] = m.ndensity_s[:, :, c].T
                f["idensity_s"][li, lj, :, :, b] = m.idensity_s[:, :, c].T
                f["rho"][li, lj, :, b] = m.rho[0, :, c]
                f["temperature"][li, lj, :, b] = m.temperature[0, :, c]
                f["velocity"][li, lj, :, :, b] = m.velocity[:, :, c].T
                f["ivelocity"][li, lj, :, 2, b] = m.ivel_up[0, :, c]
                f["vertical_velocity"][li, lj, :, :, b] = m.vert_vel[:, :, c].T
                f["gamma"][li, lj, :, b] = m.gamma[0, :, c]
                f["mean_major_mass"][li, lj, :, b] = m.mean_major_mass[0, :, c]
                f["temp_unit"][li, lj, :, b] = m.temp_unit[0, :, c]
                f["cmax"][i + 1, j + 1, :, 2, b] = m.cmax[0, 1:G - 1, c]
                f["kappa_eddy"][i, j, :, b] = m.eddy[0, :, c]
                f["altitude"][li, lj, :, b] = m.altitude
                f["gravity"][li, lj, :, b] = m.gravity
                f["dalt"][li, lj, :, b] = m.dalt_c
                f["inv_r"][li, lj, :, b] = m.inv_r
                f["mlatitude"][li, lj, n_alt + 1, b] = m.mlat[c]
                f["sza"][i, j, b] = m.sza[c]
                f["cos_latitude"][lj, b] = m.cos_lat[c]
    return f


# (lon, lat, alt, field, block) axes of each array and its lower bounds
AXES = {
    "ndensity_s": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)), "idensity_s": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)),
    "velocity": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)), "ivelocity": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)),
    "vertical_velocity": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)), "log_ns": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)),
    "species_density": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)),
    "species_density_old": ((0, 1, 2, 3, 4), (-1, -1, -1, 1, 1)),
    "cmax": ((0, 1, 2, 3, 4), (0, 0, 0, 1, 1)),
    "kappa_eddy": ((0, 1, 2, None, 3), (1, 1, -1, 1, 1)),
    "cos_latitude": ((None, 0, None, None, 1), (1, -1, 1, 1, 1)),
    "sza": ((0, 1, None, None, 2), (1, 1, 1, 1, 1)),
    "mean_major_mass": ((0, 1, 2, None, 3), (-1, -1, -1, 1, 1)),
    "temp_unit": ((0, 1, 2, None, 3), (-1, -1, -1, 1, 1)),
}
for k in ("rho", "temperature", "ndensity", "gamma", "altitude", "gravity", "dalt", "inv_r", "mlatitude"):
    AXES[k] = ((0, 1, 2, None, 3), (-1, -1, -1, 1, 1))


def descriptor(ptr, strides_elems, name, block_slice=None):
    axes, lower = AXES[name]
    fa = abi.GitmFArray()
    fa.data = abi.dptr(ptr)
    for d in range(5):
        fa.lower[d] = lower[d]
        fa.stride[d] = 0 if axes[d] is None else strides_elems[axes[d]]
    return fa


def state_struct(n_alts, n_blk, getptr):
    st = abi.GitmFortranState()
    st.n_lons, st.n_lats, st.n_alts, st.n_blocks = NLON, NLAT, n_alts, n_blk
    for name in abi.FORTRAN_ARRAYS:
        ptr, strides = getptr(name)
        setattr(st, name, descriptor(ptr, strides, name))
    return st


@pytest.mark.parametrize("on_device", [0, 1])
@pytest.mark.parametrize("n_blk,n_alt", [(2, 30), (4, 50), (1, 8), (3, 64), (5, 100)],
                         ids=["2blocks_nalts30", "4blocks_nalts50", "1block_nalts8", "3blocks_nalts64",
                              "5blocks_nalts100"])
def test_fortran_layout_matches_oracle(oracle_lib, on_device, n_blk, n_alt):
    import torch
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = abi.default_params(compute_coefficients=0)
    m = synthetic.make_member(NLON * NLAT * n_blk, n_alt, seed=41)
    # CosLatitude(iLat, iBlock) is one value per latitude row
    for b in range(n_blk):
        for j in range(NLAT):
            row = slice(b * 81 + j * 9, b * 81 + j * 9 + 9)
            m.cos_lat[row] = m.cos_lat[b * 81 + j * 9]
    f = fortran_arrays(m, n_blk)
    ns_in = f["ndensity_s"].copy()
    # the oracle on the same columns (native layout, host memory)
    r = m.copy()
    r.log_ns = np.zeros_like(m.ndensity_s)
    r.ndensity = np.zeros_like(m.rho)
    st_ref = oracle_lib.advance(r, p, 2.0, 1)
    assert (st_ref == 0).all()
    ref = dict(r.arrays())
    ctx = V.VerticalContext(p)
    for blk in range(1, n_blk + 1):
        # MeanMajorMass / TempUnit hold one block (calc_rates(iBlock)): give
        # the descriptor this block's slice through a zero block stride
        if on_device:
            tens = {k: torch.from_numpy(v).cuda() for k, v in f.items()}

            def getptr(name):
                t = tens[name]
                strides = list(t.stride())
                ptr = t.data_ptr()
                if name in ("mean_major_mass", "temp_unit"):
                    ptr += (blk - 1) * strides[3] * 8
                    strides[3] = 0
                return ptr, strides
        else:
            def getptr(name):
                a = f[name]
                strides = [s // 8 for s in a.strides]
                ptr = a.ctypes.data
                if name in ("mean_major_mass", "temp_unit"):
                    ptr += (blk - 1) * strides[3] * 8
                    strides[3] = 0
                return ptr, strides
        st = state_struct(n_alt, n_blk, getptr)
        rc = _lib.lib().gitm_vert_advance_fortran(ctx.handle, C.byref(st), blk, blk, 2.0, on_device)
        assert rc == abi.OK, ctx.last_error()
        if on_device:
            torch.cuda.synchronize()
            for k in f:
                f[k] = np.asfortranarray(tens[k].cpu().numpy())
    ctx.close()
    # gather the Fortran arrays back into the native layout and compare
    n = NLON * NLAT * n_blk
    G = n_alt + 4
    got = {"ndensity_s": np.zeros((6, G, n)), "idensity_s": np.zeros((10, G, n)), "rho": np.zeros((1, G, n)),
           "temperature": np.zeros((1, G, n)), "velocity": np.zeros((3, G, n)), "vert_vel": np.zeros((6, G, n)),
           "log_ns": np.zeros((6, G, n)), "ndensity": np.zeros((1, G, n))}
    sd_new, sd_old = np.zeros((20, G, n)), np.zeros((20, G, n))
    for b in range(n_blk):
        for j in range(NLAT):
            for i in range(NLON):
                c = b * 81 + j * 9 + i
                li, lj = i + 2, j + 2
                got["ndensity_s"][:, :, c] = f["ndensity_s"][li, lj, :, :6, b].T
                got["idensity_s"][:, :, c] = f["idensity_s"][li, lj, :, :, b].T
                got["rho"][0, :, c] = f["rho"][li, lj, :, b]
                got["temperature"][0, :, c] = f["temperature"][li, lj, :, b]
                got["velocity"][:, :, c] = f["velocity"][li, lj, :, :, b].T
                got["vert_vel"][:, :, c] = f["vertical_velocity"][li, lj, :, :, b].T
                got["log_ns"][:, :, c] = f["log_ns"][li, lj, :, :, b].T
                got["ndensity"][0, :, c] = f["ndensity"][li, lj, :, b]
                sd_new[:, :, c] = f["species_density"][li, lj, :, :, b].T
                sd_old[:, :, c] = f["species_density_old"][li, lj, :, :, b].T
                # SpeciesDensityOld = state before (advance_vertical.f90:152-155)
                np.testing.assert_array_equal(f["species_density_old"][li, lj, :, :6, b], ns_in[li, lj, :, :6, b])
    assert_state_close(got, ref, tuple(got))
    # SpeciesDensity = NDensityS and IDensityS after the step (advance_vertical.f90:214-217)
    np.testing.assert_array_equal(sd_new[:6], got["ndensity_s"])
    np.testing.assert_array_equal(sd_new[11:20], got["idensity_s"][:9])
    # halo cells are untouched
    np.testing.assert_array_equal(f["ndensity_s"][0, :, :, :, :], ns_in[0, :, :, :, :])
