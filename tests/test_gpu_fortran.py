"""The Fortran-layout drop-in (gitm_vert_advance_fortran) on ModGITM-shaped
arrays in Fortran order, against the native path on the same columns."""
import ctypes as C

import numpy as np
import pytest

from gitm_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

NLON, NLAT, NALT, NBLK = 9, 9, 30, 2


def fortran_arrays(m):
    """ModGITM arrays (Fortran order, halo'd) holding member m's columns,
    column c = (iBlock-1)*81 + (iLat-1)*9 + (iLon-1)."""
    G = NALT + 4
    H = (NLON + 4, NLAT + 4, G)
    rng = np.random.default_rng(1)

    def halo(*extra):
        return np.asfortranarray(rng.normal(size=H + extra + (NBLK,)))  # junk in halos

    f = {
        "ndensity_s": halo(11), "idensity_s": halo(10), "rho": halo(), "temperature": halo(),
        "velocity": halo(3), "ivelocity": halo(3), "vertical_velocity": halo(6), "log_ns": halo(6),
        "ndensity": halo(), "species_density": halo(20), "species_density_old": halo(20),
        "gamma": halo(), "altitude": halo(), "gravity": halo(), "dalt": halo(), "inv_r": halo(),
        "mlatitude": halo(),
        "mean_major_mass": np.asfortranarray(rng.normal(size=H + (NBLK,))),  # per block slices
        "temp_unit": np.asfortranarray(rng.normal(size=H + (NBLK,))),
        "cmax": np.asfortranarray(rng.normal(size=(NLON + 2, NLAT + 2, NALT + 2, 3, NBLK))),
        "kappa_eddy": np.asfortranarray(rng.normal(size=(NLON, NLAT, G, NBLK))),
        "cos_latitude": np.asfortranarray(rng.normal(size=(NLAT + 4, NBLK))),
        "sza": np.asfortranarray(rng.normal(size=(NLON, NLAT, NBLK))),
    }
    for b in range(NBLK):
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
                f["mlatitude"][li, lj, NALT + 1, b] = m.mlat[c]
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


def state_struct(arrays, getptr):
    st = abi.GitmFortranState()
    st.n_lons, st.n_lats, st.n_alts, st.n_blocks = NLON, NLAT, NALT, NBLK
    for name in abi.FORTRAN_ARRAYS:
        ptr, strides = getptr(name)
        setattr(st, name, descriptor(ptr, strides, name))
    return st


@pytest.mark.parametrize("on_device", [0, 1])
def test_fortran_layout_matches_native(on_device):
    import torch
    from gitm_b200 import _lib
    from gitm_b200 import vertical as V
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p = abi.default_params(compute_coefficients=0)
    m = synthetic.make_member(NLON * NLAT * NBLK, NALT, seed=41)
    # CosLatitude(iLat, iBlock) is one value per latitude row
    for b in range(NBLK):
        for j in range(NLAT):
            row = slice(b * 81 + j * 9, b * 81 + j * 9 + 9)
            m.cos_lat[row] = m.cos_lat[b * 81 + j * 9]
    f = fortran_arrays(m)
    ns_in = f["ndensity_s"].copy()
    # native reference on the same columns, through the entry point the
    # Fortran form calls (device arrays: gitm_vert_advance_native; host
    # arrays: gitm_vert_advance_native_host), so that the same kernel runs
    ctx = V.VerticalContext(p)
    if on_device:
        dm = V.device_member(m)
        V.advance_vertical_all(ctx, [dm], 2.0)
        ref = dm.to_numpy()
    else:
        h = m.copy()
        V.advance_vertical_all_host(ctx, [h], 2.0)
        ref = dict(h.arrays())
    for blk in range(1, NBLK + 1):
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
        st = state_struct(f, getptr)
        rc = _lib.lib().gitm_vert_advance_fortran(ctx.handle, C.byref(st), blk, blk, 2.0, on_device)
        assert rc == abi.OK, ctx.last_error()
        if on_device:
            torch.cuda.synchronize()
            for k in f:
                f[k] = np.asfortranarray(tens[k].cpu().numpy())
    G = NALT + 4
    for b in range(NBLK):
        for j in range(NLAT):
            for i in range(NLON):
                c = b * 81 + j * 9 + i
                li, lj = i + 2, j + 2
                np.testing.assert_array_equal(f["ndensity_s"][li, lj, :, :6, b], ref["ndensity_s"][:, :, c].T)
                np.testing.assert_array_equal(f["idensity_s"][li, lj, :, :, b], ref["idensity_s"][:, :, c].T)
                np.testing.assert_array_equal(f["rho"][li, lj, :, b], ref["rho"][0, :, c])
                np.testing.assert_array_equal(f["temperature"][li, lj, :, b], ref["temperature"][0, :, c])
                np.testing.assert_array_equal(f["velocity"][li, lj, :, :, b], ref["velocity"][:, :, c].T)
                np.testing.assert_array_equal(f["vertical_velocity"][li, lj, :, :, b], ref["vert_vel"][:, :, c].T)
                np.testing.assert_array_equal(f["log_ns"][li, lj, :, :, b], ref["log_ns"][:, :, c].T)
                np.testing.assert_array_equal(f["ndensity"][li, lj, :, b], ref["ndensity"][0, :, c])
                # SpeciesDensityOld = state before, SpeciesDensity = after (advance_vertical.f90:152-155,214-217)
                np.testing.assert_array_equal(f["species_density_old"][li, lj, :, :6, b], ns_in[li, lj, :, :6, b])
                np.testing.assert_array_equal(f["species_density"][li, lj, :, :6, b], ref["ndensity_s"][:, :, c].T)
                np.testing.assert_array_equal(f["species_density"][li, lj, :, 11:20, b], ref["idensity_s"][:9, :, c].T)
    # halo cells are untouched
    np.testing.assert_array_equal(f["ndensity_s"][0, :, :, :, :], ns_in[0, :, :, :, :])
