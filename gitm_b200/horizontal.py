"""The horizontal advance (advance_horizontal) on the GPU: gitm_hz_advance.

The arrays are GITM's module arrays in their Fortran layout: a block array
X(-1:nLons+2, -1:nLats+2, -1:nAlts+2[, k], nBlocks) is held here as a
C-ordered array of shape (nBlocks[, k], nAlts+4, nLats+4, nLons+4), the same
bytes.  ``HzBlocks`` holds one set of them (numpy on the host, or torch CUDA
tensors after ``to_device``); ``advance_horizontal(ctx, blocks, dt)`` runs
advance_horizontal(iBlock) for every block through libgitmvert.so.

``synthetic_blocks`` builds seeded blocks of a globe with the grid metrics of
initialize.f90:193-291 (TanLatitude, CosLatitude, the lon/lat cell and face
distances and their inverses, the GradLon/GradLat coefficients of
UAM_Gradient) and smooth state fields whose ghost cells hold the same
analytic fields (a stand-in for exchange_messages_sphere).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import abi
from . import synthetic as S

# block arrays: (name, extent of the extra field dimension or 0)
STATE = (("rho", 0), ("temperature", 0), ("velocity", 3), ("vert_vel", S.NSPECIES),
         ("ndensity_s", abi.NSPECIES_TOTAL), ("idensity_s", S.NIONS))
INPUTS3 = (("gamma", 0), ("cmax", 3), ("ivelocity", 3), ("ivelocity_par", 3), ("radial_distance", 0),
           ("inv_radial_distance", 0), ("inv_dlon_dist_gb", 0), ("inv_dlon_dist_fb", 0), ("dlon_dist_fb", 0),
           ("inv_dlat_dist_gb", 0), ("inv_dlat_dist_fb", 0), ("dlat_dist_fb", 0))
LAT1 = ("latitude", "tan_latitude", "cos_latitude")       # (nBlocks, nLats+4)
GRAD_LON = ("grad_lon_m", "grad_lon_0", "grad_lon_p")    # (nBlocks, nLons)
GRAD_LAT = ("grad_lat_m", "grad_lat_0", "grad_lat_p")    # (nBlocks, nLats)
OUTPUTS = ("rho", "temperature", "velocity", "vert_vel", "ndensity_s", "idensity_s", "temp_source")


@dataclasses.dataclass
class HzBlocks:
    n_lons: int
    n_lats: int
    n_alts: int
    n_blocks: int
    arrays: dict
    n_blocks_lon: int = 0  # the sphere's block grid (block = iLat * n_blocks_lon + iLon), for the exchange
    n_blocks_lat: int = 0

    def copy(self) -> "HzBlocks":
        return HzBlocks(self.n_lons, self.n_lats, self.n_alts, self.n_blocks,
                        {k: (None if v is None else v.copy()) for k, v in self.arrays.items()},
                        self.n_blocks_lon, self.n_blocks_lat)

    def batch(self) -> abi.GitmHzBlocks:
        """GitmHzBlocks of these arrays (host numpy or CUDA tensors)."""
        b = abi.GitmHzBlocks()
        b.n_lons, b.n_lats, b.n_alts, b.n_blocks = self.n_lons, self.n_lats, self.n_alts, self.n_blocks
        for name in abi.HZ_BLOCK_FIELDS:
            a = self.arrays.get(name)
            if a is None:
                addr = 0
            elif isinstance(a, np.ndarray):
                assert a.dtype == np.float64 and a.flags.c_contiguous, name
                addr = a.ctypes.data
            else:
                import torch
                if not (a.is_cuda and a.dtype == torch.float64 and a.is_contiguous()):
                    raise ValueError(f"{name}: expected a contiguous float64 CUDA tensor")
                addr = a.data_ptr()
            setattr(b, name, abi.dptr(addr))
        return b

    def to_device(self, device="cuda") -> "HzBlocks":
        import torch
        return HzBlocks(self.n_lons, self.n_lats, self.n_alts, self.n_blocks,
                        {k: (None if v is None else torch.from_numpy(v).to(device)) for k, v in self.arrays.items()},
                        self.n_blocks_lon, self.n_blocks_lat)

    def to_numpy(self) -> dict:
        out = {}
        for k, v in self.arrays.items():
            if v is None:
                out[k] = None
            elif isinstance(v, np.ndarray):
                out[k] = v
            else:
                out[k] = v.detach().cpu().numpy()
        return out


def advance_horizontal(ctx, blocks: HzBlocks, dt: float, params=None, stream=None):
    """gitm_hz_advance on device blocks (CUDA tensors); raises GitmStop when a
    block's neutral densities went negative."""
    from ._lib import lib
    from .vertical import GitmStop, _check
    params = params or abi.default_hz_params()
    b = blocks.batch()
    s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
    _check(lib().gitm_hz_advance(ctx.handle, C.byref(params), C.byref(b), dt, C.c_void_p(s)), ctx.handle,
           "hz_advance")
    word, nbad = hz_status(ctx, clear=True)
    if word:
        raise GitmStop(word, nbad, "advance_horizontal: negative neutral density")


def exchange_batch(blocks: HzBlocks, north_pole=True, south_pole=True, use_ion_advection=True,
                   non_magnetic=False) -> abi.GitmHzExchange:
    """GitmHzExchange of these arrays (host numpy or CUDA tensors)."""
    x = abi.GitmHzExchange()
    x.n_lons, x.n_lats, x.n_alts = blocks.n_lons, blocks.n_lats, blocks.n_alts
    x.n_blocks_lon, x.n_blocks_lat = blocks.n_blocks_lon, blocks.n_blocks_lat
    x.north_pole, x.south_pole = int(north_pole), int(south_pole)
    x.use_ion_advection, x.non_magnetic = int(use_ion_advection), int(non_magnetic)
    for name in abi.HZ_EXCHANGE_FIELDS:
        a = blocks.arrays.get(name)
        addr = 0 if a is None else (a.ctypes.data if isinstance(a, np.ndarray) else a.data_ptr())
        setattr(x, name, abi.dptr(addr))
    return x


def exchange_messages(ctx, blocks: HzBlocks, stream=None, **flags):
    """gitm_hz_exchange (exchange_messages_sphere) on device blocks; raises
    GitmStop when a block's Temperature < 100 or Rho < 0 (the reference stops)."""
    from ._lib import lib
    from .vertical import GitmStop, _check
    x = exchange_batch(blocks, **flags)
    s = 0 if stream is None else int(getattr(stream, "cuda_stream", stream))
    _check(lib().gitm_hz_exchange(ctx.handle, C.byref(x), C.c_void_p(s)), ctx.handle, "hz_exchange")
    word, nbad = hz_status(ctx, clear=True)
    if word:
        raise GitmStop(word, nbad, "exchange_messages_sphere: Temperature < 100 or Rho < 0")


def hz_status(ctx, clear: bool = False):
    from ._lib import lib
    from .vertical import _check
    w = C.c_uint32()
    n = C.c_int64()
    _check(lib().gitm_hz_status(ctx.handle, C.byref(w), C.byref(n), int(clear)), ctx.handle, "hz_status")
    return int(w.value), int(n.value)


# ---------------------------------------------------------------- synthetic
def _pattern(rng, lon, lat, amp):
    """A smooth field on the sphere: a few low-order modes with random phases."""
    a = rng.uniform(0, 2 * np.pi, 4)
    return amp * (np.cos(lat) * np.cos(lon + a[0]) + 0.6 * np.sin(2 * lat) * np.sin(2 * lon + a[1]) +
                  0.3 * np.cos(3 * lat) * np.cos(3 * lon + a[2]) + 0.2 * np.sin(lat + a[3]))


def synthetic_blocks(n_lons: int = 9, n_lats: int = 9, n_alts: int = 50, n_blocks_lon: int = 4,
                     n_blocks_lat: int = 2, seed: int = 0) -> HzBlocks:
    """Blocks of n_lons x n_lats cells tiling the globe (n_blocks_lon x
    n_blocks_lat), with their ghost cells, at n_alts altitudes."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nb = n_blocks_lon * n_blocks_lat
    NI, NJ, NK = n_lons + 4, n_lats + 4, n_alts + 4
    dlon = 2 * np.pi / (n_blocks_lon * n_lons)
    dlat = np.pi / (n_blocks_lat * n_lats)
    ii = np.arange(-1, n_lons + 3)
    jj = np.arange(-1, n_lats + 3)
    lon = np.empty((nb, NI))
    lat = np.empty((nb, NJ))
    for b in range(nb):
        bi, bj = b % n_blocks_lon, b // n_blocks_lon
        lon[b] = (bi * n_lons + ii - 0.5) * dlon
        lat[b] = -np.pi / 2 + (bj * n_lats + jj - 0.5) * dlat
    # one column's vertical structure, modulated horizontally
    base = S.make_member(1, n_alts, seed=seed)
    alt = base.altitude.copy()
    R = S.RBODY + alt  # RadialDistance_GB (initialize.f90:158-159), the same at every lon / lat
    LON = lon[:, None, None, :]
    LAT = lat[:, None, :, None]
    shape = (nb, NK, NJ, NI)

    def mod(amp):
        return np.broadcast_to(_pattern(rng, LON, LAT, amp), shape)

    A = {}
    T0 = base.temperature[0, :, 0][None, :, None, None]
    A["temperature"] = np.ascontiguousarray(T0 * (1 + mod(0.05)))
    nd = np.zeros((nb, abi.NSPECIES_TOTAL, NK, NJ, NI))
    for s in range(S.NSPECIES):
        nd[:, s] = base.ndensity_s[s, :, 0][None, :, None, None] * (1 + mod(0.2))
    for s in range(S.NSPECIES, abi.NSPECIES_TOTAL):  # minor species, not advanced here
        nd[:, s] = 1e10
    A["ndensity_s"] = nd
    A["rho"] = np.ascontiguousarray(np.einsum("s,bskji->bkji", S.MASS, nd[:, :S.NSPECIES]))
    vel = np.zeros((nb, 3, NK, NJ, NI))
    vel[:, 0] = mod(60.0)
    vel[:, 1] = mod(40.0)
    vel[:, 2] = base.velocity[2, :, 0][None, :, None, None] + mod(2.0)
    A["velocity"] = vel
    vv = np.zeros((nb, S.NSPECIES, NK, NJ, NI))
    for s in range(S.NSPECIES):
        vv[:, s] = base.vert_vel[s, :, 0][None, :, None, None] + mod(1.0)
    A["vert_vel"] = vv
    ion = np.zeros((nb, S.NIONS, NK, NJ, NI))
    for s in range(S.NIONS - 1):
        ion[:, s] = base.idensity_s[s, :, 0][None, :, None, None] * (1 + mod(0.3))
    ion[:, S.NIONS - 1] = ion[:, :S.NIONS - 1].sum(axis=1)
    A["idensity_s"] = ion
    A["gamma"] = np.ascontiguousarray(base.gamma[0, :, 0][None, :, None, None] * (1 + mod(0.005)))
    iv = np.zeros((nb, 3, NK, NJ, NI))
    iv[:, 0] = mod(150.0)
    iv[:, 1] = mod(100.0)
    iv[:, 2] = mod(20.0)
    A["ivelocity"] = iv
    ivp = np.zeros((nb, 3, NK, NJ, NI))
    ivp[:, 0] = mod(30.0)
    ivp[:, 1] = mod(30.0)
    ivp[:, 2] = mod(40.0)
    A["ivelocity_par"] = ivp
    # cMax_GDB(0:nLons+1, 0:nLats+1, 0:nAlts+1, 3, nBlocks) as
    # calc_timestep_horizontal forms its east / north parts: |V| + sound speed
    cs = np.sqrt(A["gamma"] * A["temperature"])
    cm = np.zeros((nb, 3, NK, NJ, NI))
    cm[:, 0] = np.abs(vel[:, 0]) + cs
    cm[:, 1] = np.abs(vel[:, 1]) + cs
    cm[:, 2] = np.abs(vel[:, 2]) + cs
    A["cmax"] = np.ascontiguousarray(cm[:, :, 1:-1, 1:-1, 1:-1])
    # geometry (initialize.f90:193-291)
    RR = np.broadcast_to(R[None, :, None, None], shape)
    A["radial_distance"] = np.ascontiguousarray(RR)
    A["inv_radial_distance"] = np.ascontiguousarray(1 / RR)
    A["latitude"] = lat.copy()
    A["tan_latitude"] = np.minimum(np.abs(np.tan(lat)), 100.0) * np.sign(lat)
    A["cos_latitude"] = np.cos(lat)
    dlat_gb = np.ones(shape)
    dlat_fb = np.ones(shape)
    dlon_gb = np.ones(shape)
    dlon_fb = np.ones(shape)
    cosl = A["cos_latitude"]
    # Fortran index x of a (-1 : n+2) dimension is array index x + 1
    for b in range(nb):
        Lt = lambda j: lat[b, j + 1]  # noqa: E731  Latitude(j)
        Ln = lambda i: lon[b, i + 1]  # noqa: E731  Longitude(i)
        for j in range(0, n_lats + 2):      # iLat 0 .. nLats+1
            cmx = max(abs(cosl[b, j + 1]), 0.01)
            for i in range(0, n_lons + 2):  # iLon 0 .. nLons+1
                dlat_gb[b, :, j + 1, i + 1] = 0.5 * (Lt(j + 1) - Lt(j - 1)) * R
                dlat_fb[b, :, j + 1, i + 1] = (Lt(j) - Lt(j - 1)) * 0.5 * (R + R)
                dlon_gb[b, :, j + 1, i + 1] = 0.5 * (Ln(i + 1) - Ln(i - 1)) * R * cmx
                dlon_fb[b, :, j + 1, i + 1] = (Ln(i) - Ln(i - 1)) * 0.5 * (R + R) * cmx
            # longitude ghost cells (and, as the reference does, dLatDist_FB's)
            dlon_fb[b, :, j + 1, 0] = dlon_fb[b, :, j + 1, 1]
            dlon_fb[b, :, j + 1, NI - 1] = dlon_fb[b, :, j + 1, NI - 2]
            dlat_fb[b, :, j + 1, 0] = dlat_fb[b, :, j + 1, 1]
            dlat_fb[b, :, j + 1, NI - 1] = dlat_fb[b, :, j + 1, NI - 2]
        dlon_fb[b, :, 0, :] = dlon_fb[b, :, 1, :]
        dlon_fb[b, :, NJ - 1, :] = dlon_fb[b, :, NJ - 2, :]
        dlat_fb[b, :, 0, :] = dlat_fb[b, :, 1, :]
        dlat_fb[b, :, NJ - 1, :] = dlat_fb[b, :, NJ - 2, :]
    A["inv_dlat_dist_gb"] = 1.0 / dlat_gb
    A["inv_dlat_dist_fb"] = 1.0 / dlat_fb
    A["dlat_dist_fb"] = dlat_fb
    A["inv_dlon_dist_gb"] = 1.0 / dlon_gb
    A["inv_dlon_dist_fb"] = 1.0 / dlon_fb
    A["dlon_dist_fb"] = dlon_fb

    def grad_coefs(x, n):
        m = np.empty((nb, n))
        z = np.empty((nb, n))
        p = np.empty((nb, n))
        for k in range(1, n + 1):
            dm = x[:, k + 1] - x[:, k]
            dp = x[:, k + 2] - x[:, k + 1]
            r2 = (dm / dp) ** 2
            inv = 1.0 / (r2 * dp + dm)
            p[:, k - 1] = inv * r2
            z[:, k - 1] = inv * (1 - r2)
            m[:, k - 1] = -inv
        return m, z, p

    A["grad_lon_m"], A["grad_lon_0"], A["grad_lon_p"] = grad_coefs(lon, n_lons)
    A["grad_lat_m"], A["grad_lat_0"], A["grad_lat_p"] = grad_coefs(lat, n_lats)
    A["temp_source"] = np.zeros((nb, n_alts, n_lats, n_lons))
    # ion and electron temperatures (moved by the exchange, not read by the advance)
    A["itemperature"] = np.ascontiguousarray(A["temperature"] * (1.1 + mod(0.02)))
    A["etemperature"] = np.ascontiguousarray(A["temperature"] * (1.5 + mod(0.05)))
    A = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in A.items()}
    return HzBlocks(n_lons, n_lats, n_alts, nb, A, n_blocks_lon, n_blocks_lat)
