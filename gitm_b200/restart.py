"""GITM restart files in and out of the native column layout.

write_restart / read_restart (restart.f90:1-130, 351-471) keep, per block,
a Fortran unformatted sequential file ``bNNNN.rst`` (gfortran records: a
4-byte length, the data, the length again) with, in this order:

  Longitude(-1:nLons+2)                  Latitude(-1:nLats+2)
  Altitude_GB(1,1,-1:nAlts+2)            (the full (lon, lat, alt) array
                                          with UseTopography)
  NDensityS(:,:,:,s)   s = 1..nSpeciesTotal, one record each
  IDensityS(:,:,:,i)   i = 1..nIons, one record each
  Temperature * TempUnit (K)             ITemperature        eTemperature
  Velocity(:,:,:,1:3)                    IVelocity(:,:,:,1:3)
  VerticalVelocity(:,:,:,1:nSpecies)     f107                Rho

(each (lon, lat, alt) array over -1..n+2 in every direction, Fortran order,
FP64).  ``read_block`` / ``write_block`` move one block; ``member_from_restart``
turns a restart directory into a ``synthetic.Member`` whose columns are the
interior (lon, lat) cells of the blocks, lon fastest, then lat, then block,
ready for ``vertical.device_member`` and the step; ``member_to_blocks`` puts
a stepped member's state back into the block arrays.

What the step needs and a restart does not hold comes from the formulas
GITM itself uses: the altitude-grid geometry (initialize.f90:148-170), the
normalised Temperature (Temperature * TempUnit / TempUnit with the
MeanMajorMass of read_restart, restart.f90:419-427), the eddy coefficient
profile from the pressure (Earth.f90:375-408, coefficient EddyDiffusionCoef)
and CosLatitude from Latitude; SZA and MLatitude depend on time and the
magnetic field and are passed in (defaults: 0).
"""
from __future__ import annotations

import math
import os
import struct

import numpy as np

from . import synthetic as S

N_SPECIES = 6          # ModEarth.f90:18
N_SPECIES_TOTAL = 11   # ModEarth.f90:26
N_IONS = 10            # ModEarth.f90:38 (ie_)


# ------------------------------------------------------------------ records
def _write_record(f, arr) -> None:
    data = np.asarray(arr, dtype="<f8").tobytes(order="F")
    n = struct.pack("<i", len(data))
    f.write(n)
    f.write(data)
    f.write(n)


def _read_record(f) -> bytes:
    head = f.read(4)
    if len(head) < 4:
        raise EOFError("restart file ends before the expected record")
    (n,) = struct.unpack("<i", head)
    data = f.read(n)
    (m,) = struct.unpack("<i", f.read(4))
    if m != n or len(data) != n:
        raise ValueError("corrupt Fortran record (length markers %d / %d)" % (n, m))
    return data


def _array(rec: bytes, shape) -> np.ndarray:
    a = np.frombuffer(rec, dtype="<f8")
    if a.size != int(np.prod(shape)):
        raise ValueError("record of %d values where %s was expected" % (a.size, tuple(shape)))
    return a.reshape(shape, order="F").astype(np.float64)


# ------------------------------------------------------------------ blocks
def block_name(i_block: int) -> str:
    """The file name of global block i_block (1-based): b0001.rst ..."""
    return "b%04d.rst" % i_block


def read_block(path: str, n_lons: int, n_lats: int, n_alts: int, n_species_total: int = N_SPECIES_TOTAL,
               n_ions: int = N_IONS, n_species: int = N_SPECIES, topography: bool = False) -> dict:
    """One block file as arrays shaped like GITM's (halo included, Fortran
    index order): lon (nLons+4), lat (nLats+4), alt (nAlts+4) or
    (nLons+4, nLats+4, nAlts+4), nd (X, nSpeciesTotal), ion (X, nIons), t_k,
    ti, te (X), vel, ivel (X, 3), vv (X, nSpecies), f107 (scalar), rho (X),
    with X = (nLons+4, nLats+4, nAlts+4)."""
    X = (n_lons + 4, n_lats + 4, n_alts + 4)
    out = {}
    with open(path, "rb") as f:
        out["lon"] = _array(_read_record(f), (n_lons + 4,))
        out["lat"] = _array(_read_record(f), (n_lats + 4,))
        out["alt"] = _array(_read_record(f), X if topography else (n_alts + 4,))
        out["nd"] = np.stack([_array(_read_record(f), X) for _ in range(n_species_total)], axis=-1)
        out["ion"] = np.stack([_array(_read_record(f), X) for _ in range(n_ions)], axis=-1)
        out["t_k"] = _array(_read_record(f), X)
        out["ti"] = _array(_read_record(f), X)
        out["te"] = _array(_read_record(f), X)
        out["vel"] = _array(_read_record(f), X + (3,))
        out["ivel"] = _array(_read_record(f), X + (3,))
        out["vv"] = _array(_read_record(f), X + (n_species,))
        out["f107"] = float(_array(_read_record(f), (1,))[0])
        out["rho"] = _array(_read_record(f), X)
    return out


def write_block(path: str, blk: dict) -> None:
    """Writes one block file in write_restart's record order (keys as
    read_block returns them; Mars's surface records are not written)."""
    with open(path, "wb") as f:
        _write_record(f, blk["lon"])
        _write_record(f, blk["lat"])
        _write_record(f, blk["alt"])
        for s in range(blk["nd"].shape[-1]):
            _write_record(f, blk["nd"][..., s])
        for i in range(blk["ion"].shape[-1]):
            _write_record(f, blk["ion"][..., i])
        for k in ("t_k", "ti", "te", "vel", "ivel", "vv"):
            _write_record(f, blk[k])
        _write_record(f, np.array([blk["f107"]]))
        _write_record(f, blk["rho"])


def restart_temp_unit(nd: np.ndarray) -> np.ndarray:
    """TempUnit as read_restart forms it (restart.f90:419-427): the mass of
    the six major species over the number of the first three."""
    den = nd[..., 0] + nd[..., 1] + nd[..., 2]
    mmm = np.zeros(nd.shape[:-1])
    for s in range(N_SPECIES):
        mmm = mmm + S.MASS[s] * nd[..., s] / den
    return mmm / S.KB


# ------------------------------------------------------------------ members
def member_from_restart(directory: str, n_lons: int, n_lats: int, n_alts: int, n_blocks: int,
                        block_start: int = 1, topography: bool = False, sza=0.0, mlat=0.0,
                        eddy_coef: float = S.EDDY_COEF, n_species_total: int = N_SPECIES_TOTAL,
                        n_ions: int = N_IONS) -> S.Member:
    """The interior columns of blocks block_start..block_start+n_blocks-1 of
    a restart directory as a Member (see the module doc for the column order
    and the derived inputs)."""
    blocks = [read_block(os.path.join(directory, block_name(block_start + b)), n_lons, n_lats, n_alts,
                         n_species_total, n_ions, N_SPECIES, topography) for b in range(n_blocks)]
    G = n_alts + 4
    il, jl = slice(2, n_lons + 2), slice(2, n_lats + 2)   # interior lon / lat (1..n)

    def cols(a):
        """(lon, lat, alt[, k]) interior -> [k][alt][column], lon fastest."""
        a = a[il, jl]                                       # (nLons, nLats, G[, k])
        if a.ndim == 3:
            a = a[..., None]
        a = np.transpose(a, (3, 2, 1, 0))                   # (k, G, nLats, nLons)
        return a.reshape(a.shape[0], G, -1)

    def gather(key, k_take=None):
        parts = []
        for blk in blocks:
            a = blk[key]
            if k_take is not None:
                a = a[..., :k_take]
            parts.append(cols(a))
        return np.ascontiguousarray(np.concatenate(parts, axis=-1))

    nd = gather("nd", N_SPECIES)
    ion = gather("ion")
    t_k = gather("t_k")[0]
    tu_r = np.concatenate([cols(restart_temp_unit(blk["nd"]))[0] for blk in blocks], axis=-1)
    temperature = t_k / tu_r
    vel = gather("vel")
    vv = gather("vv")
    ivel_up = gather("ivel")[2:3]
    rho = gather("rho")
    n_cols = nd.shape[-1]
    # altitude grid: one shared column unless topography or the blocks differ
    if topography:
        alt = np.concatenate([cols(blk["alt"])[0] for blk in blocks], axis=-1)
        shared = bool(np.all(alt == alt[:, :1]))
        alt = alt[:, 0].copy() if shared else np.ascontiguousarray(alt)
    else:
        alts = [blk["alt"] for blk in blocks]
        shared = all(np.array_equal(a, alts[0]) for a in alts)
        alt = alts[0].copy() if shared else np.ascontiguousarray(
            np.concatenate([np.repeat(a[:, None], n_lons * n_lats, axis=1) for a in alts], axis=1))
    if alt.ndim == 1:
        dalt, inv_r, grav = S.grid_geometry(alt)
    else:
        geo = [S.grid_geometry(alt[:, c]) for c in range(alt.shape[1])]
        dalt, inv_r, grav = (np.ascontiguousarray(np.stack([g[q] for g in geo], axis=1)) for q in range(3))
    lat = np.concatenate([np.repeat(blk["lat"][jl][:, None], n_lons, axis=1).reshape(-1) for blk in blocks])
    # eddy coefficient from the pressure (Earth.f90:375-408)
    pressure = temperature * rho[0]
    eddy = np.where(pressure > S.EDDY_P0, eddy_coef,
                    np.where(pressure > S.EDDY_P1,
                             eddy_coef * (pressure - S.EDDY_P1) / (S.EDDY_P0 - S.EDDY_P1), 0.0))
    gamma, _, mmm, tu, cmax = S.producers(nd, temperature, vv)
    m = S.Member(
        n_alts=n_alts, n_cols=n_cols, ndensity_s=nd, idensity_s=ion, rho=rho,
        temperature=temperature[None].copy(), velocity=vel, vert_vel=vv,
        gamma=gamma[None].copy(), mean_major_mass=mmm[None].copy(), temp_unit=tu[None].copy(),
        cmax=cmax[None].copy(), ivel_up=np.ascontiguousarray(ivel_up), eddy=eddy[None].copy(),
        cos_lat=np.cos(lat), sza=np.broadcast_to(np.asarray(sza, dtype=np.float64), (n_cols,)).copy(),
        mlat=np.broadcast_to(np.asarray(mlat, dtype=np.float64), (n_cols,)).copy(),
        altitude=alt, gravity=grav, dalt_c=dalt, inv_r=inv_r)
    m.log_ns = np.zeros((N_SPECIES, G, n_cols))
    m.ndensity = np.zeros((1, G, n_cols))
    return m


def member_to_blocks(m: S.Member, blocks: list, n_lons: int, n_lats: int) -> list:
    """The member's state written back into copies of the block arrays it
    came from (interior columns; halo cells and the minor species keep their
    values): NDensityS 1..6, IDensityS, Temperature (K, with read_restart's
    TempUnit of the new densities), Velocity, VerticalVelocity, Rho."""
    G = m.n_alts + 4
    per = n_lons * n_lats
    il, jl = slice(2, n_lons + 2), slice(2, n_lats + 2)

    def back(a_cols):
        """[k][G][per] -> (nLons, nLats, G, k)."""
        k = a_cols.shape[0]
        return np.transpose(a_cols.reshape(k, G, n_lats, n_lons), (3, 2, 1, 0))

    out = []
    for b, blk in enumerate(blocks):
        c = slice(b * per, (b + 1) * per)
        nb = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in blk.items()}
        nb["nd"][il, jl, :, :N_SPECIES] = back(m.ndensity_s[..., c])
        nb["ion"][il, jl] = back(m.idensity_s[..., c])
        nb["vel"][il, jl] = back(m.velocity[..., c])
        nb["vv"][il, jl] = back(m.vert_vel[..., c])
        nb["rho"][il, jl] = back(m.rho[..., c])[..., 0]
        tu = restart_temp_unit(nb["nd"][il, jl])
        nb["t_k"][il, jl] = back(m.temperature[..., c])[..., 0] * tu
        out.append(nb)
    return out


def synthetic_blocks(n_lons: int, n_lats: int, n_alts: int, n_blocks: int, seed: int = 0) -> list:
    """Block arrays with seeded synthetic columns (synthetic.make_member) in
    every cell, halos included: a stand-in for a restart directory, which
    the reference does not ship."""
    X = (n_lons + 4, n_lats + 4, n_alts + 4)
    per = (n_lons + 4) * (n_lats + 4)
    out = []
    for b in range(n_blocks):
        lat_edges = np.linspace(-math.pi / 2, math.pi / 2, n_blocks + 1)
        dlat = (lat_edges[b + 1] - lat_edges[b]) / n_lats
        lat = lat_edges[b] + dlat * (np.arange(-2, n_lats + 2) + 0.5)
        lon = 2 * math.pi / n_lons * (np.arange(-2, n_lons + 2) + 0.5)
        lat_cols = np.tile(np.degrees(lat)[:, None], (1, n_lons + 4)).reshape(-1)  # lon fastest
        m = S.make_member(per, n_alts, seed=seed + b, lat_deg=np.clip(lat_cols, -89.9, 89.9))

        def grid(a):  # [k][G][per] -> (lon, lat, alt, k)
            return np.transpose(a.reshape(a.shape[0], n_alts + 4, n_lats + 4, n_lons + 4), (3, 2, 1, 0))
        nd = np.zeros(X + (N_SPECIES_TOTAL,))
        nd[..., :N_SPECIES] = grid(m.ndensity_s)
        nd[..., N_SPECIES:] = 1.0e10
        blk = {"lon": lon, "lat": lat, "alt": m.altitude.copy(), "nd": nd, "ion": grid(m.idensity_s),
               "ti": np.full(X, 1000.0), "te": np.full(X, 1500.0), "vel": grid(m.velocity),
               "ivel": np.concatenate([np.zeros(X + (2,)), grid(m.ivel_up)], axis=-1),
               "vv": grid(m.vert_vel), "f107": 150.0, "rho": grid(m.rho)[..., 0]}
        blk["t_k"] = grid(m.temperature)[..., 0] * restart_temp_unit(nd)
        out.append(blk)
    return out
