"""Seeded synthetic GITM columns (numpy, host memory).

There is no dataset for this path; the workloads are synthetic columns drawn
from ``numpy.random.Generator(PCG64(seed))`` with the shapes and value
distributions of GITM's Earth thermosphere:

* altitude grid 100-600 km stretched to about 0.3 local scale heights, built
  with the ``init_altitude`` recurrence (init_altitude.f90:87-118) with the
  stretch factor rescaled so cell nAlts sits at 600 km (the iteration of
  init_altitude_old, init_altitude.f90:124-192); geometry as initialize.f90:
  148-170 (dAlt_GB, InvRadialDistance_GB, Gravity_GB);
* Bates temperature T = Tinf - (Tinf - 190) exp(-0.02 (z - 100 km)/km),
  Tinf ~ U[700, 1500] K per column (190 K below 100 km);
* species O, O2, N2, N(4S), NO, He in diffusive equilibrium
  n_s(z) = n0_s (T(100 km) / T(z)) exp(-int dz / H_s), H_s = k T / (m_s g)
  (the T ratio keeps long vertical-only rollouts bounded), with n0_s
  log-uniform within +-0.3 dex of 5e17, 3e18, 1e19, 1e15, 1e14, 1e13 m^-3;
* winds: east/north N(0, 50 m/s), bulk vertical N(0, 2 m/s), species
  vertical N(0, 1 m/s), each a random profile smooth in altitude
  (``smooth_profiles``) rather than cell-to-cell noise, so long rollouts do
  not start from grid-scale waves;
* ions: Chapman layers for the 9 ions, IVelocity up N(0, 20 m/s);
* KappaEddyDiffusion from the pressure profile of
  calc_eddy_diffusion_coefficient (Earth.f90:376-411) with the coefficient
  scaled lognormally (sigma 0.3);
* derived coefficients (Gamma, MeanMajorMass, TempUnit, cMax) from the
  state with the producers of calc_pressure.f90:56-83,
  calc_rates.Earth.f90:34-50 and calc_timestep.f90:109-118.

Arrays are in the native layout [field, cell, column] (numpy C order), so a
column is the fastest-varying index.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

AMU = 1.6726e-27
KB = 1.3807e-23
RBODY = 6372.0 * 1000.0
GC = 9.8
NSPECIES = 6
NIONS = 10

# init_planet masses (ModEarth.f90:271-281), species order O, O2, N2, N, NO, He
_MO = 16.0 * AMU
_MN = 14.0 * AMU
MASS = np.array([_MO, 2 * _MO, 2 * _MN, _MN, _MN + _MO, 4.0 * AMU])
VIBRATION = np.array([5.0, 7.0, 7.0, 5.0, 7.0, 5.0])  # ModEarth.f90:307-312
BASE_DENSITY = np.array([5e17, 3e18, 1e19, 1e15, 1e14, 1e13])

# Chapman layers of the 9 ions (O+(4S), NO+, O2+, N2+, N+, O+(2D), O+(2P), H+, He+):
# peak density [m^-3], peak altitude [km], scale height [km]
ION_LAYERS = np.array([
    [8e11, 280.0, 60.0],
    [2e11, 120.0, 12.0],
    [1e11, 130.0, 15.0],
    [5e9, 150.0, 20.0],
    [2e10, 250.0, 50.0],
    [1e10, 270.0, 55.0],
    [3e9, 270.0, 55.0],
    [1e10, 550.0, 150.0],
    [5e9, 500.0, 120.0],
])

EDDY_COEF = 50.0  # ModInputs.f90:302-304
EDDY_P0 = 0.01
EDDY_P1 = 0.005


def bates_temperature(z_m: np.ndarray, tinf) -> np.ndarray:
    """Bates profile above 100 km; 190 K (isothermal) in the ghost cells below,
    where the Bates formula would fall towards 0 K."""
    dz = np.maximum(z_m / 1000.0 - 100.0, 0.0)
    return tinf - (tinf - 190.0) * np.exp(-0.02 * dz)


def _gravity(z):
    return GC * (RBODY / (RBODY + z)) ** 2


def make_altitude_grid(n_alts: int, tinf: float = 1000.0, alt_min: float = 100.0e3,
                       alt_top: float = 600.0e3) -> np.ndarray:
    """Altitudes of cells -1..nAlts+2 (length nAlts+4), in metres."""
    # mean mass of a reference column on a fine grid
    zf = np.linspace(alt_min - 20e3, alt_top + 200e3, 4001)
    tf = bates_temperature(zf, tinf)
    gf = _gravity(zf)
    dens = []
    for s in range(NSPECIES):
        inv_h = MASS[s] * gf / (KB * tf)
        integ = np.concatenate([[0.0], np.cumsum(0.5 * (inv_h[1:] + inv_h[:-1]) * np.diff(zf))])
        i100 = np.searchsorted(zf, alt_min)
        dens.append(BASE_DENSITY[s] * np.exp(-(integ - integ[i100])))
    dens = np.array(dens)
    mbar = (MASS[:, None] * dens).sum(0) / dens.sum(0)
    hf = KB * tf / (mbar * gf)

    def scale_height(z):
        return float(np.interp(z, zf, hf))

    def build(fac):
        sh = np.zeros(n_alts + 1)  # ScaleHeights(1:nAlts) -> sh[1:]
        for i in range(1, n_alts + 1):
            geo = alt_min if i == 1 else alt_min + sh[1:i].sum() * fac
            sh[i] = scale_height(geo)
        alt = np.zeros(n_alts + 4)  # index g = iAlt + 1
        alt[2] = alt_min
        alt[1] = alt_min - fac * sh[1]
        alt[0] = alt_min - 2 * fac * sh[1]
        for i in range(2, n_alts + 2):
            alt[i + 1] = alt[i] + fac * sh[i - 1]
        alt[n_alts + 3] = alt[n_alts + 2] + fac * sh[n_alts]
        return alt

    lo, hi = 0.01, 5.0
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if build(mid)[n_alts + 1] > alt_top:
            hi = mid
        else:
            lo = mid
    return build(0.5 * (lo + hi))


def grid_geometry(alt: np.ndarray):
    """dAlt_GB, InvRadialDistance_GB, Gravity_GB (initialize.f90:148-170)."""
    n = alt.shape[0]
    n_alts = n - 4
    dalt = np.zeros(n)
    for g in range(1, n - 1):  # iAlt 0..nAlts+1
        dalt[g] = 0.5 * (alt[g + 1] - alt[g - 1])
    dalt[0] = dalt[1]
    dalt[n - 1] = dalt[n - 2]
    rd = RBODY + alt
    inv_r = 1 / rd
    x = RBODY * inv_r
    grav = -GC * (x * x)
    for g in range(2, n_alts + 2):  # iAlt 1..nAlts (stretched grid)
        y = RBODY / rd[g]
        grav[g] = -GC * (y * y)
    return dalt, inv_r, grav


def producers(nden_s, temperature, vert_vel):
    """Gamma, NDensity, MeanMajorMass, TempUnit, cMax with the reference's
    operation order (calc_pressure.f90:17-21,56-83; calc_rates.Earth.f90:
    34-50; calc_timestep.f90:114-118).  Inputs [6,G,C], [G,C], [6,G,C]."""
    n = np.zeros_like(temperature)
    for s in range(NSPECIES):
        n = n + nden_s[s]
    gm = np.zeros_like(temperature)
    for s in range(NSPECIES):
        gm = gm + nden_s[s] / (VIBRATION[s] - 2)
    gamma = gm * 2.0 / n + 1
    mmm = np.zeros_like(temperature)
    for s in range(NSPECIES):
        mmm = mmm + MASS[s] * nden_s[s] / (n + 1.0)
    mmm = np.where(mmm == 0, MASS[0], mmm)
    temp_unit = mmm / KB
    cmax = np.zeros_like(temperature)
    mx = np.abs(vert_vel[0])
    for s in range(1, NSPECIES):
        mx = np.maximum(mx, np.abs(vert_vel[s]))
    cmax[1:-1] = (mx + np.sqrt(gamma * temperature))[1:-1]
    return gamma, n, mmm, temp_unit, cmax


@dataclasses.dataclass
class Member:
    """One member: n_cols columns sharing nAlts and one altitude grid.
    Field names follow GitmColumnBatch (include/gitm_vert.h)."""

    n_alts: int
    n_cols: int
    ndensity_s: np.ndarray
    idensity_s: np.ndarray
    rho: np.ndarray
    temperature: np.ndarray
    velocity: np.ndarray
    vert_vel: np.ndarray
    gamma: np.ndarray
    mean_major_mass: np.ndarray
    temp_unit: np.ndarray
    cmax: np.ndarray
    ivel_up: np.ndarray
    eddy: np.ndarray
    cos_lat: np.ndarray
    sza: np.ndarray
    mlat: np.ndarray
    altitude: np.ndarray
    gravity: np.ndarray
    dalt_c: np.ndarray
    inv_r: np.ndarray
    lbc: np.ndarray | None = None
    log_ns: np.ndarray | None = None
    ndensity: np.ndarray | None = None
    heating: np.ndarray | None = None
    heating_scale: np.ndarray | None = None

    STATE = ("ndensity_s", "idensity_s", "rho", "temperature", "velocity", "vert_vel")
    COEFFS = ("gamma", "mean_major_mass", "temp_unit", "cmax")
    INPUTS = ("ivel_up", "eddy", "cos_lat", "sza", "mlat", "altitude", "gravity",
              "dalt_c", "inv_r")

    @property
    def G(self) -> int:
        return self.n_alts + 4

    def copy(self) -> "Member":
        kw = {}
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            kw[f.name] = v.copy() if isinstance(v, np.ndarray) else v
        return Member(**kw)

    def arrays(self):
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, np.ndarray):
                yield f.name, v


def smooth_profiles(rng, alt: np.ndarray, n_cols: int, n_modes: int = 6,
                    scale_km: float = 120.0) -> np.ndarray:
    """[G, n_cols] random profiles with unit variance at every altitude and
    a vertical correlation length of about scale_km (a random Fourier series
    in altitude), so winds have the stated N(0, sigma) spread without
    cell-to-cell noise."""
    z = (alt - alt[0])[:, None] / (scale_km * 1000.0)
    out = np.zeros((alt.shape[0], n_cols))
    for k in range(n_modes):
        amp = rng.normal(0.0, 1.0, n_cols)
        ph = rng.uniform(0.0, 2 * math.pi, n_cols)
        kk = rng.uniform(0.5, 2.0, n_cols)
        out += amp[None, :] * np.cos(kk[None, :] * z + ph[None, :])
    return out * math.sqrt(2.0 / n_modes)


def make_member(n_cols: int, n_alts: int = 50, seed: int = 0, tinf_shift: float = 0.0,
                lat_deg: np.ndarray | None = None, with_lbc: bool = False,
                with_outputs: bool = True, with_heating: bool = False) -> Member:
    rng = np.random.Generator(np.random.PCG64(seed))
    G = n_alts + 4
    alt = make_altitude_grid(n_alts)
    dalt, inv_r, grav = grid_geometry(alt)
    z = alt[:, None]  # [G,1]
    tinf = rng.uniform(700.0, 1500.0, n_cols) + tinf_shift
    tinf = np.maximum(tinf, 400.0)
    T = bates_temperature(z, tinf[None, :])  # [G,C]
    g = _gravity(z)
    # diffusive equilibrium from cell 1 (100 km), trapezoid between cells
    n0 = BASE_DENSITY[:, None] * 10.0 ** rng.uniform(-0.3, 0.3, (NSPECIES, n_cols))
    nden = np.zeros((NSPECIES, G, n_cols))
    for s in range(NSPECIES):
        inv_h = MASS[s] * g / (KB * T)  # [G,C]
        seg = 0.5 * (inv_h[1:] + inv_h[:-1]) * np.diff(alt)[:, None]  # [G-1,C]
        integ = np.concatenate([np.zeros((1, n_cols)), np.cumsum(seg, axis=0)], axis=0)
        # T(100 km)/T(z): the thermal-expansion factor that makes the profile
        # hydrostatic for the model's momentum equation when T varies with z
        nden[s] = (n0[s][None, :] * (T[2][None, :] / T)
                   * np.exp(-(integ - integ[2][None, :])))
    # ions: Chapman layers with per-column jitter, floor 1 m^-3
    iden = np.zeros((NIONS, G, n_cols))
    zk = alt / 1000.0
    for i in range(NIONS - 1):
        peak, zp, hh = ION_LAYERS[i]
        pk = peak * 10.0 ** rng.uniform(-0.3, 0.3, n_cols)
        zpk = zp + rng.uniform(-20.0, 20.0, n_cols)
        zeta = (zk[:, None] - zpk[None, :]) / hh
        iden[i] = np.maximum(pk[None, :] * np.exp(0.5 * (1.0 - zeta - np.exp(-zeta))), 1.0)
    iden[NIONS - 1] = iden[: NIONS - 1].sum(0)
    vel = np.stack([50.0 * smooth_profiles(rng, alt, n_cols), 50.0 * smooth_profiles(rng, alt, n_cols),
                    2.0 * smooth_profiles(rng, alt, n_cols)])
    ww = np.stack([smooth_profiles(rng, alt, n_cols) for _ in range(NSPECIES)])
    ivel_up = 20.0 * smooth_profiles(rng, alt, n_cols)[None]

    gamma, ntot, mmm, tu, _ = producers(nden, np.zeros((G, n_cols)), ww)
    temperature = T / tu  # Temperature = T k / m (normalised)
    gamma, ntot, mmm, tu, cmax = producers(nden, temperature, ww)
    rho = np.zeros((G, n_cols))
    for s in range(NSPECIES):
        rho = rho + MASS[s] * nden[s]
    pressure = temperature * rho
    kcoef = EDDY_COEF * np.exp(rng.normal(0.0, 0.3, n_cols))[None, :]
    eddy = np.where(pressure > EDDY_P0, kcoef,
                    np.where(pressure > EDDY_P1,
                             kcoef * (pressure - EDDY_P1) / (EDDY_P0 - EDDY_P1), 0.0))
    if lat_deg is None:
        lat_deg = rng.uniform(-89.0, 89.0, n_cols)
    cos_lat = np.cos(np.asarray(lat_deg, dtype=np.float64) * math.pi / 180.0)
    sza = rng.uniform(0.0, math.pi, n_cols)
    mlat = rng.uniform(-90.0, 90.0, n_cols)
    lbc = None
    if with_lbc:
        # MSIS-like lower-boundary values: the column's own cells -1, 0 perturbed
        lbc = np.zeros((2, 10, n_cols))
        for k in range(2):
            for s in range(NSPECIES):
                lbc[k, s] = np.log(nden[s, k]) + rng.normal(0.0, 0.05, n_cols)
            lbc[k, 6] = T[k] * (1.0 + rng.normal(0.0, 0.02, n_cols))
            lbc[k, 7] = np.log(rho[k])
            lbc[k, 8] = rng.normal(0.0, 10.0, n_cols)
            lbc[k, 9] = rng.normal(0.0, 10.0, n_cols)
    m = Member(
        n_alts=n_alts, n_cols=n_cols,
        ndensity_s=np.ascontiguousarray(nden), idensity_s=np.ascontiguousarray(iden),
        rho=rho[None].copy(), temperature=temperature[None].copy(),
        velocity=np.ascontiguousarray(vel), vert_vel=np.ascontiguousarray(ww),
        gamma=gamma[None].copy(), mean_major_mass=mmm[None].copy(),
        temp_unit=tu[None].copy(), cmax=cmax[None].copy(),
        ivel_up=np.ascontiguousarray(ivel_up), eddy=eddy[None].copy(),
        cos_lat=cos_lat.copy(), sza=sza, mlat=mlat,
        altitude=alt.copy(), gravity=grav.copy(), dalt_c=dalt.copy(), inv_r=inv_r.copy(),
        lbc=lbc,
    )
    if with_outputs:
        m.log_ns = np.zeros((NSPECIES, G, n_cols))
        m.ndensity = np.zeros((1, G, n_cols))
    if with_heating:
        # EUV heating: 1e-8 K/s at 100 km scaled by rho(100 km) / rho(z), in
        # the normalised units of Temperature (K/s / TempUnit), with a
        # lognormal (sigma 0.3) factor per column; a separate random stream
        # keeps the other fields identical with and without heating
        hr = np.random.Generator(np.random.PCG64([seed, 1]))
        m.heating = (1.0e-8 * rho[2][None, :] / rho / tu)[None].copy()
        m.heating_scale = np.exp(hr.normal(0.0, 0.3, n_cols))
    return m


def globe_member(deg_lat: float, deg_lon: float, n_alts: int = 50, seed: int = 0,
                 **kw) -> Member:
    """A whole globe at deg_lat x deg_lon: columns ordered lon fastest."""
    nlat = int(round(180.0 / deg_lat))
    nlon = int(round(360.0 / deg_lon))
    lats = -90.0 + deg_lat * (np.arange(nlat) + 0.5)
    lat = np.repeat(lats, nlon)
    return make_member(nlat * nlon, n_alts=n_alts, seed=seed, lat_deg=lat, **kw)


def to_modvertical(m: Member, params) -> dict:
    """The ModVertical-form arrays advance_vertical builds for each column
    (advance_vertical.f90:90-133), in native layout."""
    G, n = m.G, m.n_cols
    improved = bool(params.use_improved_ion_advection)
    log_ins = np.zeros((NIONS, G, n))
    log_ins[: NIONS - 1] = m.idensity_s[: NIONS - 1] if improved else np.log(m.idensity_s[: NIONS - 1])
    ivel = np.zeros((3, G, n))
    ivel[2] = m.ivel_up[0]
    om = params.omega_body
    return dict(
        n_alts=m.n_alts, n_cols=n,
        log_rho=np.log(m.rho), temp=m.temperature * m.temp_unit, vel_gd=m.velocity.copy(),
        log_ns=np.log(m.ndensity_s), vert_vel=m.vert_vel.copy(), log_ins=log_ins, ivel=ivel,
        cmax=m.cmax.copy(), mean_major_mass=m.mean_major_mass.copy(), gamma=m.gamma.copy(),
        eddy=m.eddy.copy(), centrifugal=(m.cos_lat * om) * (m.cos_lat * om),
        coriolis=2 * m.cos_lat * om, sza=m.sza.copy(), mlat=m.mlat.copy(),
        lbc=None if m.lbc is None else m.lbc.copy(),
        altitude=m.altitude.copy(), gravity=m.gravity.copy(), dalt_c=m.dalt_c.copy(),
        inv_r=m.inv_r.copy(),
    )
