"""ctypes mirrors of the structs in include/gitm_vert.h.

The field order and types must match the C header exactly; the C-ABI test in
tests/ checks the sizes against the library's own ``sizeof`` report.
"""
from __future__ import annotations

import ctypes as C

NSPECIES = 6
NIONS = 10
NIONS_ADVECT = 2
MAX_NALTS = 128
LBC_NVALUES = 10

OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_NOMEM = -3
ERR_COLUMN = -4
ERR_TIMEOUT = -5
ERR_UNSUPPORTED = -6

ST_NEG_DENSITY = 1
ST_NEG_ION_TOP = 2
ST_LU_SINGULAR = 4
ST_NONFINITE = 8
ST_BAD_NALTS = 16
ST_ADJ_BRANCH = 32
ST_LOW_TEMPERATURE = 64  # the horizontal exchange's Temperature < 100 check

SOLVER_RUSANOV = 0
SOLVER_AUSM = 1

_dp = C.POINTER(C.c_double)


class GitmVertParams(C.Structure):
    _fields_ = [
        ("solver", C.c_int32),
        ("use_neutral_friction", C.c_int32),
        ("use_coriolis", C.c_int32),
        ("use_ion_advection", C.c_int32),
        ("use_improved_ion_advection", C.c_int32),
        ("use_nighttime_ion_bcs", C.c_int32),
        ("use_damping", C.c_int32),
        ("use_msis_bcs", C.c_int32),
        ("compute_coefficients", C.c_int32),
        ("compute_eddy", C.c_int32),
        ("beta_limiter", C.c_double),
        ("max_vertical_velocity", C.c_double),
        ("min_tec", C.c_double),
        ("omega_body", C.c_double),
        ("vert_tau", C.c_double),
        ("thermal_diff_coef", C.c_double * NSPECIES),
        ("eddy_coef", C.c_double),
        ("eddy_pressure0", C.c_double),
        ("eddy_pressure1", C.c_double),
    ]


def default_params(**overrides) -> GitmVertParams:
    """Reference defaults (ModInputs.f90, ModEarth.f90:325, calc_rates.Earth.f90:83-84)."""
    import math

    p = GitmVertParams()
    p.solver = SOLVER_RUSANOV
    p.use_neutral_friction = 1
    p.use_coriolis = 1
    p.use_ion_advection = 1
    p.use_improved_ion_advection = 1
    p.use_nighttime_ion_bcs = 1
    p.use_damping = 0
    p.use_msis_bcs = 0
    p.compute_coefficients = 1
    p.beta_limiter = 2.0
    p.max_vertical_velocity = 1000.0
    p.min_tec = 2.0
    p.omega_body = 2.0 * 3.141592653589793 / (24.0 * 3600.0)
    p.vert_tau = 1.0e9
    for i in range(NSPECIES):
        p.thermal_diff_coef[i] = 0.0
    p.thermal_diff_coef[5] = -0.38
    p.compute_eddy = 0
    p.eddy_coef = 50.0        # EddyDiffusionCoef, ModInputs.f90:302
    p.eddy_pressure0 = 0.01   # EddyDiffusionPressure0 (Pa), :303
    p.eddy_pressure1 = 0.005  # EddyDiffusionPressure1 (Pa), :304
    for k, v in overrides.items():
        if k == "thermal_diff_coef":
            for i in range(NSPECIES):
                p.thermal_diff_coef[i] = v[i]
        else:
            setattr(p, k, v)
    return p


class GitmColumnBatch(C.Structure):
    _fields_ = [
        ("n_alts", C.c_int32),
        ("grid_per_column", C.c_int32),
        ("n_cols", C.c_int64),
        ("ndensity_s", _dp),
        ("idensity_s", _dp),
        ("rho", _dp),
        ("temperature", _dp),
        ("velocity", _dp),
        ("vert_vel", _dp),
        ("log_ns", _dp),
        ("ndensity", _dp),
        ("gamma", _dp),
        ("mean_major_mass", _dp),
        ("temp_unit", _dp),
        ("cmax", _dp),
        ("ivel_up", _dp),
        ("eddy", _dp),
        ("cos_lat", _dp),
        ("sza", _dp),
        ("mlat", _dp),
        ("lbc", _dp),
        ("altitude", _dp),
        ("gravity", _dp),
        ("dalt_c", _dp),
        ("inv_r", _dp),
        ("heating", _dp),
        ("heating_scale", _dp),
    ]


class GitmColumnAdjoint(C.Structure):
    _fields_ = [
        ("ndensity_s", _dp),
        ("idensity_s", _dp),
        ("rho", _dp),
        ("temperature", _dp),
        ("velocity", _dp),
        ("vert_vel", _dp),
        ("log_ns", _dp),
        ("ndensity", _dp),
        ("eddy", _dp),
        ("heating_scale", _dp),
    ]


class GitmModVerticalBatch(C.Structure):
    _fields_ = [
        ("n_alts", C.c_int32),
        ("grid_per_column", C.c_int32),
        ("n_cols", C.c_int64),
        ("log_rho", _dp),
        ("temp", _dp),
        ("vel_gd", _dp),
        ("log_ns", _dp),
        ("vert_vel", _dp),
        ("log_ins", _dp),
        ("ivel", _dp),
        ("cmax", _dp),
        ("mean_major_mass", _dp),
        ("gamma", _dp),
        ("eddy", _dp),
        ("centrifugal", _dp),
        ("coriolis", _dp),
        ("sza", _dp),
        ("mlat", _dp),
        ("lbc", _dp),
        ("altitude", _dp),
        ("gravity", _dp),
        ("dalt_c", _dp),
        ("inv_r", _dp),
    ]


class GitmLaunchConfig(C.Structure):
    _fields_ = [
        ("threads", C.c_int32),
        ("cols_per_cta", C.c_int32),
        ("steps_per_launch", C.c_int32),
        ("ctas_per_sm", C.c_int32),
    ]


class GitmFArray(C.Structure):
    _fields_ = [
        ("data", _dp),
        ("stride", C.c_int64 * 5),
        ("lower", C.c_int32 * 5),
    ]


FORTRAN_ARRAYS = (
    "ndensity_s", "idensity_s", "rho", "temperature", "velocity", "ivelocity",
    "vertical_velocity", "log_ns", "ndensity", "species_density",
    "species_density_old", "gamma", "mean_major_mass", "temp_unit", "cmax",
    "kappa_eddy", "altitude", "gravity", "dalt", "inv_r", "cos_latitude", "sza",
    "mlatitude",
)


class GitmFortranState(C.Structure):
    _fields_ = [
        ("n_lons", C.c_int32),
        ("n_lats", C.c_int32),
        ("n_alts", C.c_int32),
        ("n_blocks", C.c_int32),
    ] + [(name, GitmFArray) for name in FORTRAN_ARRAYS]


NSPECIES_TOTAL = 11  # GITM_NSPECIES_TOTAL: NDensityS's species extent

HZ_BLOCK_FIELDS = ("rho", "temperature", "velocity", "vert_vel", "ndensity_s", "idensity_s", "temp_source",
                   "gamma", "cmax", "ivelocity", "ivelocity_par", "latitude", "tan_latitude", "cos_latitude",
                   "radial_distance", "inv_radial_distance", "inv_dlon_dist_gb", "inv_dlon_dist_fb",
                   "dlon_dist_fb", "inv_dlat_dist_gb", "inv_dlat_dist_fb", "dlat_dist_fb", "grad_lon_m",
                   "grad_lon_0", "grad_lon_p", "grad_lat_m", "grad_lat_0", "grad_lat_p")


class GitmHzParams(C.Structure):
    _fields_ = [
        ("use_coriolis", C.c_int32),
        ("use_ion_advection", C.c_int32),
        ("use_improved_ion_advection", C.c_int32),
        ("non_magnetic", C.c_int32),
        ("reserved0", C.c_int32),
        ("omega_body", C.c_double),
        ("beta_limiter", C.c_double),
    ]


def default_hz_params(**overrides) -> GitmHzParams:
    """Reference defaults (ModInputs.f90: UseCoriolis, UseIonAdvection,
    UseImprovedIonAdvection true; BetaLimiter 2; OmegaBodyInput 2 pi / day);
    Earth is magnetic (NonMagnetic false)."""
    p = GitmHzParams()
    p.use_coriolis = 1
    p.use_ion_advection = 1
    p.use_improved_ion_advection = 1
    p.non_magnetic = 0
    p.omega_body = 2.0 * 3.141592653589793 / (24.0 * 3600.0)
    p.beta_limiter = 2.0
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


class GitmHzBlocks(C.Structure):
    _fields_ = [("n_lons", C.c_int32), ("n_lats", C.c_int32), ("n_alts", C.c_int32), ("n_blocks", C.c_int32)] + \
        [(name, _dp) for name in HZ_BLOCK_FIELDS]


HZ_EXCHANGE_FIELDS = ("rho", "temperature", "itemperature", "etemperature", "velocity", "vert_vel", "ndensity_s",
                      "idensity_s", "ivelocity", "ivelocity_par", "latitude")


class GitmHzExchange(C.Structure):
    _fields_ = [("n_lons", C.c_int32), ("n_lats", C.c_int32), ("n_alts", C.c_int32), ("n_blocks_lon", C.c_int32),
                ("n_blocks_lat", C.c_int32), ("north_pole", C.c_int32), ("south_pole", C.c_int32),
                ("use_ion_advection", C.c_int32), ("non_magnetic", C.c_int32), ("reserved0", C.c_int32)] + \
        [(name, _dp) for name in HZ_EXCHANGE_FIELDS]


def dptr(addr: int):
    """A ctypes double* from an integer address (0 -> NULL)."""
    return C.cast(C.c_void_p(addr), _dp) if addr else _dp()
