/*
 * gitm_vert.h -- C ABI of the B200 implementation of GITM's vertical advance.
 *
 * The reference has no plugin API for this path: the Fortran host calls
 *   advance_vertical_all()                     src/advance_vertical.f90:8-39
 *   advance_vertical(iLon, iLat, iBlock)       src/advance_vertical.f90:45-219
 *   advance_vertical_1d_rusanov()              src/vertical_solver_rusanov.f90:10-384
 *   advance_vertical_1d_ausm()                 src/vertical_solver_ausm.f90:26-433
 *   calc_timestep_vertical()                   src/calc_timestep.f90:85-157
 * with every input and output passed through Fortran modules (ModGITM,
 * ModVertical, ModInputs, ModPlanet, ModSources).  The entry points below take
 * those module variables as explicit arguments.  All arithmetic is IEEE FP64.
 *
 * Conventions
 *   - Altitude cells run over the reference's -1 .. nAlts+2 (G = nAlts + 4
 *     cells); cell index g = iAlt + 1.
 *   - "Native layout": one array per variable, element (field f, cell g,
 *     column c) at  p[(f * G + g) * n_cols + c]  -- the column index is the
 *     fastest-varying dimension, so every altitude stencil is a coalesced
 *     row access.
 *   - Every function returns GITM_OK (0) or a negative GITM_ERR_* code and
 *     never aborts the process; the message is in gitm_vert_last_error().
 *   - Per-column numerical failures that make the reference call stop_gitm
 *     (src/library.f90:33-51) are reported as GITM_ST_* bits in a per-column
 *     status word instead; a call that finds any returns GITM_ERR_COLUMN.
 *   - Functions taking a `stream` argument are asynchronous on that CUDA
 *     stream (NULL = legacy default stream) unless stated otherwise.
 */
#ifndef GITM_VERT_H
#define GITM_VERT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Earth species table sizes (src/ModEarth.f90:12-40). */
#define GITM_NSPECIES 6      /* O(3P), O2, N2, N(4S), NO, He               */
#define GITM_NIONS 10        /* 9 ions + electrons (ie_ = 10)              */
#define GITM_NIONS_ADVECT 2  /* nIonsAdvect                                */
#define GITM_MAX_NALTS 128   /* largest nAlts a launch accepts             */
#define GITM_LBC_NVALUES 10  /* MSIS lower-boundary table: LogNS(6), Temp,
                                LogRho, Vel east, Vel north                */

/* Return codes. */
#define GITM_OK 0
#define GITM_ERR_ARG (-1)        /* bad argument (null pointer, bad size)   */
#define GITM_ERR_CUDA (-2)       /* a CUDA runtime call failed              */
#define GITM_ERR_NOMEM (-3)      /* device allocation failed                */
#define GITM_ERR_COLUMN (-4)     /* at least one column set a GITM_ST_ bit  */
#define GITM_ERR_TIMEOUT (-5)    /* the host watchdog gave up waiting       */
#define GITM_ERR_UNSUPPORTED (-6)

/* Per-column status bits (reference stop_gitm triggers). */
#define GITM_ST_NEG_DENSITY 1u  /* minval(NDensityS) <= 0  advance_vertical.f90:96-100 */
#define GITM_ST_NEG_ION_TOP 2u  /* negative ion next to top set_vertical_bcs.Earth.f90:617-620 */
#define GITM_ST_LU_SINGULAR 4u  /* zero row / pivot       ludcmp.f:11-14 */
#define GITM_ST_NONFINITE 8u    /* NaN/Inf in the result  check_for_nans.f90:4-139 */
#define GITM_ST_BAD_NALTS 16u   /* member nAlts out of range for the launch */
#define GITM_ST_ADJ_BRANCH 32u  /* the adjoint met a branch it does not
                                   differentiate (negative ions next to the
                                   top, set_vertical_bcs.Earth.f90:608-649);
                                   that column's gradient is not valid      */

/* Solver selection (ModInputs.f90:242 UseAUSMSolver). */
#define GITM_SOLVER_RUSANOV 0
#define GITM_SOLVER_AUSM 1

/*
 * Run-time flags and parameters of the path.  Field names follow ModInputs /
 * ModPlanet; gitm_vert_default_params() fills the reference defaults.
 */
typedef struct GitmVertParams {
  int32_t solver;                     /* UseAUSMSolver ? AUSM : Rusanov       */
  int32_t use_neutral_friction;       /* UseNeutralFriction  (T)  ModInputs.f90:240 */
  int32_t use_coriolis;               /* UseCoriolis         (T)  ModInputs.f90:235 */
  int32_t use_ion_advection;          /* UseIonAdvection     (T)  ModInputs.f90:311 */
  int32_t use_improved_ion_advection; /* UseImprovedIonAdvection (T) ModInputs.f90:259 */
  int32_t use_nighttime_ion_bcs;      /* UseNighttimeIonBCs  (T)  ModInputs.f90:260 */
  int32_t use_damping;                /* UseDamping          (F)  ModInputs.f90:221 */
  int32_t use_msis_bcs;               /* UseMSIS (T in GITM); 1 = take the lower
                                         boundary from GitmColumnBatch.lbc    */
  int32_t compute_coefficients;       /* 1 = recompute Gamma, NDensity,
                                         MeanMajorMass, TempUnit and cMax from
                                         the state before each step
                                         (calc_pressure.f90:56-83,
                                          calc_rates.Earth.f90:34-50,
                                          calc_timestep.f90:109-118); 0 = use the
                                         arrays the caller passes            */
  int32_t compute_eddy;               /* 1 = after each step, KappaEddyDiffusion
                                         (GitmColumnBatch.eddy, cells 1..nAlts)
                                         is recomputed from Pressure =
                                         Temperature * Rho of the state the step
                                         started from, as calc_sources does
                                         (calc_sources.f90:26, Earth.f90:376-411,
                                         calc_pressure.f90:23): the next step
                                         uses it.  GITM-array form only; the
                                         adjoint takes the eddy coefficient as
                                         an input and refuses this mode.      */
  double beta_limiter;                /* BetaLimiter (2.0)  ModInputs.f90:104 */
  double max_vertical_velocity;       /* MaximumVerticalVelocity (1000) ModInputs.f90:224 */
  double min_tec;                     /* MinTEC (2.0)        ModInputs.f90:261 */
  double omega_body;                  /* OmegaBodyInput (2 pi / 86400 s) ModInputs.f90:285 */
  double vert_tau;                    /* VertTau (1e9 s)     ModEarth.f90:325 */
  double thermal_diff_coef[GITM_NSPECIES]; /* ThermalDiffCoefS calc_rates.Earth.f90:83-84 */
  double eddy_coef;                   /* EddyDiffusionCoef (50 m^2/s)  ModInputs.f90:302 */
  double eddy_pressure0;              /* EddyDiffusionPressure0 (0.01 Pa)  ModInputs.f90:303 */
  double eddy_pressure1;              /* EddyDiffusionPressure1 (0.005 Pa) ModInputs.f90:304 */
} GitmVertParams;

/*
 * One member of a batch: n_cols columns that share nAlts and (unless
 * grid_per_column) one altitude grid.  Pointers are DEVICE pointers for the
 * plan API and HOST pointers for gitm_vert_advance_native_host().  All state
 * arrays are updated in place.  Arrays marked [f] hold f fields.
 *
 * Inputs/outputs (advance_vertical.f90:80-217 reads and writes these):
 *   ndensity_s [6]  NDensityS          idensity_s [10] IDensityS (slot 10 = e-)
 *   rho             Rho                temperature     Temperature (T k / m)
 *   velocity   [3]  Velocity (E,N,Up)  vert_vel   [6]  VerticalVelocity
 * Optional outputs (may be NULL):
 *   log_ns     [6]  LogNS              ndensity        NDensity
 * Coefficients, one field each (read; written when compute_coefficients=1,
 * in which case they may be NULL):
 *   gamma (Gamma), mean_major_mass (MeanMajorMass), temp_unit (TempUnit),
 *   cmax (cMax_GDB(:,:,:,iUp_); cells 0..nAlts+1 are used)
 * Inputs (read-only unless noted):
 *   ivel_up         IVelocity(:,:,:,iUp_)
 *   eddy            KappaEddyDiffusion (cells 1..nAlts are used; written
 *                   when compute_eddy = 1)
 *   cos_lat, sza, mlat  [n_cols]  CosLatitude, SZA (rad), MLatitude(nAlts) (deg)
 *   lbc  [2][10][n_cols] or NULL: lower boundary values for cells -1 and 0
 *        (the MSIS call of set_vertical_bcs.Earth.f90:112-137)
 *   altitude, gravity, dalt_c, inv_r: Altitude_GB, Gravity_GB, dAlt_GB,
 *        InvRadialDistance_GB -- [G] when grid_per_column = 0, [G][n_cols]
 *        when grid_per_column = 1.
 * Optional heating update after each step (may be NULL):
 *   heating         EuvHeating (normalised K/s, cells 1..nAlts are used)
 *   heating_scale   [n_cols] factor on heating per column (NULL = 1)
 *   With heating set, every step ends with the temperature line of
 *   add_sources (add_sources.f90:53-66) with EuvHeating as its only nonzero
 *   term: Temperature(1:nAlts) += dt * heating_scale * heating.
 */
typedef struct GitmColumnBatch {
  int32_t n_alts;
  int32_t grid_per_column;
  int64_t n_cols;
  double* ndensity_s;
  double* idensity_s;
  double* rho;
  double* temperature;
  double* velocity;
  double* vert_vel;
  double* log_ns;
  double* ndensity;
  double* gamma;
  double* mean_major_mass;
  double* temp_unit;
  double* cmax;
  const double* ivel_up;
  double* eddy;
  const double* cos_lat;
  const double* sza;
  const double* mlat;
  const double* lbc;
  const double* altitude;
  const double* gravity;
  const double* dalt_c;
  const double* inv_r;
  const double* heating;
  const double* heating_scale;
} GitmColumnBatch;

/*
 * ModVertical-form columns (the arguments of advance_vertical_1d_rusanov /
 * _ausm, ModVertical.f90:15-48), native layout, updated in place:
 *   log_rho, temp (Temp in K), vel_gd [3], log_ns [6], vert_vel [6],
 *   log_ins [10] (slot 10 is never read; it is left as passed), ivel [3] (read),
 *   cmax, mean_major_mass, gamma, eddy (read), centrifugal, coriolis,
 *   sza, mlat [n_cols] (read), grid as in GitmColumnBatch.
 */
typedef struct GitmModVerticalBatch {
  int32_t n_alts;
  int32_t grid_per_column;
  int64_t n_cols;
  double* log_rho;
  double* temp;
  double* vel_gd;
  double* log_ns;
  double* vert_vel;
  double* log_ins;
  const double* ivel;
  const double* cmax;
  const double* mean_major_mass;
  const double* gamma;
  const double* eddy;
  const double* centrifugal;
  const double* coriolis;
  const double* sza;
  const double* mlat;
  const double* lbc;
  const double* altitude;
  const double* gravity;
  const double* dalt_c;
  const double* inv_r;
} GitmModVerticalBatch;

typedef struct GitmVertCtx GitmVertCtx;
typedef struct GitmVertPlan GitmVertPlan;

/* Launch shape of the fused step kernel (chosen by the autotuner). */
typedef struct GitmLaunchConfig {
  int32_t threads;          /* threads per CTA (multiple of 32)            */
  int32_t cols_per_cta;     /* columns held by one CTA (0 = as many as fit) */
  int32_t steps_per_launch; /* RK4 steps a column tile runs while resident  */
  int32_t ctas_per_sm;      /* persistent grid = ctas_per_sm x SMs (0 = one
                               CTA per tile, no persistence)               */
} GitmLaunchConfig;

/* ---- library / context ------------------------------------------------ */

const char* gitm_vert_version(void);
void gitm_vert_default_params(GitmVertParams* params);

/* Creates a context on CUDA device `device`.  Replaces the module set-up that
 * the reference does in init_planet / set_inputs (ModEarth.f90:265-338). */
int gitm_vert_create(const GitmVertParams* params, int device, GitmVertCtx** ctx);
int gitm_vert_destroy(GitmVertCtx* ctx);
const char* gitm_vert_last_error(const GitmVertCtx* ctx);
int gitm_vert_set_params(GitmVertCtx* ctx, const GitmVertParams* params);

/* ---- batched native-layout path (device pointers) --------------------- */

/* Uploads the member table and the per-grid mesh coefficients once; a plan
 * can then be advanced repeatedly, including inside a CUDA graph capture.
 * Replaces the column loop advance_vertical.f90:20-29 for all members. */
int gitm_vert_plan_create(GitmVertCtx* ctx, const GitmColumnBatch* members,
                          int n_members, GitmVertPlan** plan);
int gitm_vert_plan_destroy(GitmVertPlan* plan);
int gitm_vert_plan_set_config(GitmVertPlan* plan, const GitmLaunchConfig* cfg);
int gitm_vert_plan_get_config(const GitmVertPlan* plan, GitmLaunchConfig* cfg);
/* Runs n_steps RK4 steps of dt seconds (Dt in ModGITM) on every column.
 * Asynchronous; only kernel launches are issued, so it can be captured. */
int gitm_vert_plan_advance(GitmVertPlan* plan, double dt, int n_steps, void* stream);
/* Times candidate launch shapes (every built CTA size, 1, n_steps / 2 and
 * n_steps steps per launch, persistent grids of 0-3 CTAs per SM) over
 * n_steps steps on a scratch copy of the state and keeps the
 * fastest; the plan's state is not modified.  Synchronous. */
int gitm_vert_plan_autotune(GitmVertPlan* plan, double dt, int n_steps,
                            GitmLaunchConfig* chosen);
/* Synchronises, ORs every column's status word into *status_or and counts
 * the columns with a nonzero word; clears the words when `clear`. */
int gitm_vert_plan_status(GitmVertPlan* plan, uint32_t* status_or,
                          int64_t* n_bad, int clear);
/* Per-column status words, device array in member order (n_cols total). */
uint32_t* gitm_vert_plan_status_words(GitmVertPlan* plan);
/* Host watchdog, no counterpart in the reference: waits until the work
 * issued on `stream` so far has finished, polling an event, and returns
 * GITM_ERR_TIMEOUT when timeout_s passes first.  The work in flight still
 * completes; the context stays usable.  timeout_s = 0 only asks whether the
 * stream is idle. */
int gitm_vert_plan_wait(GitmVertPlan* plan, void* stream, double timeout_s);
/* Number of kernel launches one gitm_vert_plan_advance(.., n_steps, ..) issues. */
int gitm_vert_plan_launch_count(const GitmVertPlan* plan, int n_steps);

/* One-shot form of the plan API (the plain per-call drop-in): builds a plan,
 * advances, synchronises, reads the status and frees the plan.  Device
 * pointers; synchronous. */
int gitm_vert_advance_native(GitmVertCtx* ctx, const GitmColumnBatch* members,
                             int n_members, double dt, int n_steps);

/* Same with HOST pointers: copies every array of every member to the device,
 * advances and copies the state (and the optional outputs) back.  The copies
 * are chunked over columns and overlapped with the step kernels.
 * Synchronous. */
int gitm_vert_advance_native_host(GitmVertCtx* ctx, const GitmColumnBatch* members,
                                  int n_members, double dt, int n_steps);

/* No counterpart in the reference.  n_steps RK4 steps of one member, like
 * the plan API, but allocating no device memory: for callers that cannot
 * allocate while they run -- a host whose GPU memory is held by its own pool,
 * and per-step loops that must not pay an allocation's device
 * synchronisation.  Device pointers only (host arrays are refused with
 * GITM_ERR_ARG); asynchronous on `stream`.
 *   - The member descriptor, tile list, grid coefficients and RK
 *     accumulators live in one file-scope device array of 12.3 MiB that every
 *     GPU loading the library holds until the process exits;
 *     gitm_vert_create looks up its device address.
 *   - Limits: n_cols <= 262144 and one altitude grid per member
 *     (grid_per_column = 0); larger or per-column-grid members are rejected
 *     with GITM_ERR_ARG.
 *   - Every call reuses the array, so calls that overlap on the GPU race:
 *     issue them in order (one stream, or synchronise between streams).
 *   - status_words (device, n_cols words) are zeroed and then receive each
 *     column's GITM_ST_ bits; read them after the stream completes. */
int gitm_vert_advance_native_noalloc(GitmVertCtx* ctx, const GitmColumnBatch* member,
                                     double dt, int n_steps, uint32_t* status_words,
                                     void* stream);

/* ---- ModVertical-form path --------------------------------------------- */

/* One RK4 step of advance_vertical_1d_rusanov / _ausm (chosen by
 * params.solver) on ModVertical-form columns (device pointers).  Synchronous.
 * Replaces vertical_solver_rusanov.f90:10-384 / vertical_solver_ausm.f90:26-433. */
int gitm_vert_advance_1d(GitmVertCtx* ctx, const GitmModVerticalBatch* batch,
                         double dt, uint32_t* status_words_device);

/* ---- CFL time step ------------------------------------------------------ */

/* calc_timestep_vertical (calc_timestep.f90:85-157) over all members: writes
 * cMax(0:nAlts+1) for every column and returns min(dt_in, CFL-limited dt,
 * dt_end) in *dt_out.  The reference's MPI_Allreduce(MIN) becomes an
 * on-device reduction.  Device pointers; synchronous. */
int gitm_vert_cfl_dt(GitmVertCtx* ctx, const GitmColumnBatch* members,
                     int n_members, double cfl, double dt_in, double dt_end,
                     double* dt_out);

/* ---- Fortran-layout drop-in -------------------------------------------- */

/* A Fortran array section: element (iLon, iLat, iAlt, iField, iBlock) sits at
 * data + sum_d (index_d - lower[d]) * stride[d]  (strides in elements;
 * stride 0 for a dimension the array does not have). */
typedef struct GitmFArray {
  double* data;
  int64_t stride[5];
  int32_t lower[5];
} GitmFArray;

/* The ModGITM / ModSources / ModEUV arrays advance_vertical touches
 * (ModGITM.f90:51-119, allocated ModGITM.f90:188-260). */
typedef struct GitmFortranState {
  int32_t n_lons, n_lats, n_alts, n_blocks;
  GitmFArray ndensity_s, idensity_s, rho, temperature, velocity, ivelocity,
      vertical_velocity, log_ns, ndensity, species_density,
      species_density_old, gamma, mean_major_mass, temp_unit, cmax,
      kappa_eddy, altitude, gravity, dalt, inv_r, cos_latitude, sza,
      mlatitude;
} GitmFortranState;

/* advance_vertical for every (iLon, iLat) of blocks block_first..block_last
 * (1-based, inclusive): gathers the columns, runs the step, and scatters
 * every array advance_vertical.f90:152-217 writes.  `on_device` = 1 when the
 * GitmFArray pointers are device pointers, 0 for host memory (copied in and
 * out).  Synchronous.  Replaces advance_vertical.f90:25-27. */
int gitm_vert_advance_fortran(GitmVertCtx* ctx, const GitmFortranState* st,
                              int block_first, int block_last, double dt,
                              int on_device);

/* ---- adjoint ------------------------------------------------------------
 * No counterpart in the reference (GITM has no adjoint): the reverse-mode
 * derivative of one step of gitm_vert_plan_advance, for gradients of
 * rollouts.  Adjoint arrays have the layout of the GitmColumnBatch field of
 * the same name.  On entry the state arrays hold ybar, the adjoint of the
 * step's outputs; on return they hold xbar, the adjoint of the step's inputs
 * (the plan's member arrays, which must hold the step's INPUT state; they are
 * not modified).  log_ns and ndensity (may be NULL) are the adjoints of those
 * optional outputs.  eddy and heating_scale (may be NULL) accumulate the
 * adjoints of KappaEddyDiffusion and of the per-column heating factor.
 * Branches (limiter cases, clamps, boundary switches, max of |w|) are
 * differentiated on the side the step took; the electron slot of
 * idensity_s is not an input of the step (its xbar is 0). */
typedef struct GitmColumnAdjoint {
  double* ndensity_s;
  double* idensity_s;
  double* rho;
  double* temperature;
  double* velocity;
  double* vert_vel;
  const double* log_ns;
  const double* ndensity;
  double* eddy;
  double* heating_scale;
} GitmColumnAdjoint;

/* The adjoint of one step of every member of the plan (one GitmColumnAdjoint
 * per member, device pointers).  Supported: GITM-array plans, the Rusanov
 * solver.  Columns whose step met GITM_ST_ADJ_BRANCH set that bit in the
 * plan's status words.  saved_states: the states gitm_vert_plan_advance_saving
 * wrote for this step, or NULL to recompute them inside the adjoint kernel.
 * Asynchronous on `stream` (the descriptors are read before the call
 * returns). */
int gitm_vert_plan_adjoint(GitmVertPlan* plan, const GitmColumnAdjoint* bars, double dt,
                           const double* saved_states, void* stream);

/* Doubles of the device buffer one gitm_vert_plan_advance_saving call fills
 * (the gathered state and the five post-boundary stage states of every
 * column). */
int64_t gitm_vert_plan_saved_state_doubles(const GitmVertPlan* plan);

/* One step of gitm_vert_plan_advance (GITM-array plan, Rusanov) that also
 * writes the step's stage states to `states` (device, the size above) for a
 * later gitm_vert_plan_adjoint of the same step.  Asynchronous on `stream`. */
int gitm_vert_plan_advance_saving(GitmVertPlan* plan, double dt, double* states, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GITM_VERT_H */
