/*
 * gitm_hz.h -- C ABI of the horizontal advance (advance_horizontal) in
 * libgitmvert.so.
 *
 * Replaces advance_horizontal(iBlock) (advance_horizontal.f90:58-924: the
 * RK4 longitude / latitude Rusanov update of Rho, Velocity, Temperature,
 * VerticalVelocity, NDensityS and the advected IDensityS at every altitude,
 * with calc_rusanov_lons / _lats and calc_facevalues_lons / _lats at
 * :821-1034, then the divergence of the parallel ion velocity, :423-517,
 * with UAM_Gradient, gradient.f90:4-104) for every block of a call.  What
 * advance_horizontal_all (:8-49) does around it stays with the caller:
 * exchange_messages_sphere fills the ghost cells before the call, calc_rates
 * and calc_physics run before it, set_horizontal_bcs and the second exchange
 * after it.  UseTopography is not supported (the dVarDAlt terms of
 * calc_rusanov_lons / _lats are absent).
 *
 * Arrays are GITM's own module arrays in their Fortran layout, on the device:
 * the address of the first element and the bounds GITM allocates them with
 * (ModGITM.f90, ModSources.f90), so a GPU-resident GITM passes its arrays
 * without a copy:
 *   "block array"  X(-1:nLons+2, -1:nLats+2, -1:nAlts+2, nBlocks)
 *   "block array [k]"  X(-1:nLons+2, -1:nLats+2, -1:nAlts+2, k, nBlocks)
 * gitm_hz_advance is asynchronous on the stream it is given;
 * gitm_hz_status waits for that stream and reads the status words.
 */
#ifndef GITM_HZ_H
#define GITM_HZ_H

#include <stdint.h>

#include "gitm_vert.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GITM_NSPECIES_TOTAL 11 /* nSpeciesTotal (ModEarth.f90:26): NDensityS's 4th extent */
#define GITM_ST_LOW_TEMPERATURE 64u /* Temperature < 100 after the exchange
                                       exchange_messages_sphere.f90:80-84 */

typedef struct GitmHzParams {
  int32_t use_coriolis;               /* UseCoriolis                          */
  int32_t use_ion_advection;          /* UseIonAdvection                      */
  int32_t use_improved_ion_advection; /* UseImprovedIonAdvection: the parallel
                                         ion-velocity divergence term          */
  int32_t non_magnetic;               /* NonMagnetic: that term uses IVelocity
                                         instead of IVelocityPar               */
  int32_t reserved0;
  double omega_body;                  /* OmegaBodyInput (2 pi / 86400 s)      */
  double beta_limiter;                /* BetaLimiter (2.0) of Limiter_mc      */
} GitmHzParams;

typedef struct GitmHzBlocks {
  int32_t n_lons, n_lats, n_alts, n_blocks;
  /* state: ghost cells read, interior cells (1..nLons, 1..nLats, 1..nAlts)
   * written; IDensityS's electron slot is rewritten as the sum of the ions
   * (with the divergence term: on every cell, ghost cells included) */
  double* rho;            /* Rho                  block array            */
  double* temperature;    /* Temperature          block array            */
  double* velocity;       /* Velocity             block array [3]        */
  double* vert_vel;       /* VerticalVelocity     block array [nSpecies] */
  double* ndensity_s;     /* NDensityS            block array [nSpeciesTotal] */
  double* idensity_s;     /* IDensityS            block array [nIons]    */
  double* temp_source;    /* HorizontalTempSource (1:nLons,1:nLats,1:nAlts,nBlocks),
                             NewTemp - Temperature; may be NULL          */
  /* read */
  const double* gamma;    /* Gamma                block array            */
  const double* cmax;     /* cMax_GDB(0:nLons+1, 0:nLats+1, 0:nAlts+1, 3, nBlocks)
                             (ModGITM.f90:250: one ghost cell, not two) */
  const double* ivelocity;      /* IVelocity      block array [3]        */
  const double* ivelocity_par;  /* IVelocityPar   block array [3] (NULL when
                                   non_magnetic or without the divergence) */
  const double* latitude;       /* Latitude(-1:nLats+2, nBlocks)           */
  const double* tan_latitude;   /* TanLatitude(-1:nLats+2, nBlocks)        */
  const double* cos_latitude;   /* CosLatitude(-1:nLats+2, nBlocks)        */
  const double* radial_distance;     /* RadialDistance_GB    block array  */
  const double* inv_radial_distance; /* InvRadialDistance_GB block array  */
  const double* inv_dlon_dist_gb;    /* InvDLonDist_GB       block array  */
  const double* inv_dlon_dist_fb;    /* InvDLonDist_FB       block array  */
  const double* dlon_dist_fb;        /* dLonDist_FB          block array  */
  const double* inv_dlat_dist_gb;    /* InvDLatDist_GB       block array  */
  const double* inv_dlat_dist_fb;    /* InvDLatDist_FB       block array  */
  const double* dlat_dist_fb;        /* dLatDist_FB          block array  */
  const double* grad_lon_m, *grad_lon_0, *grad_lon_p; /* GradLon{M,0,P}_CB(nLons, nBlocks) */
  const double* grad_lat_m, *grad_lat_0, *grad_lat_p; /* GradLat{M,0,P}_CB(nLats, nBlocks) */
} GitmHzBlocks;

/*
 * One advance_horizontal(iBlock) for every block, on `stream` (a
 * cudaStream_t; NULL = the default stream) of gitm_vert_create's context
 * (its GitmVertParams are not used).  n_lons and
 * n_lats <= 32, n_alts <= GITM_MAX_NALTS.  A block whose new neutral
 * densities go negative (the reference stops there) sets
 * GITM_ST_NEG_DENSITY in its status word; its arrays are then undefined.
 * Replaces advance_horizontal.f90:58-924 for each block.
 */
int gitm_hz_advance(GitmVertCtx* ctx, const GitmHzParams* params, const GitmHzBlocks* blocks, double dt,
                    void* stream);

/*
 * The ghost cells of a whole sphere of blocks (exchange_messages_sphere,
 * exchange_messages_sphere.f90:4-95, with the transfer of
 * ModSphereInterface.f90:395-513 and srcSphereAB's multi-block packers,
 * AB_XFER_array_util.f90, over the neighbours of AB_SPH_module.f90:
 * 180-370).  Blocks tile the sphere as block = iLat * n_blocks_lon + iLon
 * (0-based), south to north.  Every ghost cell of the two-cell ring at
 * altitudes 1..nAlts takes the value of the interior cell it covers:
 * longitude periodic, and across a connected pole the cell mirrored in
 * latitude n_blocks_lon / 2 blocks away in longitude; then the east and
 * north components of Velocity and of IVelocity / IVelocityPar are negated
 * in the ghost rows beyond a pole (every longitude and altitude, as the
 * reference does), and a block whose interior Temperature drops below 100
 * or Rho below 0 gets GITM_ST_LOW_TEMPERATURE / GITM_ST_NEG_DENSITY
 * (the reference stops).  n_blocks_lon must be even when a pole is
 * connected (the corner neighbours across the pole pair up only then), and
 * blocks hold 2 x 2 cells or more.
 */
typedef struct GitmHzExchange {
  int32_t n_lons, n_lats, n_alts, n_blocks_lon, n_blocks_lat;
  int32_t north_pole, south_pole;    /* connect across the poles (IsFullSphere: both) */
  int32_t use_ion_advection;         /* UseIonAdvection: IDensityS and the ion velocity move too */
  int32_t non_magnetic;              /* NonMagnetic: IVelocity instead of IVelocityPar */
  int32_t reserved0;
  double* rho;            /* Rho                      block array            */
  double* temperature;    /* Temperature              block array            */
  double* itemperature;   /* ITemperature             block array (may be NULL) */
  double* etemperature;   /* eTemperature             block array (may be NULL) */
  double* velocity;       /* Velocity                 block array [3]        */
  double* vert_vel;       /* VerticalVelocity         block array [nSpecies] */
  double* ndensity_s;     /* NDensityS                block array [nSpeciesTotal] */
  double* idensity_s;     /* IDensityS                block array [nIons]    */
  double* ivelocity;      /* IVelocity                block array [3]        */
  double* ivelocity_par;  /* IVelocityPar             block array [3]        */
  const double* latitude; /* Latitude(-1:nLats+2, nBlocks)                   */
} GitmHzExchange;

/* exchange_messages_sphere on device arrays, on `stream`; the status words
 * (one per block) are read with gitm_hz_status.  Replaces
 * exchange_messages_sphere.f90:4-95 for a single-process sphere. */
int gitm_hz_exchange(GitmVertCtx* ctx, const GitmHzExchange* x, void* stream);

/* Status words of the last gitm_hz_advance or gitm_hz_exchange, one per block: OR of all into
 * *or_out and the count of nonzero words into *n_bad (either may be NULL);
 * clear = 1 zeroes them.  Waits for the stream of the last call. */
int gitm_hz_status(GitmVertCtx* ctx, uint32_t* or_out, int64_t* n_bad, int clear);

#ifdef __cplusplus
}
#endif

#endif /* GITM_HZ_H */
