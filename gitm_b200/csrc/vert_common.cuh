// vert_common.cuh -- device-side constants and descriptors shared by the
// kernels of libgitmvert.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/gitm_vert.h"

namespace gv {

constexpr int NS = GITM_NSPECIES;       // neutral species
constexpr int NI = GITM_NIONS - 1;      // ions without electrons
constexpr int NADV = GITM_NIONS_ADVECT; // advected ions
constexpr int NPAS = NI - NADV;         // passive ions (only their boundary cells move)
constexpr int NPC = 11;                 // passive-ion cells kept: -1,0,1, nAlts-5..nAlts+2

// Stage-state fields held for every cell, in shared memory.
enum Field : int {
  F_LNS = 0,    // LogNS(s)     0..5
  F_W = 6,      // VertVel(s)   6..11
  F_T = 12,     // Temp
  F_VE = 13,    // Vel_GD(iEast_)
  F_VN = 14,    // Vel_GD(iNorth_)
  F_VU = 15,    // Vel_GD(iUp_)
  F_I = 16,     // LogINS(1:2)  16..17
  F_LRHO = 18,  // LogRho
  NF = 19,
  NSTENCIL = 18 // fields with a Rusanov sweep: all but LogRho
};

// Grid coefficients, [NGC][G][gcols] followed by [NBC][gcols].
enum GridCoef : int {
  GC_DALTF = 0,  // dAlt_F
  GC_H2 = 1,     // 2 * InvDAlt_F
  GC_IDF = 2,    // InvDAlt_F
  GC_IDC = 3,    // 1 / dAlt_C
  GC_GRAV = 4,   // Gravity_G
  GC_INVR = 5,   // InvRadialDistance_C
  GC_R = 6,      // 1 / InvRadialDistance_C
  GC_ALT = 7,    // Altitude_G
  GC_M0 = 8,     // 5-point GradLogConS coefficients, cells 1..nAlts
  NGC = 13
};
constexpr int NBC = 20;  // lower mesh coefs (cells 0,-1) x5, upper (nAlts+1,+2) x5

// AUSM cell constants, [NGA][G][gcols] after the boundary block: they depend
// on the grid only (vertical_solver_ausm.f90:944-946, 1314-1352, 2029-2039).
enum AusmGridCoef : int {
  GA_DALTC = 0,  // dAlt_C
  GA_AP = 1,     // AreaFunction_P12 = RightRadius**2
  GA_AM = 2,     // AreaFunction_M12 = LeftRadius**2
  GA_VOL = 3,    // LocalCellVolume = (RightRadius**3 - LeftRadius**3) / 3
  GA_KP = 4,     // LiouKpS
  GA_KU = 5,     // Ku
  GA_DAMP = 6,   // 0.35 exp(-(Altitude - Altitude(0)) / 45 km)
  NGA = 7
};

// Earth constants (ModConstants.f90:11,15; ModEarth.f90:237-281,307-312).
struct Consts {
  double mass[NS];
  double log_mass[NS];
  double k_over_m[NS];
  double inv_vib2[NS];           // 1 / (Vibration - 2)
  double kc[NS][NS];             // 1e-2 k / (Mass_i Diff0_ij): friction coefficient
  double one_minus_e[NS];        // the six distinct 1 - DiffExp values
  double log_kb;                 // log(Boltzmanns_Constant)
};

struct DevMember {
  GitmColumnBatch b;     // device pointers (GITM-array form)
  GitmModVerticalBatch mv;  // device pointers (ModVertical form)
  const double* gridc;   // grid coefficients
  int32_t gcols;         // 1 = one grid for the member, else n_cols
  int32_t pad;
  int64_t col_offset;    // index of the member's first column in the status array
};

struct Tile {
  int32_t member;
  int32_t nc;      // columns in this tile
  int64_t c0;      // first column (member-local)
};

constexpr double KB = 1.3807e-23;
constexpr double PI = 3.141592653589793;

}  // namespace gv
