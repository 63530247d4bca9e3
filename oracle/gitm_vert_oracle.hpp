// gitm_vert_oracle.hpp -- CPU restatement of GITM's vertical advance.
//
// TEST INFRASTRUCTURE ONLY.  This is the checker for the CUDA path: tests/,
// __graft_entry__.smoke() and the cpu_baseline / --impl reference legs of
// bench.py may call it; the product library never does.
//
// It restates, statement by statement, in the reference's operation order:
//   src/advance_vertical.f90:80-217          gather / scatter of one column
//   src/vertical_solver_rusanov.f90:10-779   RK4 driver, stage, Rusanov flux,
//                                            limited face values
//   src/set_vertical_bcs.Earth.f90:8-652     lower / upper ghost cells
//   src/calc_neutral_friction.f90:4-108      implicit species friction
//   src/ludcmp.f:1-60, src/lubksb.f:1-28     Crout LU with implicit pivoting
//   src/ModLimiter.f90:16-36                 monotonised-central limiter
//   src/calc_pressure.f90:56-83              Gamma, NDensity
//   src/calc_rates.Earth.f90:34-50,83-84     MeanMajorMass, TempUnit
//   src/calc_timestep.f90:109-123            cMax, CFL time step
// Constants: src/ModEarth.f90:12-40,237-281,307-312,325,
// src/ModConstants.f90:11,15,23.
//
// The reference is built with gfortran -O3 -fdefault-real-8 (every REAL is
// IEEE binary64) and without FMA (x86-64 baseline), so this file is compiled
// with -ffp-contract=off and evaluates each Fortran expression left to right
// with the same parenthesisation.  Fortran arrays keep their index ranges
// through the A1/A2 accessors (altitude -1..nAlts+2, species 1..nSpecies).
//
// Parity status: no Fortran compiler exists where this was written and the
// reference holds no golden vectors for this path, so the restatement is
// "parity unpinned" against the Fortran; tests pin it with analytic checks.
//
// Dead code of the reference (values computed and never read by anything
// that reaches an output) is not restated; each omission is listed at the
// place it would have been.
#pragma once

#include <algorithm>
#include <cmath>
#include <limits>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/gitm_vert.h"

namespace gvo {

// ---------------------------------------------------------------- constants
// ModConstants.f90:11,15,23
constexpr double AMU = 1.6726e-27;
constexpr double Boltzmanns_Constant = 1.3807e-23;
constexpr double pi = 3.141592653589793;

constexpr int nSpecies = 6;  // ModEarth.f90:18
constexpr int nIons = 10;    // ModEarth.f90:38 (ie_)
constexpr int nIonsAdvect = 2;
constexpr int iO_3P_ = 1, iO2_ = 2, iN2_ = 3, iN_4S_ = 4, iNO_ = 5, iHe_ = 6;
constexpr int iEast_ = 1, iNorth_ = 2, iUp_ = 3;

struct Planet {
  double Mass[nSpecies + 1];                    // 1-based
  double Vibration[nSpecies + 1];               // 1-based
  double Diff0[nSpecies + 1][nSpecies + 1];     // 1-based
  double DiffExp[nSpecies + 1][nSpecies + 1];   // 1-based
  Planet() {
    // init_planet, ModEarth.f90:271-281
    const double mN4S = 14.0 * AMU;
    const double mO = 16.0 * AMU;
    Mass[0] = 0.0;
    Mass[iHe_] = 4.0 * AMU;
    Mass[iN_4S_] = mN4S;
    Mass[iO_3P_] = mO;
    Mass[iN2_] = 2 * mN4S;
    Mass[iO2_] = 2 * mO;
    Mass[iNO_] = mN4S + mO;
    // ModEarth.f90:307-312
    Vibration[0] = 0.0;
    Vibration[iO_3P_] = 5.0;
    Vibration[iO2_] = 7.0;
    Vibration[iN2_] = 7.0;
    Vibration[iN_4S_] = 5.0;
    Vibration[iNO_] = 7.0;
    Vibration[iHe_] = 5.0;
    // ModEarth.f90:237-261 (both tables are symmetric, so the Fortran
    // column-major reshape and this row-major listing agree).
    static const double d0[6][6] = {
        {0.000, 0.969, 0.969, 0.969, 0.715, 3.440},
        {0.969, 0.000, 0.715, 0.969, 0.715, 3.208},
        {0.969, 0.715, 0.000, 0.969, 0.527, 2.939},
        {0.969, 0.969, 0.969, 0.000, 0.969, 2.939},
        {0.715, 0.715, 0.527, 0.969, 0.000, 2.939},
        {3.440, 3.208, 2.939, 2.939, 2.939, 0.000}};
    static const double de[6][6] = {
        {0.000, 0.774, 0.774, 0.774, 0.750, 0.749},
        {0.774, 0.000, 0.750, 0.774, 0.750, 0.710},
        {0.774, 0.750, 0.000, 0.774, 0.810, 0.718},
        {0.774, 0.774, 0.774, 0.000, 0.774, 0.718},
        {0.750, 0.750, 0.810, 0.774, 0.000, 0.718},
        {0.749, 0.710, 0.718, 0.718, 0.718, 0.000}};
    for (int i = 0; i <= nSpecies; ++i)
      for (int j = 0; j <= nSpecies; ++j) {
        Diff0[i][j] = 0.0;
        DiffExp[i][j] = 0.0;
      }
    for (int i = 1; i <= nSpecies; ++i)
      for (int j = 1; j <= nSpecies; ++j) {
        Diff0[i][j] = 1.0e17 * d0[i - 1][j - 1];
        DiffExp[i][j] = de[i - 1][j - 1];
      }
  }
};

inline const Planet& planet() {
  static const Planet p;
  return p;
}

inline bool is_photochemical(int s) { return s == iN_4S_ || s == iNO_; }  // set_vertical_bcs.Earth.f90:89-91

// ---------------------------------------------------------------- math shims
// All transcendentals go through these so an instrumented scalar type can
// count them.  For double they are the C library functions, as gfortran uses.
inline double xexp(double x) { return std::exp(x); }
inline double xlog(double x) { return std::log(x); }
inline double xpow(double x, double y) { return std::pow(x, y); }
inline double xsqrt(double x) { return std::sqrt(x); }
inline double xcos(double x) { return std::cos(x); }
inline double xtanh(double x) { return std::tanh(x); }
inline double xabs(double x) { return std::fabs(x); }
inline double val(double x) { return x; }

// Fortran MIN/MAX of reals.
template <class R> inline R fmin2(const R& a, const R& b) { return (b < a) ? b : a; }
template <class R> inline R fmax2(const R& a, const R& b) { return (b > a) ? b : a; }

// ---------------------------------------------------------------- column
// The ModVertical module (ModVertical.f90:15-48) for one column.
template <class R>
struct Column {
  int nAlts = 0;
  int G = 0;
  // state
  std::vector<R> LogRho, Temp, Vel_GD, IVel, LogNS, VertVel, LogINS;
  // coefficients
  std::vector<R> cMax, MeanMajorMass, Gamma, EddyCoef;
  std::vector<R> Gravity, Altitude, dAlt_C, InvR, dAlt_F, InvDAlt_F;
  R Centrifugal = 0, Coriolis = 0;
  double SZA = 0, MLat = 0;
  bool has_lbc = false;
  double lbc[2][GITM_LBC_NVALUES];  // cells -1, 0
  uint32_t status = 0;

  void resize(int n) {
    nAlts = n;
    G = n + 4;
    for (auto* v : {&LogRho, &Temp, &cMax, &MeanMajorMass, &Gamma, &EddyCoef,
                    &Gravity, &Altitude, &dAlt_C, &InvR, &dAlt_F, &InvDAlt_F})
      v->assign(G, R(0));
    Vel_GD.assign(3 * G, R(0));
    IVel.assign(3 * G, R(0));
    LogNS.assign(nSpecies * G, R(0));
    VertVel.assign(nSpecies * G, R(0));
    LogINS.assign(nIons * G, R(0));
  }
};

// Fortran-index accessors: A1(v, iAlt) for v(-1:nAlts+2), A2(v, iAlt, k) for
// v(-1:nAlts+2, 1:K).
#define A1(v, i) (v)[(i) + 1]
#define A2(v, i, k) (v)[((k)-1) * G + (i) + 1]

// ---------------------------------------------------------------- limiter
// ModLimiter.f90:16-36
template <class R>
inline R Limiter_mc(const R& dUp, const R& dDown, double BetaLimiter) {
  if (dUp > 0.0) {
    if (dDown > 0.0) {
      R a = BetaLimiter * dUp, b = BetaLimiter * dDown, c = (dUp + dDown) * 0.5;
      return fmin2(fmin2(a, b), c);
    }
    return R(0.0);
  } else {
    if (dDown < 0.0) {
      R a = BetaLimiter * dUp, b = BetaLimiter * dDown, c = (dUp + dDown) * 0.5;
      return fmax2(fmax2(a, b), c);
    }
    return R(0.0);
  }
}

// ---------------------------------------------------------------- Rusanov
// calc_facevalues_alts_rusanov, vertical_solver_rusanov.f90:726-779.
// Var, VarLeft/VarRight use Fortran indices via the offsets below:
// Var(-1:nAlts+2) -> Var[i+1];  VarLeft(1:nAlts+1) -> VarLeft[i].
template <class R>
void facevalues_rusanov(const Column<R>& c, const R* Var, R* VarLeft, R* VarRight,
                        double BetaLimiter) {
  const int nAlts = c.nAlts;
  const double Factor1 = 0.6250000;
  const double Factor2 = 0.0416667;
  std::vector<R> dVarLimited(nAlts + 2);  // 0:nAlts+1
  auto V = [&](int i) -> const R& { return Var[i + 1]; };
  auto IF = [&](int i) -> const R& { return c.InvDAlt_F[i + 1]; };
  for (int i = 1; i <= nAlts; ++i) {
    R h = IF(i + 1) * 2.0;
    R dVarUp = h * (Factor1 * (V(i + 1) - V(i)) - Factor2 * (V(i + 2) - V(i - 1)));
    h = IF(i) * 2.0;
    R dVarDown = h * (Factor1 * (V(i) - V(i - 1)) - Factor2 * (V(i + 1) - V(i - 2)));
    dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, BetaLimiter);
  }
  {
    int i = 0;
    R dVarUp = (V(i + 1) - V(i)) * IF(i + 1);
    R dVarDown = (V(i) - V(i - 1)) * IF(i);
    dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, BetaLimiter);
  }
  {
    int i = nAlts + 1;
    R dVarUp = (V(i + 1) - V(i)) * IF(i + 1);
    R dVarDown = (V(i) - V(i - 1)) * IF(i);
    dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, BetaLimiter);
  }
  for (int i = 1; i <= nAlts + 1; ++i) {
    VarLeft[i] = V(i - 1) + 0.5 * dVarLimited[i - 1] * c.dAlt_F[i + 1];
    VarRight[i] = V(i) - 0.5 * dVarLimited[i] * c.dAlt_F[i + 1];
  }
}

// calc_rusanov_alts_rusanov, vertical_solver_rusanov.f90:694-718.
// GradVar, DiffVar are (1:nAlts) -> [i].
template <class R>
void rusanov_alts(const Column<R>& c, const R* Var, R* GradVar, R* DiffVar,
                  double BetaLimiter) {
  const int nAlts = c.nAlts;
  std::vector<R> VarLeft(nAlts + 2), VarRight(nAlts + 2), DiffFlux(nAlts + 2);
  facevalues_rusanov(c, Var, VarLeft.data(), VarRight.data(), BetaLimiter);
  for (int i = 1; i <= nAlts; ++i)
    GradVar[i] = 0.5 * (VarLeft[i + 1] + VarRight[i + 1] - VarLeft[i] - VarRight[i]) /
                 c.dAlt_C[i + 1];
  // cMax(0:nAlts+1) is stored on cells, so cMax(i) -> cMax[i+1].
  for (int i = 1; i <= nAlts + 1; ++i)
    DiffFlux[i] = 0.5 * fmax2(c.cMax[i - 1 + 1], c.cMax[i + 1]) * (VarRight[i] - VarLeft[i]);
  for (int i = 1; i <= nAlts; ++i)
    DiffVar[i] = (DiffFlux[i + 1] - DiffFlux[i]) / c.dAlt_C[i + 1];
}

// ---------------------------------------------------------------- LU
// ludcmp.f:1-60.  a is 1-based a[i][j] (i = row), n <= 6.
template <class R>
bool ludcmp(R a[7][7], int n, int indx[7], R& d) {
  const double TINY = 1.0e-20;
  R vv[7];
  int imax = 0;
  d = 1.;
  for (int i = 1; i <= n; ++i) {
    R aamax = 0.;
    for (int j = 1; j <= n; ++j)
      if (xabs(a[i][j]) > aamax) aamax = xabs(a[i][j]);
    if (aamax == 0.) return false;  // stop_gitm('singular matrix in ludcmp')
    vv[i] = 1. / aamax;
  }
  for (int j = 1; j <= n; ++j) {
    for (int i = 1; i <= j - 1; ++i) {
      R sum = a[i][j];
      for (int k = 1; k <= i - 1; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
    }
    R aamax = 0.;
    for (int i = j; i <= n; ++i) {
      R sum = a[i][j];
      for (int k = 1; k <= j - 1; ++k) sum = sum - a[i][k] * a[k][j];
      a[i][j] = sum;
      R dum = vv[i] * xabs(sum);
      if (dum >= aamax) {
        imax = i;
        aamax = dum;
      }
    }
    if (j != imax) {
      for (int k = 1; k <= n; ++k) {
        R dum = a[imax][k];
        a[imax][k] = a[j][k];
        a[j][k] = dum;
      }
      d = -d;
      vv[imax] = vv[j];
    }
    indx[j] = imax;
    if (a[j][j] == 0.) a[j][j] = TINY;
    if (j != n) {
      R dum = 1. / a[j][j];
      for (int i = j + 1; i <= n; ++i) a[i][j] = a[i][j] * dum;
    }
  }
  return true;
}

// lubksb.f:1-28
template <class R>
void lubksb(R a[7][7], int n, const int indx[7], R b[7]) {
  int ii = 0;
  for (int i = 1; i <= n; ++i) {
    int ll = indx[i];
    R sum = b[ll];
    b[ll] = b[i];
    if (ii != 0) {
      for (int j = ii; j <= i - 1; ++j) sum = sum - a[i][j] * b[j];
    } else if (sum != 0.) {
      ii = i;
    }
    b[i] = sum;
  }
  for (int i = n; i >= 1; --i) {
    R sum = b[i];
    for (int j = i + 1; j <= n; ++j) sum = sum - a[i][j] * b[j];
    b[i] = sum / a[i][i];
  }
}

// ---------------------------------------------------------------- friction
// calc_neutral_friction.f90:4-108.  oVel, NDensityS, GradLogCon are
// (1:nAlts, 1:nSpecies) -> [(s-1)*nAlts + iAlt-1]; EddyCoef, NDensity, Temp
// are (1:nAlts) -> [iAlt-1].
template <class R>
void neutral_friction(double DtIn, R* oVel, const R* EddyCoef, const R* NDensity,
                      const R* NDensityS, const R* GradLogCon, const R* Temp, int nAlts,
                      bool UseNeutralFriction, uint32_t& status) {
  const Planet& P = planet();
  if (!UseNeutralFriction) return;
  auto I2 = [&](int iAlt, int s) { return (s - 1) * nAlts + iAlt - 1; };
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    R Vel[7];
    R CoefMatrix[7][7];
    R EddyContribution[7];
    for (int s = 1; s <= nSpecies; ++s) Vel[s] = oVel[I2(iAlt, s)];
    for (int i = 0; i <= nSpecies; ++i)
      for (int j = 0; j <= nSpecies; ++j) CoefMatrix[i][j] = 0.0;
    // InvDij (lines 72-95) is accumulated but never read: omitted.
    for (int iSpecies = 1; iSpecies <= nSpecies; ++iSpecies) {
      R kTOverM = Boltzmanns_Constant * Temp[iAlt - 1] / P.Mass[iSpecies];
      R denscale = 1.0 / NDensity[iAlt - 1];
      for (int jSpecies = 1; jSpecies <= nSpecies; ++jSpecies) {
        if (jSpecies == iSpecies) continue;
        R TempDij = (1.0e-04) *
                    (P.Diff0[iSpecies][jSpecies] *
                     (xpow(Temp[iAlt - 1], P.DiffExp[iSpecies][jSpecies]))) /
                    (NDensity[iAlt - 1] * (1.0e-06));
        CoefMatrix[iSpecies][jSpecies] =
            kTOverM * denscale * NDensityS[I2(iAlt, jSpecies)] / TempDij;
      }
      EddyContribution[iSpecies] = -1.0 * EddyCoef[iAlt - 1] * GradLogCon[I2(iAlt, iSpecies)];
    }
    R Matrix[7][7];
    for (int i = 1; i <= nSpecies; ++i)
      for (int j = 1; j <= nSpecies; ++j) Matrix[i][j] = -DtIn * CoefMatrix[i][j];
    for (int i = 1; i <= nSpecies; ++i) {
      R sum = 0.0;  // Fortran SUM over the whole row, in order
      for (int j = 1; j <= nSpecies; ++j) sum = sum + CoefMatrix[i][j];
      Matrix[i][i] = 1.0 + DtIn * (sum);
    }
    int iPivot[7];
    R Parity;
    if (ludcmp(Matrix, nSpecies, iPivot, Parity)) {
      lubksb(Matrix, nSpecies, iPivot, Vel);
    } else {
      // stop_gitm('singular matrix in ludcmp') ends the reference's run here;
      // the column has no defined result, so its velocities become NaN
      status |= GITM_ST_LU_SINGULAR;
      for (int s = 1; s <= nSpecies; ++s) Vel[s] = std::numeric_limits<double>::quiet_NaN();
    }
    for (int s = 1; s <= nSpecies; ++s) oVel[I2(iAlt, s)] = Vel[s] + EddyContribution[s];
  }
}

// ---------------------------------------------------------------- BCs
// Mesh coefficients of the 3rd-order one-sided extrapolation,
// set_vertical_bcs.Earth.f90:279-297 (lower) and :505-525 (upper).
template <class R>
void lower_mesh_coefs(const Column<R>& c, int iAlt, R C[5]) {
  const int G = c.G;
  (void)G;
  R h1 = A1(c.dAlt_F, iAlt + 2), h2 = A1(c.dAlt_F, iAlt + 3), h3 = A1(c.dAlt_F, iAlt + 4),
    h4 = A1(c.dAlt_F, iAlt + 5);
  R MeshH1 = h1;
  R MeshH2 = h1 + h2;
  R MeshH3 = h1 + h2 + h3;
  R MeshH4 = h1 + h2 + h3 + h4;
  C[0] = -1.0 * (MeshH2 * MeshH3 * MeshH4 + MeshH1 * MeshH3 * MeshH4 + MeshH1 * MeshH2 * MeshH4 +
                 MeshH1 * MeshH2 * MeshH3) /
         (MeshH1 * MeshH2 * MeshH3 * MeshH4);
  C[1] = 1.0 * (MeshH2 * MeshH3 * MeshH4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
  C[2] = -1.0 * (MeshH1 * MeshH3 * MeshH4) / (MeshH2 * h2 * h3 * (h3 + h4));
  C[3] = 1.0 * (MeshH1 * MeshH2 * MeshH4) / (MeshH3 * (h3 + h2) * h3 * h4);
  C[4] = -1.0 * (MeshH1 * MeshH2 * MeshH3) / (MeshH4 * (h2 + h3 + h4) * (h3 + h4) * h4);
}

template <class R>
void upper_mesh_coefs(const Column<R>& c, int iAlt, R C[5]) {
  const int G = c.G;
  (void)G;
  R hm1 = A1(c.dAlt_F, iAlt - 1), hm2 = A1(c.dAlt_F, iAlt - 2), hm3 = A1(c.dAlt_F, iAlt - 3),
    hm4 = A1(c.dAlt_F, iAlt - 4);
  R MeshHm1 = hm1;
  R MeshHm2 = hm1 + hm2;
  R MeshHm3 = hm1 + hm2 + hm3;
  R MeshHm4 = hm1 + hm2 + hm3 + hm4;
  C[0] = 1.0 *
         (MeshHm2 * MeshHm3 * MeshHm4 + MeshHm1 * MeshHm3 * MeshHm4 + MeshHm1 * MeshHm2 * MeshHm4 +
          MeshHm1 * MeshHm2 * MeshHm3) /
         (MeshHm1 * MeshHm2 * MeshHm3 * MeshHm4);
  C[1] = -1.0 * (MeshHm2 * MeshHm3 * MeshHm4) / (hm1 * hm2 * (hm2 + hm3) * (hm2 + hm3 + hm4));
  C[2] = 1.0 * (MeshHm1 * MeshHm3 * MeshHm4) / (MeshHm2 * hm2 * hm3 * (hm3 + hm4));
  C[3] = -1.0 * (MeshHm1 * MeshHm2 * MeshHm4) / (MeshHm3 * (hm3 + hm2) * hm3 * hm4);
  C[4] = 1.0 * (MeshHm1 * MeshHm2 * MeshHm3) / (MeshHm4 * (hm2 + hm3 + hm4) * (hm3 + hm4) * hm4);
}

// set_vertical_bcs (Earth), set_vertical_bcs.Earth.f90:8-652, on the column
// state arrays passed (they are the RK stage's copies, not always c's own).
// IVel's ghost cells are not set: nothing on the path reads them (the IVel
// Rusanov sweeps, vertical_solver_rusanov.f90:478-479, feed only the unused
// DiviVel).  The electron slot LogINS(:,nIons) is not set: it is never read.
template <class R>
void set_vertical_bcs(const Column<R>& c, const GitmVertParams& prm, R* LogRho, R* LogNS,
                      R* Vel_GD, R* Temp, R* LogINS, R* VertVel, uint32_t& status) {
  const Planet& P = planet();
  const int nAlts = c.nAlts;
  const int G = c.G;
  const bool UseMsisBCs = prm.use_msis_bcs != 0 && c.has_lbc;
  const bool UseImprovedIonAdvection = prm.use_improved_ion_advection != 0;

  std::vector<R> NS(nSpecies * G), EffectiveGravity(G);
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) A2(NS, i, s) = xexp(A2(LogNS, i, s));
  for (int i = -1; i <= nAlts + 2; ++i)
    A1(EffectiveGravity, i) = A1(c.Gravity, i) + c.Centrifugal / A1(c.InvR, i);

  // ---- bottom
  if (UseMsisBCs) {
    // lines 119-137: msis_bcs results come from the hoisted table.
    for (int iAlt = -1; iAlt <= 0; ++iAlt) {
      const double* t = c.lbc[iAlt + 1];
      for (int s = 1; s <= nSpecies; ++s) A2(LogNS, iAlt, s) = t[s - 1];
      A1(Temp, iAlt) = t[6];
      A1(LogRho, iAlt) = t[7];
      A2(Vel_GD, iAlt, iEast_) = t[8];
      A2(Vel_GD, iAlt, iNorth_) = t[9];
    }
  } else {
    for (int iAlt = -1; iAlt <= 0; ++iAlt) {
      A2(Vel_GD, iAlt, iEast_) = 0.0;
      A2(Vel_GD, iAlt, iNorth_) = 0.0;
    }
  }
  // DuringPerturb = F (ModInputs.f90:121): lines 145-148.
  for (int iAlt = -1; iAlt <= 0; ++iAlt) {
    A2(Vel_GD, iAlt, iUp_) = 0.0;
    for (int s = 1; s <= nSpecies; ++s) A2(VertVel, iAlt, s) = 0.0;
  }
  // Tides (UseGSWMTides/UseWACCMTides = F) and the mesh coefficients of
  // lines 170-189 (overwritten before use) are omitted.

  // lines 192-196
  A1(Temp, -1) = A1(Temp, 0);
  for (int d = 1; d <= 3; ++d) A2(Vel_GD, -1, d) = A2(Vel_GD, 0, d);

  for (int s = 1; s <= nSpecies; ++s) {
    if (!is_photochemical(s)) {
      // lines 205-222
      int iAlt = -1;
      R MeanGravity = -0.5 * (A1(EffectiveGravity, iAlt) + A1(EffectiveGravity, iAlt + 1));
      R MeanTemp = 0.5 * (A1(Temp, iAlt + 1) + A1(Temp, iAlt));
      R MeanMass = 0.5 * (A1(c.MeanMajorMass, iAlt + 1) + A1(c.MeanMajorMass, iAlt));
      R InvScaleHeightS = MeanGravity * MeanMass / (MeanTemp * Boltzmanns_Constant);
      A2(NS, iAlt, s) = A2(NS, iAlt + 1, s) * (A1(Temp, iAlt + 1) / A1(Temp, iAlt)) *
                        xexp(1.0 * InvScaleHeightS * A1(c.dAlt_F, iAlt));
      A2(LogNS, iAlt, s) = xlog(A2(NS, iAlt, s));
      if (s == iO_3P_) A2(LogNS, iAlt, s) = A2(LogNS, 0, s);
    } else {
      // lines 226-272
      for (int iAlt = 0; iAlt >= -1; --iAlt) {
        R C[5];
        lower_mesh_coefs(c, iAlt, C);
        R dLogNS = A2(LogNS, iAlt + 1, s) * C[0] + A2(LogNS, iAlt + 2, s) * C[1] +
                   A2(LogNS, iAlt + 3, s) * C[2] + A2(LogNS, iAlt + 4, s) * C[3] +
                   A2(LogNS, iAlt + 5, s) * C[4];
        A2(LogNS, iAlt, s) = A2(LogNS, iAlt + 1, s) - A1(c.dAlt_F, iAlt + 1) * dLogNS;
        if (dLogNS <= 0.0) A2(LogNS, iAlt, s) = A2(LogNS, iAlt + 1, s);
        if (s == iNO_) {
          if (A2(LogNS, iAlt, s) < A2(LogNS, iAlt + 1, s) - 0.333)
            A2(LogNS, iAlt, s) = A2(LogNS, iAlt + 1, s) - 0.333;
        }
      }
    }
  }

  // lines 277-378
  for (int iAlt = 0; iAlt >= -1; --iAlt) {
    R C[5];
    lower_mesh_coefs(c, iAlt, C);
    for (int s = 1; s <= nIons - 1; ++s) A2(LogINS, iAlt, s) = A2(LogINS, iAlt + 1, s);
    for (int s = 1; s <= nSpecies; ++s) {
      R dVertVel = A2(VertVel, iAlt + 1, s) * C[0] + A2(VertVel, iAlt + 2, s) * C[1] +
                   A2(VertVel, iAlt + 3, s) * C[2] + A2(VertVel, iAlt + 4, s) * C[3] +
                   A2(VertVel, iAlt + 5, s) * C[4];
      A2(VertVel, iAlt, s) = A2(VertVel, iAlt + 1, s) - A1(c.dAlt_F, iAlt + 1) * dVertVel;
    }
    for (int s = 1; s <= nSpecies; ++s) A2(NS, iAlt, s) = xexp(A2(LogNS, iAlt, s));
    R SumRho = 0.0;
    for (int s = 1; s <= nSpecies; ++s) SumRho = SumRho + P.Mass[s] * A2(NS, iAlt, s);
    A1(LogRho, iAlt) = xlog(SumRho);
    A2(Vel_GD, iAlt, iUp_) = 0.0;
    for (int s = 1; s <= nSpecies; ++s)
      A2(Vel_GD, iAlt, iUp_) = A2(Vel_GD, iAlt, iUp_) + A2(NS, iAlt, s) * P.Mass[s] *
                                                             A2(VertVel, iAlt, s) /
                                                             xexp(A1(LogRho, iAlt));
    if (iAlt == -1 && UseMsisBCs) {
      for (int d = iEast_; d <= iNorth_; ++d) {
        R dv = A2(Vel_GD, iAlt + 1, d) * C[0] + A2(Vel_GD, iAlt + 2, d) * C[1] +
               A2(Vel_GD, iAlt + 3, d) * C[2] + A2(Vel_GD, iAlt + 4, d) * C[3] +
               A2(Vel_GD, iAlt + 5, d) * C[4];
        A2(Vel_GD, iAlt, d) = A2(Vel_GD, iAlt + 1, d) - A1(c.dAlt_F, iAlt + 1) * dv;
      }
    }
  }

  // lines 382-395
  for (int s = 1; s <= nSpecies; ++s) {
    if (is_photochemical(s) && (A2(VertVel, 1, s) > 0.0) && (s != iO_3P_)) {
      A2(VertVel, 0, s) = -1.0 * A2(VertVel, 1, s);
      A2(VertVel, -1, s) = -1.0 * A2(VertVel, 1, s);
    }
  }

  // ---- top, lines 420-458
  for (int i = nAlts + 1; i <= nAlts + 2; ++i) {
    A2(Vel_GD, i, iEast_) = A2(Vel_GD, nAlts, iEast_);
    A2(Vel_GD, i, iNorth_) = A2(Vel_GD, nAlts, iNorth_);
  }
  for (int s = 1; s <= nSpecies; ++s) {
    A2(VertVel, nAlts + 1, s) = A2(VertVel, nAlts, s);
    A2(VertVel, nAlts + 2, s) = A2(VertVel, nAlts, s);
    if (is_photochemical(s) && (A2(VertVel, nAlts, s) < 0.0)) {
      A2(VertVel, nAlts + 1, s) = -A2(VertVel, nAlts, s);
      A2(VertVel, nAlts + 2, s) = -A2(VertVel, nAlts - 1, s);
    }
  }
  if (A2(Vel_GD, nAlts, iUp_) < 0.0) {
    A2(Vel_GD, nAlts + 1, iUp_) = -A2(Vel_GD, nAlts, iUp_);
    A2(Vel_GD, nAlts + 2, iUp_) = -A2(Vel_GD, nAlts, iUp_);
  } else {
    A2(Vel_GD, nAlts + 1, iUp_) = A2(Vel_GD, nAlts, iUp_);
    A2(Vel_GD, nAlts + 2, iUp_) = A2(Vel_GD, nAlts, iUp_);
  }
  // IVel top ghosts (lines 423-424, 452-458): not read, omitted.
  A1(Temp, nAlts + 1) = A1(Temp, nAlts);
  A1(Temp, nAlts + 2) = A1(Temp, nAlts);
  // LogRho(nAlts+1:nAlts+2) of lines 465-467 are overwritten at 598-604.

  // lines 471-486
  for (int s = 1; s <= nSpecies; ++s) {
    for (int iAlt = nAlts + 1; iAlt <= nAlts + 2; ++iAlt) {
      R MeanGravity = -0.5 * (A1(EffectiveGravity, iAlt) + A1(EffectiveGravity, iAlt - 1));
      R MeanTemp = 0.5 * (A1(Temp, iAlt - 1) + A1(Temp, iAlt));
      R InvScaleHeightS = MeanGravity * P.Mass[s] / (MeanTemp * Boltzmanns_Constant);
      A2(NS, iAlt, s) = A2(NS, iAlt - 1, s) * (A1(Temp, iAlt - 1) / A1(Temp, iAlt)) *
                        xexp(-InvScaleHeightS * A1(c.dAlt_F, iAlt));
      A2(LogNS, iAlt, s) = xlog(A2(NS, iAlt, s));
    }
  }

  // lines 488-501
  bool UsePlasmasphereBC = false;
  if (prm.use_nighttime_ion_bcs) {
    if (c.SZA > pi / 2 &&
        ((c.MLat > 30.0 && c.MLat < 70.0) || (c.MLat > -60.0 && c.MLat < -30.0)))
      UsePlasmasphereBC = true;
  }
  R tec = 0.0;
  if (UseImprovedIonAdvection) {
    for (int i = 1; i <= nAlts; ++i) tec = tec + A1(c.dAlt_F, i) * A2(LogINS, i, 1);
  } else {
    for (int i = 1; i <= nAlts; ++i) tec = tec + A1(c.dAlt_F, i) * xexp(A2(LogINS, i, 1));
  }
  tec = tec / 1e16;

  // lines 503-596
  for (int iAlt = nAlts + 1; iAlt <= nAlts + 2; ++iAlt) {
    R Cm[5];
    upper_mesh_coefs(c, iAlt, Cm);
    for (int s = 1; s <= nIons - 1; ++s) {
      R n0, n1, n2, n3, n4, n5;
      if (UseImprovedIonAdvection) {
        // check_for_negative_densities, lines 608-649
        R mn = A2(LogINS, iAlt - 5, s);
        for (int k = iAlt - 4; k <= iAlt; ++k) mn = fmin2(mn, A2(LogINS, k, s));
        if (mn < 0.0) {
          if (A2(LogINS, iAlt - 6, s) < 0.0) status |= GITM_ST_NEG_ION_TOP;
          for (int k = iAlt - 5; k <= iAlt - 1; ++k) {
            if (A2(LogINS, k, s) < 0.0) {
              if (A2(LogINS, k - 1, s) > 0.0 && A2(LogINS, k + 1, s) > 0.0)
                A2(LogINS, k, s) = (A2(LogINS, k - 1, s) + A2(LogINS, k + 1, s)) / 2.0;
              else
                A2(LogINS, k, s) = A2(LogINS, k - 1, s) * 0.95;
            }
          }
          if (A2(LogINS, iAlt, s) < 0.0) A2(LogINS, iAlt, s) = A2(LogINS, iAlt - 1, s) * 0.95;
        }
        n0 = xlog(A2(LogINS, iAlt, s));
        n1 = xlog(A2(LogINS, iAlt - 1, s));
        n2 = xlog(A2(LogINS, iAlt - 2, s));
        n3 = xlog(A2(LogINS, iAlt - 3, s));
        n4 = xlog(A2(LogINS, iAlt - 4, s));
        n5 = xlog(A2(LogINS, iAlt - 5, s));
      } else {
        n0 = A2(LogINS, iAlt, s);
        n1 = A2(LogINS, iAlt - 1, s);
        n2 = A2(LogINS, iAlt - 2, s);
        n3 = A2(LogINS, iAlt - 3, s);
        n4 = A2(LogINS, iAlt - 4, s);
        n5 = A2(LogINS, iAlt - 5, s);
      }
      R dn = Cm[0] * n1 + Cm[1] * n2 + Cm[2] * n3 + Cm[3] * n4 + Cm[4] * n5;
      if (tec < prm.min_tec && UsePlasmasphereBC) {
        // do nothing
      } else {
        if (dn > -(0.001 * n0 / A1(c.dAlt_F, nAlts))) dn = -(0.001 * n0 / A1(c.dAlt_F, nAlts));
        n0 = n1 + dn * A1(c.dAlt_F, iAlt);
        if (UseImprovedIonAdvection)
          A2(LogINS, iAlt, s) = xexp(n0);
        else
          A2(LogINS, iAlt, s) = n0;
      }
    }
  }

  // lines 598-604
  for (int iAlt = nAlts + 1; iAlt <= nAlts + 2; ++iAlt) {
    R SumRho = 0.0;
    for (int s = 1; s <= nSpecies; ++s) SumRho = SumRho + P.Mass[s] * xexp(A2(LogNS, iAlt, s));
    A1(LogRho, iAlt) = xlog(SumRho);
  }
}

// 4th-order 5-point gradient on the non-uniform mesh at cell iAlt,
// vertical_solver_rusanov.f90:515-533; MC = MeshCoef0..4.
template <class R>
void gradlogcons_coefs(const Column<R>& c, int iAlt, R MC[5]) {
  const int G = c.G;
  (void)G;
  R h1 = A1(c.dAlt_F, iAlt - 1), h2 = A1(c.dAlt_F, iAlt + 0), h3 = A1(c.dAlt_F, iAlt + 1),
    h4 = A1(c.dAlt_F, iAlt + 2);
  R MeshH2 = h2 + h1;
  R MeshH3 = h3 + h2 + h1;
  R MeshH4 = h4 + h3 + h2 + h1;
  MC[0] = (h2 * h3 * (h3 + h4)) / (h1 * MeshH2 * MeshH3 * MeshH4);
  MC[1] = -1.0 * (MeshH2 * h3 * (h3 + h4)) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
  MC[3] = MeshH2 * h2 * (h4 + h3) / (MeshH3 * (h2 + h3) * h3 * h4);
  MC[4] = -1.0 * MeshH2 * h2 * h3 / (MeshH4 * (h2 + h3 + h4) * (h3 + h4) * h4);
  MC[2] = (h2 * h3 * (h3 + h4) + MeshH2 * h3 * (h3 + h4) - MeshH2 * h2 * (h3 + h4) -
           MeshH2 * h2 * h3) /
          (MeshH2 * h2 * h3 * (h3 + h4));
}

// ---------------------------------------------------------------- stage
// advance_vertical_1stage, vertical_solver_rusanov.f90:387-686.  Inputs are
// the stage state; New* arrays enter holding copies of it (the driver copies
// before the call) and leave with cells 1..nAlts updated.
template <class R>
void rusanov_stage(const Column<R>& c, const GitmVertParams& prm, double Dt, const R* LogRho,
                   const R* LogNS, const R* Vel_GD, const R* Temp, R* NewLogRho, R* NewLogNS,
                   R* NewVel_GD, R* NewTemp, const R* LogINS, R* NewLogINS, const R* IVel,
                   const R* VertVel, R* NewVertVel, uint32_t& status) {
  const Planet& P = planet();
  const int nAlts = c.nAlts;
  const int G = c.G;
  const double Beta = prm.beta_limiter;
  std::vector<R> NS(nSpecies * G), Rho(G), LogNum(G), NT(G);

  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) A2(NS, i, s) = xexp(A2(LogNS, i, s));
  for (int i = -1; i <= nAlts + 2; ++i) A1(Rho, i) = xexp(A1(LogRho, i));
  for (int i = -1; i <= nAlts + 2; ++i) {
    R sum = 0.0;
    for (int s = 1; s <= nSpecies; ++s) sum = sum + A2(NS, i, s);
    A1(LogNum, i) = xlog(sum);
  }
  for (int i = -1; i <= nAlts + 2; ++i) A1(NT, i) = xexp(A1(LogNum, i));

  // (1:nAlts) arrays indexed [iAlt]
  std::vector<R> GradTemp(nAlts + 1), DiffTemp(nAlts + 1), DivVel(nAlts + 1);
  std::vector<R> GradVel(3 * (nAlts + 1)), DiffVel(3 * (nAlts + 1));
  std::vector<R> GradLogNS(nSpecies * (nAlts + 1)), DiffLogNS(nSpecies * (nAlts + 1));
  std::vector<R> GradVertVel(nSpecies * (nAlts + 1)), DiffVertVel(nSpecies * (nAlts + 1)),
      DivVertVel(nSpecies * (nAlts + 1));
  std::vector<R> GradLogINS(nIonsAdvect * (nAlts + 1)), DiffLogINS(nIonsAdvect * (nAlts + 1));
  auto J = [&](int s, int i) { return (s - 1) * (nAlts + 1) + i; };

  // The LogRho and LogNum sweeps (lines 472-473), the IVel sweeps (478-479),
  // DiviVel (484) and the sweeps of ions nIonsAdvect+1..nIons-1 (498-502)
  // produce values nothing reads: omitted.
  rusanov_alts(c, Temp, GradTemp.data(), DiffTemp.data(), Beta);
  for (int d = 1; d <= 3; ++d)
    rusanov_alts(c, &Vel_GD[(d - 1) * G], &GradVel[J(d, 0)], &DiffVel[J(d, 0)], Beta);
  for (int i = 1; i <= nAlts; ++i)
    DivVel[i] = GradVel[J(iUp_, i)] + 2 * A2(Vel_GD, i, iUp_) * A1(c.InvR, i);

  for (int s = 1; s <= nSpecies; ++s) {
    rusanov_alts(c, &LogNS[(s - 1) * G], &GradLogNS[J(s, 0)], &DiffLogNS[J(s, 0)], Beta);
    rusanov_alts(c, &VertVel[(s - 1) * G], &GradVertVel[J(s, 0)], &DiffVertVel[J(s, 0)], Beta);
    for (int i = 1; i <= nAlts; ++i)
      DivVertVel[J(s, i)] = GradVertVel[J(s, i)] + 2 * A2(VertVel, i, s) * A1(c.InvR, i);
  }
  for (int s = 1; s <= nIonsAdvect; ++s)
    rusanov_alts(c, &LogINS[(s - 1) * G], &GradLogINS[J(s, 0)], &DiffLogINS[J(s, 0)], Beta);

  // lines 506-509
  std::vector<R> LogConS(nSpecies * G);
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i)
      A2(LogConS, i, s) = xlog(P.Mass[s] * A2(NS, i, s) / A1(Rho, i));

  // lines 511-543; GradLogConS is (1:nAlts, nSpecies) -> [(s-1)*nAlts + iAlt-1]
  std::vector<R> GradLogConS(nSpecies * nAlts);
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    R MC[5];
    gradlogcons_coefs(c, iAlt, MC);
    for (int s = 1; s <= nSpecies; ++s)
      GradLogConS[(s - 1) * nAlts + iAlt - 1] =
          MC[0] * A2(LogConS, iAlt - 2, s) + MC[1] * A2(LogConS, iAlt - 1, s) +
          MC[2] * A2(LogConS, iAlt, s) + MC[3] * A2(LogConS, iAlt + 1, s) +
          MC[4] * A2(LogConS, iAlt + 2, s);
  }

  // lines 548-617.  The sponge NuSP (575-579) is never applied: omitted.
  std::vector<R> VertTau(nAlts + 1, R(prm.vert_tau));
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    for (int s = 1; s <= nSpecies; ++s)
      A2(NewLogNS, iAlt, s) =
          A2(LogNS, iAlt, s) -
          Dt * (DivVertVel[J(s, iAlt)] + A2(VertVel, iAlt, s) * GradLogNS[J(s, iAlt)]) +
          Dt * DiffLogNS[J(s, iAlt)];
    for (int s = 1; s <= nIonsAdvect; ++s)
      A2(NewLogINS, iAlt, s) = A2(NewLogINS, iAlt, s) -
                               Dt * (A2(IVel, iAlt, iUp_) * GradLogINS[J(s, iAlt)]) +
                               Dt * DiffLogINS[J(s, iAlt)];
    A2(NewVel_GD, iAlt, iUp_) = 0.0;
    if (prm.use_damping)
      VertTau[iAlt] = 15 - (1 - xexp(-1.0 * A1(c.Altitude, iAlt) / 1000.0 / 40.0)) * 5.0;
    for (int s = 1; s <= nSpecies; ++s) {
      A2(NewVertVel, iAlt, s) =
          A2(VertVel, iAlt, s) -
          Dt * (A2(VertVel, iAlt, s) * GradVertVel[J(s, iAlt)] -
                (A2(Vel_GD, iAlt, iNorth_) * A2(Vel_GD, iAlt, iNorth_) +
                 A2(Vel_GD, iAlt, iEast_) * A2(Vel_GD, iAlt, iEast_)) *
                    A1(c.InvR, iAlt) +
                A1(Temp, iAlt) * GradLogNS[J(s, iAlt)] * Boltzmanns_Constant / P.Mass[s] +
                GradTemp[iAlt] * Boltzmanns_Constant / P.Mass[s] - A1(c.Gravity, iAlt)) +
          Dt * DiffVertVel[J(s, iAlt)] - A2(VertVel, iAlt, s) / VertTau[iAlt];
      if (prm.use_coriolis)
        A2(NewVertVel, iAlt, s) =
            A2(NewVertVel, iAlt, s) +
            Dt * (c.Centrifugal / A1(c.InvR, iAlt) + c.Coriolis * A2(Vel_GD, iAlt, iEast_));
      A2(NewVertVel, iAlt, s) =
          A2(NewVertVel, iAlt, s) -
          Dt * (prm.thermal_diff_coef[s - 1] * Boltzmanns_Constant * GradTemp[iAlt]) / P.Mass[s];
    }
  }

  // lines 632-641
  if (prm.use_neutral_friction) {
    std::vector<R> nVel(nSpecies * nAlts), NSs(nSpecies * nAlts), Ed(nAlts), NTs(nAlts),
        Ts(nAlts);
    for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
      Ed[iAlt - 1] = A1(c.EddyCoef, iAlt);
      NTs[iAlt - 1] = A1(NT, iAlt);
      Ts[iAlt - 1] = A1(Temp, iAlt);
      for (int s = 1; s <= nSpecies; ++s) {
        nVel[(s - 1) * nAlts + iAlt - 1] = A2(NewVertVel, iAlt, s);
        NSs[(s - 1) * nAlts + iAlt - 1] = A2(NS, iAlt, s);
      }
    }
    neutral_friction(Dt, nVel.data(), Ed.data(), NTs.data(), NSs.data(), GradLogConS.data(),
                     Ts.data(), nAlts, true, status);
    for (int iAlt = 1; iAlt <= nAlts; ++iAlt)
      for (int s = 1; s <= nSpecies; ++s)
        A2(NewVertVel, iAlt, s) = nVel[(s - 1) * nAlts + iAlt - 1];
  }

  // lines 643-658
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    for (int s = 1; s <= nSpecies; ++s) {
      A2(NewVertVel, iAlt, s) = fmax2(R(-prm.max_vertical_velocity), A2(NewVertVel, iAlt, s));
      A2(NewVertVel, iAlt, s) = fmin2(R(prm.max_vertical_velocity), A2(NewVertVel, iAlt, s));
      A2(NewVel_GD, iAlt, iUp_) =
          A2(NewVel_GD, iAlt, iUp_) +
          A2(NewVertVel, iAlt, s) * (P.Mass[s] * A2(NS, iAlt, s) / A1(Rho, iAlt));
    }
  }

  // lines 660-680
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    A2(NewVel_GD, iAlt, iEast_) = A2(NewVel_GD, iAlt, iEast_) -
                                  Dt * A2(Vel_GD, iAlt, iUp_) * GradVel[J(iEast_, iAlt)] +
                                  Dt * DiffVel[J(iEast_, iAlt)];
    A2(NewVel_GD, iAlt, iNorth_) = A2(NewVel_GD, iAlt, iNorth_) -
                                   Dt * A2(Vel_GD, iAlt, iUp_) * GradVel[J(iNorth_, iAlt)] +
                                   Dt * DiffVel[J(iNorth_, iAlt)];
    A1(NewTemp, iAlt) =
        A1(NewTemp, iAlt) -
        Dt * (A2(Vel_GD, iAlt, iUp_) * GradTemp[iAlt] +
              (A1(c.Gamma, iAlt) - 1.0) * (A1(Temp, iAlt) * DivVel[iAlt])) +
        Dt * DiffTemp[iAlt];
  }
  // lines 681-684
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    R NewSumRho = 0.0;
    for (int s = 1; s <= nSpecies; ++s)
      NewSumRho = NewSumRho + P.Mass[s] * xexp(A2(NewLogNS, iAlt, s));
    A1(NewLogRho, iAlt) = xlog(NewSumRho);
  }
}

// ---------------------------------------------------------------- RK4 driver
// advance_vertical_1d_rusanov, vertical_solver_rusanov.f90:10-384, on the
// column's own state (c.LogRho ... c.VertVel).
template <class R>
void advance_vertical_1d_rusanov(Column<R>& c, const GitmVertParams& prm, double Dt) {
  const int G = c.G;
  auto& st = c.status;
  set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                   c.LogINS.data(), c.VertVel.data(), st);

  // The state as a list of arrays so the RK algebra is one loop.
  std::vector<R>* S[6] = {&c.LogNS, &c.LogINS, &c.LogRho, &c.Vel_GD, &c.Temp, &c.VertVel};
  std::vector<R> Orig[6], New[6], K[4][6];
  for (int v = 0; v < 6; ++v) Orig[v] = *S[v];

  const double cstage[3] = {0.5, 0.5, 1.0};
  for (int k = 0; k < 4; ++k) {
    for (int v = 0; v < 6; ++v) New[v] = *S[v];
    rusanov_stage(c, prm, Dt, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                  New[2].data(), New[0].data(), New[3].data(), New[4].data(), c.LogINS.data(),
                  New[1].data(), c.IVel.data(), c.VertVel.data(), New[5].data(), st);
    for (int v = 0; v < 6; ++v) {
      K[k][v].resize(S[v]->size());
      for (size_t i = 0; i < S[v]->size(); ++i) K[k][v][i] = New[v][i] - (*S[v])[i];
    }
    if (k < 3) {
      for (int v = 0; v < 6; ++v)
        for (size_t i = 0; i < S[v]->size(); ++i)
          (*S[v])[i] = Orig[v][i] + cstage[k] * K[k][v][i];
      set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                       c.LogINS.data(), c.VertVel.data(), st);
    }
  }
  // lines 350-366
  for (int v = 0; v < 6; ++v)
    for (size_t i = 0; i < S[v]->size(); ++i)
      (*S[v])[i] = Orig[v][i] + (1.0 / 6.0) * (K[0][v][i] + 2.0 * K[1][v][i] +
                                               2.0 * K[2][v][i] + K[3][v][i]);
  set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                   c.LogINS.data(), c.VertVel.data(), st);
  (void)G;
}

// ---------------------------------------------------------------- grid
// Per-column derived geometry, advance_vertical.f90:141-151.
template <class R>
void derive_faces(Column<R>& c) {
  const int nAlts = c.nAlts;
  const int G = c.G;
  for (int i = 0; i <= nAlts + 2; ++i) A1(c.dAlt_F, i) = A1(c.Altitude, i) - A1(c.Altitude, i - 1);
  A1(c.dAlt_F, -1) = A1(c.dAlt_F, 0);
  for (int i = -1; i <= nAlts + 2; ++i) A1(c.InvDAlt_F, i) = 1.0 / A1(c.dAlt_F, i);
}

// ---------------------------------------------------------------- producers
// calc_pressure.f90:17-21,56-83 (NDensity, Gamma), calc_rates.Earth.f90:34-50
// (MeanMajorMass, TempUnit), calc_timestep.f90:109-118 (cMax).  One column.
struct Producers {
  std::vector<double> NDensity, Gamma, MeanMajorMass, TempUnit, cMax;
};

inline void produce_coefficients(int nAlts, const double* nden_s /*[6][G] col-stride 1*/,
                                 const double* temperature, const double* vert_vel,
                                 Producers& out) {
  const Planet& P = planet();
  const int G = nAlts + 4;
  out.NDensity.assign(G, 0.0);
  out.Gamma.assign(G, 0.0);
  out.MeanMajorMass.assign(G, 0.0);
  out.TempUnit.assign(G, 0.0);
  out.cMax.assign(G, 0.0);
  for (int g = 0; g < G; ++g) {
    double N = 0.0;
    for (int s = 1; s <= nSpecies; ++s) N = N + nden_s[(s - 1) * G + g];
    out.NDensity[g] = N;
    double gm = 0.0;
    for (int s = 1; s <= nSpecies; ++s) gm = gm + nden_s[(s - 1) * G + g] / (P.Vibration[s] - 2);
    out.Gamma[g] = gm * 2.0 / N + 1;
    double mmm = 0.0;
    for (int s = 1; s <= nSpecies; ++s)
      mmm = mmm + P.Mass[s] * nden_s[(s - 1) * G + g] / (N + 1.0);
    if (mmm == 0) mmm = P.Mass[1];
    out.MeanMajorMass[g] = mmm;
    out.TempUnit[g] = mmm / Boltzmanns_Constant;
  }
  // cMax on cells 0..nAlts+1 (g = 1..nAlts+2); the end cells keep 0.
  for (int g = 1; g <= nAlts + 2; ++g) {
    double mx = std::fabs(vert_vel[g]);
    for (int s = 2; s <= nSpecies; ++s) mx = std::max(mx, std::fabs(vert_vel[(s - 1) * G + g]));
    out.cMax[g] = mx + std::sqrt(out.Gamma[g] * temperature[g]);
  }
}

#undef A1
#undef A2

}  // namespace gvo
