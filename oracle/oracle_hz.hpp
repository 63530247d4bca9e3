// oracle_hz.hpp -- CPU restatement of advance_horizontal (one block, every
// altitude) for the oracle.
//
// TEST INFRASTRUCTURE ONLY (see oracle_capi.cpp).  Follows
// advance_horizontal.f90:58-1034 statement by statement, in its loop order
// and with its expression grouping: per altitude the RK4 of :147-345 around
// horizontal_solver (:535-818), with calc_rusanov_lons / _lats (:821-922)
// and calc_facevalues_lons / _lats (:928-1034); the result stores of
// :346-421; then the parallel ion-velocity divergence of :423-517 with
// UAM_Gradient (gradient.f90:4-104).  UseTopography is not restated (it is
// not supported by the CUDA path either).  Parity: unpinned (no Fortran
// compiler here), like the vertical oracle.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "../include/gitm_hz.h"
#include "gitm_vert_oracle.hpp"

namespace gvo_hz {

using gvo::Limiter_mc;

// Fortran-layout block arrays with lower bounds -1 (GitmHzBlocks).
struct Shape {
  int nLons, nLats, nAlts, nBlocks;
  int NI() const { return nLons + 4; }
  int NJ() const { return nLats + 4; }
  int NK() const { return nAlts + 4; }
  // X(i, j, k, f, b) of a block array with nf fields (lower bounds -1)
  int64_t at(int i, int j, int k, int f, int nf, int b) const {
    return ((((int64_t(b) * nf + f) * NK() + (k + 1)) * NJ() + (j + 1)) * NI() + (i + 1));
  }
  int64_t at(int i, int j, int k, int b) const { return at(i, j, k, 0, 1, b); }
};

constexpr int nSpecies = GITM_NSPECIES;
constexpr int nIons = GITM_NIONS;
constexpr int nIonsAdvect = GITM_NIONS_ADVECT;
constexpr int iEast = 0, iNorth = 1, iUp = 2;

// A 2-D plane Q(-1:nLons+2, -1:nLats+2) of one altitude.
struct Plane {
  int nLons, nLats;
  std::vector<double> v;
  void init(int nl, int nt) {
    nLons = nl;
    nLats = nt;
    v.assign(size_t(nl + 4) * (nt + 4), 0.0);
  }
  double& operator()(int i, int j) { return v[size_t(j + 1) * (nLons + 4) + (i + 1)]; }
  double operator()(int i, int j) const { return v[size_t(j + 1) * (nLons + 4) + (i + 1)]; }
};

// calc_facevalues_lons / _lats (advance_horizontal.f90:928-1034) on one line
// Var(-1:n+2): IFB(i) = InvD*Dist_FB and DFB(i) = d*Dist_FB at face i of the
// line; VarLeft / VarRight (1:n+1) -> [i].
template <class FV, class FI, class FD>
void facevalues_line(int n, FV Var, FI IFB, FD DFB, double beta, std::vector<double>& VarLeft,
                     std::vector<double>& VarRight) {
  const double Factor1 = 0.6250000;
  const double Factor2 = 0.0416667;
  std::vector<double> dVarLimited(n + 2);  // 0:n+1
  double h, dVarUp, dVarDown;
  int i = 0;
  h = IFB(i + 1) * 2;
  dVarUp = h * (Factor1 * (Var(i + 1) - Var(i)) - Factor2 * (Var(i + 2) - Var(i - 1)));
  dVarDown = (Var(i) - Var(i - 1)) * IFB(i);
  dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, beta);
  for (i = 1; i <= n; ++i) {
    h = IFB(i + 1) * 2;
    dVarUp = h * (Factor1 * (Var(i + 1) - Var(i)) - Factor2 * (Var(i + 2) - Var(i - 1)));
    h = IFB(i) * 2;
    dVarDown = h * (Factor1 * (Var(i) - Var(i - 1)) - Factor2 * (Var(i + 1) - Var(i - 2)));
    dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, beta);
  }
  i = n + 1;
  dVarUp = (Var(i + 1) - Var(i)) * IFB(i + 1);
  h = IFB(i) * 2;
  dVarDown = h * (Factor1 * (Var(i) - Var(i - 1)) - Factor2 * (Var(i + 1) - Var(i - 2)));
  dVarLimited[i] = Limiter_mc(dVarUp, dVarDown, beta);
  VarLeft.assign(n + 2, 0.0);
  VarRight.assign(n + 2, 0.0);
  for (i = 1; i <= n + 1; ++i) {
    VarLeft[i] = Var(i - 1) + 0.5 * dVarLimited[i - 1] * DFB(i);
    VarRight[i] = Var(i) - 0.5 * dVarLimited[i] * DFB(i);
  }
}

// advance_horizontal(iBlock) for block b.  Returns a GITM_ST_ word.
inline uint32_t advance_horizontal_block(const GitmHzParams& prm, const GitmHzBlocks& B, int b, double Dt) {
  const Shape S{B.n_lons, B.n_lats, B.n_alts, B.n_blocks};
  const int nLons = S.nLons, nLats = S.nLats, nAlts = S.nAlts;
  uint32_t status = 0;
  auto blk = [&](const double* a, int i, int j, int k) { return a[S.at(i, j, k, b)]; };
  auto blkf = [&](const double* a, int i, int j, int k, int f, int nf) { return a[S.at(i, j, k, f, nf, b)]; };
  auto lat1 = [&](const double* a, int j) { return a[int64_t(b) * (nLats + 4) + (j + 1)]; };
  auto B_set = [](double* a, int64_t o, double v) { a[o] = v; };
  // cMax_GDB(0:nLons+1, 0:nLats+1, 0:nAlts+1, 3, nBlocks)
  auto cmax = [&](int i, int j, int k, int d) {
    return B.cmax[((((int64_t(b) * 3 + d) * (nAlts + 2) + k) * (nLats + 2) + j) * (nLons + 2)) + i];
  };

  // the 2-D planes of the current altitude (:87-95)
  Plane Rho_C, Temp_C, gamma_C;
  Plane Vel_CD[3], IVel_CD[3], Num_CV[nSpecies], VertVel_CV[nSpecies], INum_CV[nIonsAdvect];
  for (Plane* p : {&Rho_C, &Temp_C, &gamma_C}) p->init(nLons, nLats);
  for (int d = 0; d < 3; ++d) {
    Vel_CD[d].init(nLons, nLats);
    IVel_CD[d].init(nLons, nLats);
  }
  for (int s = 0; s < nSpecies; ++s) {
    Num_CV[s].init(nLons, nLats);
    VertVel_CV[s].init(nLons, nLats);
  }
  for (int s = 0; s < nIonsAdvect; ++s) INum_CV[s].init(nLons, nLats);
  // New*, Orig*, K* on the interior cells as planes too (ghosts unused)
  const int NF = 5 + 2 * nSpecies + nIonsAdvect;  // Rho, Temp, Vel(3), Num, VertVel, INum
  auto field = [&](int f) -> Plane& {
    if (f == 0) return Rho_C;
    if (f == 1) return Temp_C;
    if (f < 5) return Vel_CD[f - 2];
    if (f < 5 + nSpecies) return Num_CV[f - 5];
    if (f < 5 + 2 * nSpecies) return VertVel_CV[f - 5 - nSpecies];
    return INum_CV[f - 5 - 2 * nSpecies];
  };
  std::vector<Plane> New(NF), Orig(NF), K1(NF), K2(NF), K3(NF), K4(NF);
  for (int f = 0; f < NF; ++f)
    for (Plane* p : {&New[f], &Orig[f], &K1[f], &K2[f], &K3[f], &K4[f]}) p->init(nLons, nLats);

  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    for (int j = -1; j <= nLats + 2; ++j)
      for (int i = -1; i <= nLons + 2; ++i) {
        gamma_C(i, j) = blk(B.gamma, i, j, iAlt);
        Rho_C(i, j) = blk(B.rho, i, j, iAlt);
        for (int d = 0; d < 3; ++d) Vel_CD[d](i, j) = blkf(B.velocity, i, j, iAlt, d, 3);
        for (int s = 0; s < nSpecies; ++s) {
          VertVel_CV[s](i, j) = blkf(B.vert_vel, i, j, iAlt, s, nSpecies);
          Num_CV[s](i, j) = blkf(B.ndensity_s, i, j, iAlt, s, GITM_NSPECIES_TOTAL);
        }
        Temp_C(i, j) = blk(B.temperature, i, j, iAlt);
        for (int d = 0; d < 3; ++d) IVel_CD[d](i, j) = blkf(B.ivelocity, i, j, iAlt, d, 3);
        for (int s = 0; s < nIonsAdvect; ++s) INum_CV[s](i, j) = blkf(B.idensity_s, i, j, iAlt, s, nIons);
      }

    // ---- horizontal_solver (:535-818): New += -Dt (...) + Dt (...)
    auto horizontal_solver = [&]() {
      // calc_rusanov_lons (:876-922) and calc_rusanov_lats (:821-873)
      auto rusanov_lons = [&](const Plane& Var, Plane& GradVar, Plane& DiffVar) {
        std::vector<double> VarWest, VarEast;
        for (int iLat = 1; iLat <= nLats; ++iLat) {
          facevalues_line(
              nLons, [&](int i) { return Var(i, iLat); },
              [&](int i) { return blk(B.inv_dlon_dist_fb, i, iLat, iAlt); },
              [&](int i) { return blk(B.dlon_dist_fb, i, iLat, iAlt); }, prm.beta_limiter, VarWest, VarEast);
          std::vector<double> DiffFlux(nLons + 2);
          for (int i = 1; i <= nLons + 1; ++i)
            DiffFlux[i] = 0.5 * std::max(cmax(i - 1, iLat, iAlt, iEast), cmax(i, iLat, iAlt, iEast)) *
                          (VarEast[i] - VarWest[i]);
          for (int i = 1; i <= nLons; ++i) {
            const double InvdLon = blk(B.inv_dlon_dist_gb, i, iLat, iAlt);
            GradVar(i, iLat) = 0.5 * (VarWest[i + 1] + VarEast[i + 1] - VarWest[i] - VarEast[i]) * InvdLon;
            DiffVar(i, iLat) = (DiffFlux[i + 1] - DiffFlux[i]) * InvdLon;
          }
        }
      };
      auto rusanov_lats = [&](const Plane& Var, Plane& GradVar, Plane& DiffVar) {
        std::vector<double> VarSouth, VarNorth;
        for (int iLon = 1; iLon <= nLons; ++iLon) {
          facevalues_line(
              nLats, [&](int j) { return Var(iLon, j); },
              [&](int j) { return blk(B.inv_dlat_dist_fb, iLon, j, iAlt); },
              [&](int j) { return blk(B.dlat_dist_fb, iLon, j, iAlt); }, prm.beta_limiter, VarSouth, VarNorth);
          std::vector<double> DiffFlux(nLats + 2);
          for (int j = 1; j <= nLats + 1; ++j)
            DiffFlux[j] = 0.5 *
                          std::max(cmax(iLon, j - 1, iAlt, iNorth), cmax(iLon, j, iAlt, iNorth)) *
                          (VarNorth[j] - VarSouth[j]);
          for (int j = 1; j <= nLats; ++j) {
            const double InvdLat = blk(B.inv_dlat_dist_gb, iLon, j, iAlt);
            GradVar(iLon, j) = 0.5 * (VarSouth[j + 1] + VarNorth[j + 1] - VarSouth[j] - VarNorth[j]) * InvdLat;
            DiffVar(iLon, j) = (DiffFlux[j + 1] - DiffFlux[j]) * InvdLat;
          }
        }
      };
      std::vector<Plane> GLon(NF), GLat(NF), DLon(NF), DLat(NF);
      for (int f = 0; f < NF; ++f) {
        for (Plane* p : {&GLon[f], &GLat[f], &DLon[f], &DLat[f]}) p->init(nLons, nLats);
        // the order of the calls does not change any value
        rusanov_lons(field(f), GLon[f], DLon[f]);
        rusanov_lats(field(f), GLat[f], DLat[f]);
      }
      auto gLon = [&](int f, int i, int j) { return GLon[f](i, j); };
      auto gLat = [&](int f, int i, int j) { return GLat[f](i, j); };
      auto dLon = [&](int f, int i, int j) { return DLon[f](i, j); };
      auto dLat = [&](int f, int i, int j) { return DLat[f](i, j); };
      const int fR = 0, fT = 1, fV = 2, fN = 5, fW = 5 + nSpecies, fI = 5 + 2 * nSpecies;
      for (int iLat = 1; iLat <= nLats; ++iLat) {
        const double SinLat = std::sin(lat1(B.latitude, iLat));
        const double CosLat = lat1(B.cos_latitude, iLat);
        const double CoriolisSin = SinLat * 2 * prm.omega_body;
        const double CoriolisCos = CosLat * 2 * prm.omega_body;
        const double CentrifugalParameter = (prm.omega_body * prm.omega_body) * CosLat * SinLat;
        const double TanLat = lat1(B.tan_latitude, iLat);
        for (int iLon = 1; iLon <= nLons; ++iLon) {
          const double InvR = blk(B.inv_radial_distance, iLon, iLat, iAlt);
          const double VN = Vel_CD[iNorth](iLon, iLat), VE = Vel_CD[iEast](iLon, iLat),
                       VU = Vel_CD[iUp](iLon, iLat);
          // DivVel_C (:614-617)
          const double DivVel = gLat(fV + iNorth, iLon, iLat) + gLon(fV + iEast, iLon, iLat) - TanLat * VN * InvR;
          // :688-694
          New[fR](iLon, iLat) = New[fR](iLon, iLat) -
                                Dt * (Rho_C(iLon, iLat) * DivVel + gLat(fR, iLon, iLat) * VN + gLon(fR, iLon, iLat) * VE) +
                                Dt * (dLon(fR, iLon, iLat) + dLat(fR, iLon, iLat));
          // :696-703
          for (int s = 0; s < nSpecies; ++s)
            New[fN + s](iLon, iLat) =
                New[fN + s](iLon, iLat) -
                Dt * (Num_CV[s](iLon, iLat) * DivVel + gLat(fN + s, iLon, iLat) * VN + gLon(fN + s, iLon, iLat) * VE) +
                Dt * (dLon(fN + s, iLon, iLat) + dLat(fN + s, iLon, iLat));
          // :719-736
          for (int s = 0; s < nIonsAdvect; ++s)
            New[fI + s](iLon, iLat) = New[fI + s](iLon, iLat) -
                                      Dt * (+gLat(fI + s, iLon, iLat) * IVel_CD[iNorth](iLon, iLat) +
                                            gLon(fI + s, iLon, iLat) * IVel_CD[iEast](iLon, iLat)) +
                                      Dt * (dLon(fI + s, iLon, iLat) + dLat(fI + s, iLon, iLat));
          const double T = Temp_C(iLon, iLat), Rh = Rho_C(iLon, iLat);
          // :749-759
          New[fV + iEast](iLon, iLat) =
              New[fV + iEast](iLon, iLat) -
              Dt * (VN * gLat(fV + iEast, iLon, iLat) + VE * gLon(fV + iEast, iLon, iLat) +
                    VE * (VU - TanLat * VN) * InvR + gLon(fT, iLon, iLat) + gLon(fR, iLon, iLat) * T / Rh) +
              Dt * (dLon(fV + iEast, iLon, iLat) + dLat(fV + iEast, iLon, iLat));
          // :765-777
          New[fV + iNorth](iLon, iLat) =
              New[fV + iNorth](iLon, iLat) -
              Dt * (VN * gLat(fV + iNorth, iLon, iLat) + VE * gLon(fV + iNorth, iLon, iLat) +
                    (VN * VU + TanLat * (VE * VE)) * InvR + gLat(fT, iLon, iLat) + gLat(fR, iLon, iLat) * T / Rh) +
              Dt * (dLon(fV + iNorth, iLon, iLat) + dLat(fV + iNorth, iLon, iLat));
          // :785-790
          New[fV + iUp](iLon, iLat) = New[fV + iUp](iLon, iLat) -
                                      Dt * (VN * gLat(fV + iUp, iLon, iLat) + VE * gLon(fV + iUp, iLon, iLat)) +
                                      Dt * (dLon(fV + iUp, iLon, iLat) + dLat(fV + iUp, iLon, iLat));
          // :794-801
          for (int s = 0; s < nSpecies; ++s)
            New[fW + s](iLon, iLat) = New[fW + s](iLon, iLat) -
                                      Dt * (VN * gLat(fW + s, iLon, iLat) + VE * gLon(fW + s, iLon, iLat)) +
                                      Dt * (dLat(fW + s, iLon, iLat) + dLon(fW + s, iLon, iLat));
          // :803-813
          if (prm.use_coriolis) {
            New[fV + iEast](iLon, iLat) = New[fV + iEast](iLon, iLat) + Dt * (+CoriolisSin * VN - CoriolisCos * VU);
            New[fV + iNorth](iLon, iLat) =
                New[fV + iNorth](iLon, iLat) -
                Dt * (CentrifugalParameter * blk(B.radial_distance, iLon, iLat, iAlt) + CoriolisSin * VE);
          }
          // :817-823
          New[fT](iLon, iLat) = New[fT](iLon, iLat) -
                                Dt * ((gamma_C(iLon, iLat) - 1) * T * DivVel + gLat(fT, iLon, iLat) * VN +
                                      gLon(fT, iLon, iLat) * VE) +
                                Dt * (dLon(fT, iLon, iLat) + dLat(fT, iLon, iLat));
        }
      }
    };

    // ---- RK4 (:168-345)
    for (int f = 0; f < NF; ++f)
      for (int j = 1; j <= nLats; ++j)
        for (int i = 1; i <= nLons; ++i) {
          New[f](i, j) = field(f)(i, j);
          Orig[f](i, j) = field(f)(i, j);
        }
    std::vector<Plane>* Ks[4] = {&K1, &K2, &K3, &K4};
    for (int st = 0; st < 4; ++st) {
      horizontal_solver();
      for (int f = 0; f < NF; ++f)
        for (int j = 1; j <= nLats; ++j)
          for (int i = 1; i <= nLons; ++i) (*Ks[st])[f](i, j) = New[f](i, j) - field(f)(i, j);
      if (st == 3) break;
      for (int f = 0; f < NF; ++f)
        for (int j = 1; j <= nLats; ++j)
          for (int i = 1; i <= nLons; ++i) {
            const double k = (*Ks[st])[f](i, j);
            const double up = (st < 2) ? 0.5 * k + Orig[f](i, j) : k + Orig[f](i, j);
            field(f)(i, j) = up;
            New[f](i, j) = up;
          }
    }
    for (int f = 0; f < NF; ++f)
      for (int j = 1; j <= nLats; ++j)
        for (int i = 1; i <= nLons; ++i)
          New[f](i, j) = Orig[f](i, j) + (1.0 / 6.0) * (K1[f](i, j) + 2.0 * K2[f](i, j) + 2.0 * K3[f](i, j) + K4[f](i, j));

    // ---- stores (:346-421)
    const int fR = 0, fT = 1, fV = 2, fN = 5, fW = 5 + nSpecies, fI = 5 + 2 * nSpecies;
    bool neg = false;
    for (int j = 1; j <= nLats; ++j)
      for (int i = 1; i <= nLons; ++i) {
        B_set(B.rho, S.at(i, j, iAlt, b), New[fR](i, j));
        for (int d = 0; d < 3; ++d) B_set(B.velocity, S.at(i, j, iAlt, d, 3, b), New[fV + d](i, j));
        const double Told = blk(B.temperature, i, j, iAlt);
        if (B.temp_source)
          B.temp_source[((int64_t(b) * nAlts + iAlt - 1) * nLats + j - 1) * nLons + i - 1] = New[fT](i, j) - Told;
        B_set(B.temperature, S.at(i, j, iAlt, b), New[fT](i, j));
        for (int s = 0; s < nSpecies; ++s) {
          B_set(B.vert_vel, S.at(i, j, iAlt, s, nSpecies, b), New[fW + s](i, j));
          neg = neg || New[fN + s](i, j) < 0.0;
        }
      }
    if (neg) status |= GITM_ST_NEG_DENSITY;  // the reference stops (:359-372)
    for (int j = 1; j <= nLats; ++j)
      for (int i = 1; i <= nLons; ++i)
        for (int s = 0; s < nSpecies; ++s)
          B_set(B.ndensity_s, S.at(i, j, iAlt, s, GITM_NSPECIES_TOTAL, b), New[fN + s](i, j));
    if (prm.use_ion_advection) {
      for (int j = 1; j <= nLats; ++j)
        for (int i = 1; i <= nLons; ++i) {
          for (int s = 0; s < nIonsAdvect; ++s) {
            double v = New[fI + s](i, j);
            if (v < 1.0e2) v = 1.0e2;
            B_set(B.idensity_s, S.at(i, j, iAlt, s, nIons, b), v);
          }
          double e = 0.0;
          for (int s = 0; s < nIons - 1; ++s) e = e + blkf(B.idensity_s, i, j, iAlt, s, nIons);
          B_set(B.idensity_s, S.at(i, j, iAlt, nIons - 1, nIons, b), e);
        }
    }
  }

  // ---- the divergence of the parallel ion flow (:423-517)
  if (prm.use_ion_advection && prm.use_improved_ion_advection) {
    const double* VI = prm.non_magnetic ? B.ivelocity : B.ivelocity_par;
    std::vector<double> Div(size_t(nLons) * nLats * nAlts, 0.0);
    auto D = [&](int i, int j, int k) -> double& { return Div[(size_t(k - 1) * nLats + (j - 1)) * nLons + (i - 1)]; };
    for (int iDir = 0; iDir < 3; ++iDir) {
      auto Vi = [&](int i, int j, int k) { return blkf(VI, i, j, k, iDir, 3); };
      for (int k = 1; k <= nAlts; ++k)
        for (int j = 1; j <= nLats; ++j)
          for (int i = 1; i <= nLons; ++i) {
            // UAM_Gradient's component iDir (gradient.f90:38-102)
            double g = 0.0;
            const double InvR = blk(B.inv_radial_distance, i, j, k);
            if (iDir == iEast && nLons > 1) {
              const double InvCosLat = 1. / std::max(lat1(B.cos_latitude, j), 0.17);
              const int64_t o = int64_t(b) * nLons + (i - 1);
              g = (B.grad_lon_m[o] * Vi(i - 1, j, k) + B.grad_lon_0[o] * Vi(i, j, k) + B.grad_lon_p[o] * Vi(i + 1, j, k)) *
                  InvR * InvCosLat;
            } else if (iDir == iNorth && nLats > 1) {
              const int64_t o = int64_t(b) * nLats + (j - 1);
              g = (B.grad_lat_m[o] * Vi(i, j - 1, k) + B.grad_lat_0[o] * Vi(i, j, k) + B.grad_lat_p[o] * Vi(i, j + 1, k)) *
                  InvR;
            } else if (iDir == iUp && nAlts > 1) {
              const double Drp = blk(B.radial_distance, i, j, k + 1) - blk(B.radial_distance, i, j, k);
              const double Drm = blk(B.radial_distance, i, j, k) - blk(B.radial_distance, i, j, k - 1);
              const double DrmOverDrp = Drm / Drp;
              const double Drr2 = DrmOverDrp * DrmOverDrp;
              const double Bottom = Drm * (1 + DrmOverDrp);
              g = (Drr2 * Vi(i, j, k + 1) - Vi(i, j, k - 1) - (Drr2 - 1) * Vi(i, j, k)) / Bottom;
            }
            D(i, j, k) = D(i, j, k) + g;
            if (iDir == iNorth) {
              double TanLat = lat1(B.tan_latitude, j);
              if (TanLat > 5.0) TanLat = 5.0;
              if (TanLat < -5.0) TanLat = -5.0;
              D(i, j, k) = D(i, j, k) - TanLat * Vi(i, j, k) * InvR;
            }
            if (iDir == iUp) D(i, j, k) = D(i, j, k) + 2 * Vi(i, j, k) * InvR;
          }
    }
    for (int k = 1; k <= nAlts; ++k)
      for (int j = 1; j <= nLats; ++j)
        for (int i = 1; i <= nLons; ++i) D(i, j, k) = D(i, j, k) * lat1(B.cos_latitude, j);
    for (int s = 0; s < nIonsAdvect; ++s)
      for (int k = 1; k <= nAlts; ++k)
        for (int j = 1; j <= nLats; ++j)
          for (int i = 1; i <= nLons; ++i) {
            const double change = Dt * D(i, j, k);
            const int64_t o = S.at(i, j, k, s, nIons, b);
            B.idensity_s[o] = B.idensity_s[o] / (1 + change);
          }
    for (int k = -1; k <= nAlts + 2; ++k)
      for (int j = -1; j <= nLats + 2; ++j)
        for (int i = -1; i <= nLons + 2; ++i) {
          double e = 0.0;
          for (int s = 0; s < nIons - 1; ++s) e = e + blkf(B.idensity_s, i, j, k, s, nIons);
          B.idensity_s[S.at(i, j, k, nIons - 1, nIons, b)] = e;
        }
  }
  return status;
}

}  // namespace gvo_hz
