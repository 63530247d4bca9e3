// oracle_ausm.hpp -- CPU restatement of GITM's AUSM vertical solver.
//
// TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; see
// gitm_vert_oracle.hpp).  Restates, in the reference's statement order:
//   src/vertical_solver_ausm.f90:26-433     advance_vertical_1d_ausm (RK driver)
//   src/vertical_solver_ausm.f90:436-999    advance_vertical_1stage_ausm
//   src/vertical_solver_ausm.f90:1007-1090  calc_rusanov_alts_ausm / facevalues
//   src/vertical_solver_ausm.f90:1093-2070  calc_all_fluxes_hydro (AUSM+-up)
//   src/vertical_solver_ausm.f90:2073-2117  calc_kt_facevalues
// Values the reference computes and never reads are not restated: the
// LogPress, LogRho, LogNum, IVel, LogNS and VertVel Rusanov sweeps (only the
// Temp gradient, the wind diffusion and the ion sweeps are read), HydroNT /
// HydroPressure / HydroRho (passed to the flux routine but not used there),
// VelocityCap (:~530, never applied), the sponge and the first NewLogRho
// update (overwritten at :993-996).
#pragma once

#include "gitm_vert_oracle.hpp"

namespace gvo {

#define A1(v, i) (v)[(i) + 1]
#define A2(v, i, k) (v)[((k)-1) * G + (i) + 1]

// calc_kt_facevalues, vertical_solver_ausm.f90:2073-2117.  Outputs are
// (1:nAlts) -> [i].
template <class R>
void kt_facevalues(const Column<R>& c, const R* Var, R* LM, R* RM, R* LP, R* RP, double Beta) {
  const int nAlts = c.nAlts;
  std::vector<R> dL(nAlts + 2);  // 0:nAlts+1
  auto V = [&](int i) -> const R& { return Var[i + 1]; };
  auto IF = [&](int i) -> const R& { return c.InvDAlt_F[i + 1]; };
  auto DF = [&](int i) -> const R& { return c.dAlt_F[i + 1]; };
  for (int i = 0; i <= nAlts + 1; ++i) {
    R dVarUp = (V(i + 1) - V(i)) * IF(i + 1);
    R dVarDown = (V(i) - V(i - 1)) * IF(i);
    dL[i] = Limiter_mc(dVarUp, dVarDown, Beta);
  }
  for (int i = 1; i <= nAlts; ++i) {
    LM[i] = V(i - 1) + 0.5 * dL[i - 1] * DF(i - 1);
    RM[i] = V(i) - 0.5 * dL[i] * DF(i);
    LP[i] = V(i) + 0.5 * dL[i] * DF(i);
    RP[i] = V(i + 1) - 0.5 * dL[i + 1] * DF(i + 1);
  }
}

// calc_all_fluxes_hydro, vertical_solver_ausm.f90:1093-2070.  Per-cell outputs
// are (1:nAlts) -> [i]; per-species ones [(s-1)*(nAlts+1) + i].
template <class R>
void all_fluxes_hydro(const Column<R>& c, const GitmVertParams& prm, double DtIn, const R* RhoS,
                      const R* PressureS, const R* HydroPressureS, const R* Temp, const R* Vel_GD,
                      const R* VertVel, R* RhoSFlux, R* MomentumSFlux, R* EnergyFlux, R* MomentumFlux,
                      const R* RadDist, const std::vector<char>& SubtractHydrostatic) {
  const int nAlts = c.nAlts;
  const int G = c.G;
  const double Beta = prm.beta_limiter;
  const int N1 = nAlts + 1;
  auto J = [&](int s, int i) { return (s - 1) * N1 + i; };
  auto SH = [&](int i, int s) { return SubtractHydrostatic[(s - 1) * G + i + 1] != 0; };
  (void)Temp;

  const double MInf = 1.0e-19;
  const double LiouBeta = 1.0 / 8.0;
  std::vector<R> LogRhoS(nSpecies * G), LogPS(nSpecies * G), LogHydroPressureS(nSpecies * G);
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) {
      A2(LogRhoS, i, s) = xlog(A2(RhoS, i, s));
      A2(LogPS, i, s) = xlog(A2(PressureS, i, s));
      A2(LogHydroPressureS, i, s) = xlog(A2(HydroPressureS, i, s));
    }
  // Kp / Ku altitude profiles (:1283-1352)
  const double LogMaxKu = std::log(0.50), LogMinKu = std::log(0.25);
  const double LogMaxKp = std::log(1.0e-09), LogMinKp = std::log(1.0e-19);
  const double KpWidth = 15.0e+03, KpAltMidPoint = 160.0e+03;
  std::vector<R> LiouKpS(nSpecies * N1), Ku(nSpecies * N1);
  for (int i = 1; i <= nAlts; ++i)
    for (int s = 1; s <= nSpecies; ++s) {
      R th = xtanh((A1(c.Altitude, i) - KpAltMidPoint) / KpWidth);
      R LogKp = LogMinKp + 0.5 * (LogMaxKp - LogMinKp) * (1.0 + th);
      R LogKu = LogMinKu + 0.5 * (LogMaxKu - LogMinKu) * (1.0 + th);
      LiouKpS[J(s, i)] = xexp(LogKp);
      Ku[J(s, i)] = xexp(LogKu);
    }

  std::vector<R> RhoSL_M(nSpecies * N1), RhoSR_M(nSpecies * N1), RhoSL_P(nSpecies * N1),
      RhoSR_P(nSpecies * N1);
  std::vector<R> HPSL_M(nSpecies * N1), HPSR_M(nSpecies * N1), HPSL_P(nSpecies * N1),
      HPSR_P(nSpecies * N1);
  std::vector<R> PSL_M(nSpecies * N1), PSR_M(nSpecies * N1), PSL_P(nSpecies * N1),
      PSR_P(nSpecies * N1);
  std::vector<R> VL_M(nSpecies * N1), VR_M(nSpecies * N1), VL_P(nSpecies * N1),
      VR_P(nSpecies * N1);
  std::vector<R> t0(N1), t1(N1), t2(N1), t3(N1);
  for (int s = 1; s <= nSpecies; ++s) {
    kt_facevalues(c, &LogRhoS[(s - 1) * G], t0.data(), t1.data(), t2.data(), t3.data(), Beta);
    for (int i = 1; i <= nAlts; ++i) {
      RhoSL_M[J(s, i)] = xexp(t0[i]);
      RhoSR_M[J(s, i)] = xexp(t1[i]);
      RhoSL_P[J(s, i)] = xexp(t2[i]);
      RhoSR_P[J(s, i)] = xexp(t3[i]);
    }
  }
  for (int s = 1; s <= nSpecies; ++s) {
    kt_facevalues(c, &LogHydroPressureS[(s - 1) * G], t0.data(), t1.data(), t2.data(), t3.data(), Beta);
    for (int i = 1; i <= nAlts; ++i) {
      HPSL_M[J(s, i)] = xexp(t0[i]);
      HPSR_M[J(s, i)] = xexp(t1[i]);
      HPSL_P[J(s, i)] = xexp(t2[i]);
      HPSR_P[J(s, i)] = xexp(t3[i]);
    }
  }
  for (int s = 1; s <= nSpecies; ++s) {
    kt_facevalues(c, &LogPS[(s - 1) * G], t0.data(), t1.data(), t2.data(), t3.data(), Beta);
    for (int i = 1; i <= nAlts; ++i) {
      PSL_M[J(s, i)] = xexp(t0[i]);
      PSR_M[J(s, i)] = xexp(t1[i]);
      PSL_P[J(s, i)] = xexp(t2[i]);
      PSR_P[J(s, i)] = xexp(t3[i]);
    }
  }
  for (int s = 1; s <= nSpecies; ++s) {
    kt_facevalues(c, &VertVel[(s - 1) * G], t0.data(), t1.data(), t2.data(), t3.data(), Beta);
    for (int i = 1; i <= nAlts; ++i) {
      VL_M[J(s, i)] = t0[i];
      VR_M[J(s, i)] = t1[i];
      VL_P[J(s, i)] = t2[i];
      VR_P[J(s, i)] = t3[i];
    }
  }
  std::vector<R> RhoL_M(N1, R(0.0)), RhoR_M(N1, R(0.0)), RhoL_P(N1, R(0.0)), RhoR_P(N1, R(0.0));
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = 1; i <= nAlts; ++i) {
      RhoL_M[i] = RhoL_M[i] + RhoSL_M[J(s, i)];
      RhoR_M[i] = RhoR_M[i] + RhoSR_M[J(s, i)];
      RhoL_P[i] = RhoL_P[i] + RhoSL_P[J(s, i)];
      RhoR_P[i] = RhoR_P[i] + RhoSR_P[J(s, i)];
    }
  std::vector<R> PL_M(N1, R(0.0)), PR_M(N1, R(0.0)), PL_P(N1, R(0.0)), PR_P(N1, R(0.0));
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = 1; i <= nAlts; ++i) {
      PL_M[i] = PL_M[i] + PSL_M[J(s, i)];
      PR_M[i] = PR_M[i] + PSR_M[J(s, i)];
      PL_P[i] = PL_P[i] + PSL_P[J(s, i)];
      PR_P[i] = PR_P[i] + PSR_P[J(s, i)];
    }
  // Vel_GD face values (VGD*[d][i]); the up component is replaced by the
  // mass-weighted species value (:1503-1530)
  std::vector<R> VGL_M(3 * N1), VGR_M(3 * N1), VGL_P(3 * N1), VGR_P(3 * N1);
  for (int d = 1; d <= 3; ++d)
    kt_facevalues(c, &Vel_GD[(d - 1) * G], &VGL_M[(d - 1) * N1], &VGR_M[(d - 1) * N1],
                  &VGL_P[(d - 1) * N1], &VGR_P[(d - 1) * N1], Beta);
  auto VG = [&](std::vector<R>& v, int d, int i) -> R& { return v[(d - 1) * N1 + i]; };
  for (int i = 1; i <= nAlts; ++i) {
    VG(VGL_M, iUp_, i) = 0.0;
    VG(VGR_M, iUp_, i) = 0.0;
    VG(VGL_P, iUp_, i) = 0.0;
    VG(VGR_P, iUp_, i) = 0.0;
  }
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = 1; i <= nAlts; ++i) {
      VG(VGL_M, iUp_, i) = VG(VGL_M, iUp_, i) + RhoSL_M[J(s, i)] * VL_M[J(s, i)] / RhoL_M[i];
      VG(VGR_M, iUp_, i) = VG(VGR_M, iUp_, i) + RhoSR_M[J(s, i)] * VR_M[J(s, i)] / RhoR_M[i];
      VG(VGL_P, iUp_, i) = VG(VGL_P, iUp_, i) + RhoSL_P[J(s, i)] * VL_P[J(s, i)] / RhoL_P[i];
      VG(VGR_P, iUp_, i) = VG(VGR_P, iUp_, i) + RhoSR_P[J(s, i)] * VR_P[J(s, i)] / RhoR_P[i];
    }
  std::vector<R> GL_M(N1), GR_M(N1), GL_P(N1), GR_P(N1);
  kt_facevalues(c, c.Gamma.data(), GL_M.data(), GR_M.data(), GL_P.data(), GR_P.data(), Beta);

  auto sq = [](const R& x) { return x * x; };  // x**2.0
  std::vector<R> EL_M(N1), ER_M(N1), EL_P(N1), ER_P(N1);
  std::vector<R> HL_M(N1), HR_M(N1), HL_P(N1), HR_P(N1);
  for (int i = 1; i <= nAlts; ++i) {
    auto E = [&](const R& g, const R& P, const R& rho, const std::vector<R>& v) {
      return (1.0 / (g - 1.0)) * P +
             0.5 * rho * (sq(VG(const_cast<std::vector<R>&>(v), iUp_, i)) +
                          sq(VG(const_cast<std::vector<R>&>(v), iEast_, i)) +
                          sq(VG(const_cast<std::vector<R>&>(v), iNorth_, i)));
    };
    EL_M[i] = E(GL_M[i], PL_M[i], RhoL_M[i], VGL_M);
    ER_M[i] = E(GR_M[i], PR_M[i], RhoR_M[i], VGR_M);
    EL_P[i] = E(GL_P[i], PL_P[i], RhoL_P[i], VGL_P);
    ER_P[i] = E(GR_P[i], PR_P[i], RhoR_P[i], VGR_P);
    auto H = [&](const R& g, const R& P, const R& rho, const std::vector<R>& v) {
      return 0.5 * (sq(VG(const_cast<std::vector<R>&>(v), iUp_, i)) +
                    sq(VG(const_cast<std::vector<R>&>(v), iEast_, i)) +
                    sq(VG(const_cast<std::vector<R>&>(v), iNorth_, i))) +
             (g / (g - 1.0)) * P / rho;
    };
    HL_M[i] = H(GL_M[i], PL_M[i], RhoL_M[i], VGL_M);
    HR_M[i] = H(GR_M[i], PR_M[i], RhoR_M[i], VGR_M);
    HL_P[i] = H(GL_P[i], PL_P[i], RhoL_P[i], VGL_P);
    HR_P[i] = H(GR_P[i], PR_P[i], RhoR_P[i], VGR_P);
  }
  // Liou interface sound speed (:1568-1655)
  std::vector<R> CS_M(N1), CS_P(N1);
  for (int i = 1; i <= nAlts; ++i) {
    R SubCs = xsqrt(2.0 * ((GL_M[i] - 1.0) / (GL_M[i] + 1.0)) * HL_M[i]);
    R CSL_M = sq(SubCs) / fmax2(SubCs, VG(VGL_M, iUp_, i));
    SubCs = xsqrt(2.0 * ((GR_M[i] - 1.0) / (GR_M[i] + 1.0)) * HR_M[i]);
    R CSR_M = sq(SubCs) / fmax2(SubCs, -1.0 * VG(VGR_M, iUp_, i));
    CS_M[i] = fmin2(CSL_M, CSR_M);
    SubCs = xsqrt(2.0 * ((GL_P[i] - 1.0) / (GL_P[i] + 1.0)) * HL_P[i]);
    R CSL_P = sq(SubCs) / fmax2(SubCs, VG(VGL_P, iUp_, i));
    SubCs = xsqrt(2.0 * ((GR_P[i] - 1.0) / (GR_P[i] + 1.0)) * HR_P[i]);
    R CSR_P = sq(SubCs) / fmax2(SubCs, -1.0 * VG(VGR_P, iUp_, i));
    CS_P[i] = fmin2(CSL_P, CSR_P);
  }

  // species fluxes
  std::vector<R> RhoSFlux_M(nSpecies * N1), RhoSFlux_P(nSpecies * N1), MomSFlux_M(nSpecies * N1),
      MomSFlux_P(nSpecies * N1), NumP_M(nSpecies * N1), NumP_P(nSpecies * N1), NumV_M(nSpecies * N1),
      NumV_P(nSpecies * N1);
  for (int s = 1; s <= nSpecies; ++s) {
    for (int i = 1; i <= nAlts; ++i) {
      const int q = J(s, i);
      R MeanPS_P = 0.5 * (PSL_P[q] + PSR_P[q]);
      R MeanPS_M = 0.5 * (PSL_M[q] + PSR_M[q]);
      R MeanHPS_P = 0.5 * (HPSL_P[q] + HPSR_P[q]);
      R MeanHPS_M = 0.5 * (HPSL_M[q] + HPSR_M[q]);
      R MeanRhoS_P = 0.5 * (RhoSL_P[q] + RhoSR_P[q]);
      R MeanRhoS_M = 0.5 * (RhoSL_M[q] + RhoSR_M[q]);
      R ML_M = VL_M[q] / CS_M[i], MR_M = VR_M[q] / CS_M[i];
      R ML_P = VL_P[q] / CS_P[i], MR_P = VR_P[q] / CS_P[i];
      R M2Bar_M = 0.5 * (sq(ML_M) + sq(MR_M));
      R M2Bar_P = 0.5 * (sq(ML_P) + sq(MR_P));
      R M2Zero_M = fmin2(R(1.0), fmax2(M2Bar_M, R(MInf)));
      R M2Zero_P = fmin2(R(1.0), fmax2(M2Bar_P, R(MInf)));
      R MZero_M = xsqrt(M2Zero_M), MZero_P = xsqrt(M2Zero_P);
      R FA_M = MZero_M * (2.0 - MZero_M), FA_P = MZero_P * (2.0 - MZero_P);
      R MF1P_L_M = 0.5 * (ML_M + xabs(ML_M)), MF1N_R_M = 0.5 * (MR_M - xabs(MR_M));
      R MF1P_L_P = 0.5 * (ML_P + xabs(ML_P)), MF1N_R_P = 0.5 * (MR_P - xabs(MR_P));
      R MF2P_L_M = 0.25 * sq(ML_M + 1.0), MF2N_L_M = -0.25 * sq(ML_M - 1.0);
      R MF2P_R_M = 0.25 * sq(MR_M + 1.0), MF2N_R_M = -0.25 * sq(MR_M - 1.0);
      R MF2P_L_P = 0.25 * sq(ML_P + 1.0), MF2N_L_P = -0.25 * sq(ML_P - 1.0);
      R MF2P_R_P = 0.25 * sq(MR_P + 1.0), MF2N_R_P = -0.25 * sq(MR_P - 1.0);
      R MF4P_L_M = (xabs(ML_M) >= 1.0) ? MF1P_L_M : MF2P_L_M * (1.0 - 16.0 * LiouBeta * MF2N_L_M);
      R MF4N_R_M = (xabs(MR_M) >= 1.0) ? MF1N_R_M : MF2N_R_M * (1.0 + 16.0 * LiouBeta * MF2P_R_M);
      R MF4P_L_P = (xabs(ML_P) >= 1.0) ? MF1P_L_P : MF2P_L_P * (1.0 - 16.0 * LiouBeta * MF2N_L_P);
      R MF4N_R_P = (xabs(MR_P) >= 1.0) ? MF1N_R_P : MF2N_R_P * (1.0 + 16.0 * LiouBeta * MF2P_R_P);
      const R ModifiedZeta = 1.0;
      R MPress_M, MPress_P;
      if (SH(i, s)) {
        MPress_M = LiouKpS[q] * fmax2(R(1.0 - M2Bar_M), R(0.0)) *
                   ((PSR_M[q] - HPSR_M[q]) - (PSL_M[q] - HPSL_M[q])) /
                   (MeanRhoS_M * CS_M[i] * (FA_M * CS_M[i] + ModifiedZeta * A1(c.dAlt_C, i) / DtIn));
        MPress_P = LiouKpS[q] * fmax2(R(1.0 - M2Bar_P), R(0.0)) *
                   ((PSR_P[q] - HPSR_P[q]) - (PSL_P[q] - HPSL_P[q])) /
                   (MeanRhoS_P * CS_P[i] * (FA_P * CS_P[i] + ModifiedZeta * A1(c.dAlt_C, i) / DtIn));
      } else {
        MPress_P = LiouKpS[q] * fmax2(R(1.0 - M2Bar_P), R(0.0)) * (PSR_P[q] - PSL_P[q]) /
                   (MeanRhoS_P * CS_P[i] * (FA_P * CS_P[i] + ModifiedZeta * A1(c.dAlt_C, i) / DtIn));
        MPress_M = LiouKpS[q] * fmax2(R(1.0 - M2Bar_M), R(0.0)) * (PSR_M[q] - PSL_M[q]) /
                   (MeanRhoS_M * CS_M[i] * (FA_M * CS_M[i] + ModifiedZeta * A1(c.dAlt_C, i) / DtIn));
      }
      R IM_M = MF4P_L_M + MF4N_R_M - MPress_M;
      R IM_P = MF4P_L_P + MF4N_R_P - MPress_P;
      NumV_M[q] = CS_M[i] * IM_M;
      NumV_P[q] = CS_P[i] * IM_P;
      if (SH(i, s)) {
        NumP_P[q] = (MeanPS_P - MeanHPS_P) -
                    0.5 * Ku[q] * CS_P[i] * ((RhoSR_P[q]) * VR_P[q] - (RhoSL_P[q]) * VL_P[q]);
        NumP_M[q] = (MeanPS_M - MeanHPS_M) -
                    0.5 * Ku[q] * CS_M[i] * ((RhoSR_M[q]) * VR_M[q] - (RhoSL_M[q]) * VL_M[q]);
      } else {
        NumP_P[q] = (MeanPS_P) - 0.5 * Ku[q] * CS_P[i] * ((RhoSR_P[q]) * VR_P[q] - (RhoSL_P[q]) * VL_P[q]);
        NumP_M[q] = (MeanPS_M) - 0.5 * Ku[q] * CS_M[i] * ((RhoSR_M[q]) * VR_M[q] - (RhoSL_M[q]) * VL_M[q]);
      }
      if (NumV_P[q] >= 0.0) {
        RhoSFlux_P[q] = (RhoSL_P[q] * NumV_P[q]);
        MomSFlux_P[q] = (RhoSL_P[q] * VL_P[q] * NumV_P[q]);
      } else {
        RhoSFlux_P[q] = (RhoSR_P[q] * NumV_P[q]);
        MomSFlux_P[q] = (RhoSR_P[q] * VR_P[q] * NumV_P[q]);
      }
      if (NumV_M[q] >= 0.0) {
        RhoSFlux_M[q] = (RhoSL_M[q] * NumV_M[q]);
        MomSFlux_M[q] = (RhoSL_M[q] * VL_M[q] * NumV_M[q]);
      } else {
        RhoSFlux_M[q] = (RhoSR_M[q] * NumV_M[q]);
        MomSFlux_M[q] = (RhoSR_M[q] * VR_M[q] * NumV_M[q]);
      }
    }
  }
  // bulk fluxes (:1960-2026)
  std::vector<R> BulkV_P(N1, R(0.0)), BulkV_M(N1, R(0.0));
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = 1; i <= nAlts; ++i) {
      const int q = J(s, i);
      BulkV_P[i] = BulkV_P[i] + (RhoSL_P[q] + RhoSR_P[q]) * NumV_P[q] / (RhoL_P[i] + RhoR_P[i]);
      BulkV_M[i] = BulkV_M[i] + (RhoSL_M[q] + RhoSR_M[q]) * NumV_M[q] / (RhoL_M[i] + RhoR_M[i]);
    }
  std::vector<R> EF_P(N1), EF_M(N1), Mom_P(3 * N1), Mom_M(3 * N1);
  for (int i = 1; i <= nAlts; ++i) {
    if (BulkV_P[i] >= 0.0) {
      EF_P[i] = (EL_P[i] + PL_P[i]) * BulkV_P[i];
      for (int d = 1; d <= 3; ++d) Mom_P[(d - 1) * N1 + i] = RhoL_P[i] * VG(VGL_P, d, i) * BulkV_P[i];
    } else {
      EF_P[i] = (ER_P[i] + PR_P[i]) * BulkV_P[i];
      for (int d = 1; d <= 3; ++d) Mom_P[(d - 1) * N1 + i] = RhoR_P[i] * VG(VGR_P, d, i) * BulkV_P[i];
    }
    if (BulkV_M[i] >= 0.0) {
      EF_M[i] = (EL_M[i] + PL_M[i]) * BulkV_M[i];
      for (int d = 1; d <= 3; ++d) Mom_M[(d - 1) * N1 + i] = RhoL_M[i] * VG(VGL_M, d, i) * BulkV_M[i];
    } else {
      EF_M[i] = (ER_M[i] + PR_M[i]) * BulkV_M[i];
      for (int d = 1; d <= 3; ++d) Mom_M[(d - 1) * N1 + i] = RhoR_M[i] * VG(VGR_M, d, i) * BulkV_M[i];
    }
  }
  // spherical geometry (:2029-2068)
  for (int i = 1; i <= nAlts; ++i) {
    R LeftRadius = 0.5 * (A1(RadDist, i) + A1(RadDist, i - 1));
    R RightRadius = 0.5 * (A1(RadDist, i) + A1(RadDist, i + 1));
    R AP = sq(RightRadius);
    R AM = sq(LeftRadius);
    R Vol = (1.0 / 3.0) * (xpow(RightRadius, 3.0) - xpow(LeftRadius, 3.0));
    for (int s = 1; s <= nSpecies; ++s) {
      const int q = J(s, i);
      RhoSFlux[q] = ((AP)*RhoSFlux_P[q] - (AM)*RhoSFlux_M[q]) / Vol;
      MomentumSFlux[q] = ((AP)*MomSFlux_P[q] - (AM)*MomSFlux_M[q]) / Vol;
      MomentumSFlux[q] = MomentumSFlux[q] + (NumP_P[q] - NumP_M[q]) / A1(c.dAlt_C, i);
    }
    EnergyFlux[i] = ((AP)*EF_P[i] - (AM)*EF_M[i]) / Vol;
    for (int d = 1; d <= 3; ++d)
      MomentumFlux[(d - 1) * N1 + i] = (AP * Mom_P[(d - 1) * N1 + i] - AM * Mom_M[(d - 1) * N1 + i]) / Vol;
  }
}

// advance_vertical_1stage_ausm, vertical_solver_ausm.f90:436-999
template <class R>
void ausm_stage(const Column<R>& c, const GitmVertParams& prm, double DtIn, const R* LogRho,
                const R* LogNS, const R* Vel_GD, const R* Temp, R* NewLogRho, R* NewLogNS, R* NewVel_GD,
                R* NewTemp, const R* LogINS, R* NewLogINS, const R* IVel, const R* VertVel,
                R* NewVertVel, uint32_t& status) {
  const Planet& P = planet();
  const int nAlts = c.nAlts;
  const int G = c.G;
  const double Beta = prm.beta_limiter;
  const int N1 = nAlts + 1;

  std::vector<R> EffectiveGravity(G), NS(nSpecies * G), Rho(G), RadialDistance(G), NT(G), Press(G);
  for (int i = -1; i <= nAlts + 2; ++i)
    A1(EffectiveGravity, i) = A1(c.Gravity, i) + c.Centrifugal / A1(c.InvR, i);
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) A2(NS, i, s) = xexp(A2(LogNS, i, s));
  for (int i = -1; i <= nAlts + 2; ++i) A1(Rho, i) = xexp(A1(LogRho, i));
  for (int i = -1; i <= nAlts + 2; ++i) A1(RadialDistance, i) = 1.0 / A1(c.InvR, i);
  for (int i = -1; i <= nAlts + 2; ++i) A1(NT, i) = 0.0;
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) A1(NT, i) = A1(NT, i) + A2(NS, i, s);
  for (int i = -1; i <= nAlts + 2; ++i) A1(Press, i) = A1(NT, i) * Boltzmanns_Constant * A1(Temp, i);

  // the sweeps whose results are read (:580-640)
  std::vector<R> GradTemp(N1), DiffTmp(N1), GradTmp(N1);
  rusanov_alts(c, Temp, GradTemp.data(), DiffTmp.data(), Beta);
  std::vector<R> GradVel(3 * N1), DiffVel(3 * N1);
  for (int d = 1; d <= 2; ++d)
    rusanov_alts(c, &Vel_GD[(d - 1) * G], &GradVel[(d - 1) * N1], &DiffVel[(d - 1) * N1], Beta);
  std::vector<R> GradLogINS(nIonsAdvect * N1), DiffLogINS(nIonsAdvect * N1);
  for (int s = 1; s <= nIonsAdvect; ++s)
    rusanov_alts(c, &LogINS[(s - 1) * G], &GradLogINS[(s - 1) * N1], &DiffLogINS[(s - 1) * N1], Beta);

  // GradLogConS (:644-686)
  std::vector<R> LogConS(nSpecies * G), GradLogConS(nSpecies * nAlts);
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i)
      A2(LogConS, i, s) = xlog(P.Mass[s] * A2(NS, i, s) / A1(Rho, i));
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    R MC[5];
    gradlogcons_coefs(c, iAlt, MC);
    for (int s = 1; s <= nSpecies; ++s)
      GradLogConS[(s - 1) * nAlts + iAlt - 1] =
          MC[0] * A2(LogConS, iAlt - 2, s) + MC[1] * A2(LogConS, iAlt - 1, s) +
          MC[2] * A2(LogConS, iAlt, s) + MC[3] * A2(LogConS, iAlt + 1, s) +
          MC[4] * A2(LogConS, iAlt + 2, s);
  }

  // hydrostatic species background (:714-751)
  std::vector<R> HydroNS = NS;
  for (int s = 1; s <= nSpecies; ++s) {
    for (int iAlt = 1; iAlt <= nAlts + 2; ++iAlt) {
      R MeanMass = P.Mass[s];
      R MeanGravity = 0.5 * (A1(EffectiveGravity, iAlt) + A1(EffectiveGravity, iAlt - 1));
      R MeanTemp = 0.5 * (A1(Temp, iAlt) + A1(Temp, iAlt - 1));
      R InvScaleHeight = -1.0 * MeanMass * MeanGravity / (Boltzmanns_Constant * MeanTemp);
      A2(HydroNS, iAlt, s) = A2(HydroNS, iAlt - 1, s) * (A1(Temp, iAlt - 1) / A1(Temp, iAlt)) *
                             xexp(-1.0 * A1(c.dAlt_F, iAlt) * InvScaleHeight);
    }
    {
      const int iAlt = -1;
      R MeanMass = 0.5 * (A1(c.MeanMajorMass, -1) + A1(c.MeanMajorMass, 0));
      R MeanGravity = 0.5 * (A1(EffectiveGravity, iAlt + 1) + A1(EffectiveGravity, iAlt));
      R MeanTemp = 0.5 * (A1(Temp, iAlt + 1) + A1(Temp, iAlt));
      R InvScaleHeight = -1.0 * MeanMass * MeanGravity / (Boltzmanns_Constant * MeanTemp);
      A2(HydroNS, iAlt, s) = A2(HydroNS, iAlt + 1, s) * (A1(Temp, iAlt + 1) / A1(Temp, iAlt)) *
                             xexp(A1(c.dAlt_F, iAlt) * InvScaleHeight);
    }
  }
  std::vector<R> HydroPressureS(nSpecies * G), HydroRhoS(nSpecies * G), RhoS(nSpecies * G),
      MomentumS(nSpecies * G), PressureS(nSpecies * G), DeviationRhoS(nSpecies * G);
  std::vector<char> SubtractHydrostatic(nSpecies * G);
  for (int i = -1; i <= nAlts + 2; ++i)
    for (int s = 1; s <= nSpecies; ++s) {
      A2(HydroPressureS, i, s) = A2(HydroNS, i, s) * Boltzmanns_Constant * A1(Temp, i);
      A2(HydroRhoS, i, s) = P.Mass[s] * A2(HydroNS, i, s);
    }
  for (int s = 1; s <= nSpecies; ++s)
    for (int i = -1; i <= nAlts + 2; ++i) {
      A2(RhoS, i, s) = P.Mass[s] * A2(NS, i, s);
      A2(MomentumS, i, s) = P.Mass[s] * A2(NS, i, s) * A2(VertVel, i, s);
      A2(PressureS, i, s) = A2(NS, i, s) * A1(Temp, i) * Boltzmanns_Constant;
    }
  auto sq = [](const R& x) { return x * x; };
  std::vector<R> TotalEnergy(G), Momentum(3 * G);
  for (int i = -1; i <= nAlts + 2; ++i)
    A1(TotalEnergy, i) = A1(Press, i) / (A1(c.Gamma, i) - 1.0) +
                         0.5 * A1(Rho, i) *
                             (sq(A2(Vel_GD, i, iUp_)) + sq(A2(Vel_GD, i, iNorth_)) + sq(A2(Vel_GD, i, iEast_)));
  for (int d = 1; d <= 3; ++d)
    for (int i = -1; i <= nAlts + 2; ++i) A2(Momentum, i, d) = A1(Rho, i) * A2(Vel_GD, i, d);
  for (int i = -1; i <= nAlts + 2; ++i)
    for (int s = 1; s <= nSpecies; ++s) {
      R ratio = xabs(A2(RhoS, i, s) - A2(HydroRhoS, i, s)) / A2(RhoS, i, s);
      A2(DeviationRhoS, i, s) = A2(RhoS, i, s) - A2(HydroRhoS, i, s);
      A2(SubtractHydrostatic, i, s) = !(xabs(ratio) > 1.0);
    }

  std::vector<R> RhoSFlux(nSpecies * N1), MomentumSFlux(nSpecies * N1), EnergyFlux(N1),
      MomentumFlux(3 * N1);
  all_fluxes_hydro(c, prm, DtIn, RhoS.data(), PressureS.data(), HydroPressureS.data(), Temp, Vel_GD,
                   VertVel, RhoSFlux.data(), MomentumSFlux.data(), EnergyFlux.data(), MomentumFlux.data(),
                   RadialDistance.data(), SubtractHydrostatic);
  auto J = [&](int s, int i) { return (s - 1) * N1 + i; };

  // continuity (:844-862)
  std::vector<R> NewRhoS = RhoS;
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    for (int s = 1; s <= nSpecies; ++s) {
      A2(NewRhoS, iAlt, s) = A2(RhoS, iAlt, s) - DtIn * (RhoSFlux[J(s, iAlt)]);
      A2(NewLogNS, iAlt, s) = xlog(A2(NewRhoS, iAlt, s) / P.Mass[s]);
    }
    for (int s = 1; s <= nIonsAdvect; ++s)
      A2(NewLogINS, iAlt, s) = A2(NewLogINS, iAlt, s) -
                               DtIn * (A2(IVel, iAlt, iUp_) * GradLogINS[(s - 1) * N1 + iAlt]) +
                               DtIn * DiffLogINS[(s - 1) * N1 + iAlt];
  }
  std::vector<R> NewNS(nSpecies * G, R(0.0)), NewNT(G, R(0.0)), NewRho(G, R(0.0));
  for (int i = -1; i <= nAlts + 2; ++i)
    for (int s = 1; s <= nSpecies; ++s) {
      A2(NewNS, i, s) = A2(NewRhoS, i, s) / P.Mass[s];
      A1(NewRho, i) = A1(NewRho, i) + A2(NewRhoS, i, s);
      A1(NewNT, i) = A1(NewNT, i) + A2(NewNS, i, s);
    }

  // species momentum (:862-900); VertTau enters only through UseDamping's
  // module update, which this solver does not read
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    for (int s = 1; s <= nSpecies; ++s) {
      R NewMomentumS;
      if (!A2(SubtractHydrostatic, iAlt, s))
        NewMomentumS = A2(MomentumS, iAlt, s) - DtIn * (MomentumSFlux[J(s, iAlt)]) +
                       DtIn * A2(RhoS, iAlt, s) * A1(EffectiveGravity, iAlt);
      else
        NewMomentumS = A2(MomentumS, iAlt, s) - DtIn * (MomentumSFlux[J(s, iAlt)]) +
                       DtIn * A2(DeviationRhoS, iAlt, s) * A1(EffectiveGravity, iAlt);
      A2(NewVertVel, iAlt, s) = NewMomentumS / A2(NewRhoS, iAlt, s);
      A2(NewVertVel, iAlt, s) =
          A2(NewVertVel, iAlt, s) +
          DtIn * (A2(Vel_GD, iAlt, iNorth_) * A2(Vel_GD, iAlt, iNorth_) +
                  A2(Vel_GD, iAlt, iEast_) * A2(Vel_GD, iAlt, iEast_)) *
              A1(c.InvR, iAlt);
      if (prm.use_coriolis)
        A2(NewVertVel, iAlt, s) = A2(NewVertVel, iAlt, s) + DtIn * (c.Coriolis * A2(Vel_GD, iAlt, iEast_));
      A2(NewVertVel, iAlt, s) =
          A2(NewVertVel, iAlt, s) -
          DtIn * (prm.thermal_diff_coef[s - 1] * Boltzmanns_Constant * GradTemp[iAlt]) / P.Mass[s];
    }
  }
  // friction on the updated densities (:902-913)
  if (prm.use_neutral_friction) {
    std::vector<R> nVel(nSpecies * nAlts), NSs(nSpecies * nAlts), Ed(nAlts), NTs(nAlts), Ts(nAlts);
    for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
      Ed[iAlt - 1] = A1(c.EddyCoef, iAlt);
      NTs[iAlt - 1] = A1(NewNT, iAlt);
      Ts[iAlt - 1] = A1(Temp, iAlt);
      for (int s = 1; s <= nSpecies; ++s) {
        nVel[(s - 1) * nAlts + iAlt - 1] = A2(NewVertVel, iAlt, s);
        NSs[(s - 1) * nAlts + iAlt - 1] = A2(NewNS, iAlt, s);
      }
    }
    neutral_friction(DtIn, nVel.data(), Ed.data(), NTs.data(), NSs.data(), GradLogConS.data(), Ts.data(),
                     nAlts, true, status);
    for (int iAlt = 1; iAlt <= nAlts; ++iAlt)
      for (int s = 1; s <= nSpecies; ++s) A2(NewVertVel, iAlt, s) = nVel[(s - 1) * nAlts + iAlt - 1];
  }
  // clamp and bulk vertical wind over all cells (:916-941)
  for (int i = -1; i <= nAlts + 2; ++i)
    for (int s = 1; s <= nSpecies; ++s) {
      A2(NewVertVel, i, s) = fmax2(R(-prm.max_vertical_velocity), A2(NewVertVel, i, s));
      A2(NewVertVel, i, s) = fmin2(R(prm.max_vertical_velocity), A2(NewVertVel, i, s));
    }
  for (int i = -1; i <= nAlts + 2; ++i) A2(NewVel_GD, i, iUp_) = 0.0;
  for (int i = -1; i <= nAlts + 2; ++i)
    for (int s = 1; s <= nSpecies; ++s)
      A2(NewVel_GD, i, iUp_) = A2(NewVel_GD, i, iUp_) + A2(NewVertVel, i, s) * A2(NewRhoS, i, s) / A1(NewRho, i);
  // winds, energy, temperature (:944-986)
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    const R damp = 0.35 * xexp(-1.0 * (A1(c.Altitude, iAlt) - A1(c.Altitude, 0)) / (45.0e+03));
    R NewMom = A2(Momentum, iAlt, iEast_) - DtIn * (MomentumFlux[(iEast_ - 1) * N1 + iAlt]);
    A2(NewVel_GD, iAlt, iEast_) = NewMom / A1(NewRho, iAlt);
    A2(NewVel_GD, iAlt, iEast_) = A2(NewVel_GD, iAlt, iEast_) + damp * DtIn * DiffVel[(iEast_ - 1) * N1 + iAlt];
    NewMom = A2(Momentum, iAlt, iNorth_) - DtIn * (MomentumFlux[(iNorth_ - 1) * N1 + iAlt]);
    A2(NewVel_GD, iAlt, iNorth_) = NewMom / A1(NewRho, iAlt);
    A2(NewVel_GD, iAlt, iNorth_) =
        A2(NewVel_GD, iAlt, iNorth_) + damp * DtIn * DiffVel[(iNorth_ - 1) * N1 + iAlt];
    R NewTotalEnergy = A1(TotalEnergy, iAlt) - DtIn * EnergyFlux[iAlt] +
                       DtIn * A1(Rho, iAlt) * A2(Vel_GD, iAlt, iUp_) * A1(EffectiveGravity, iAlt);
    R NewPress = (NewTotalEnergy - 0.5 * A1(NewRho, iAlt) *
                                       (sq(A2(NewVel_GD, iAlt, iUp_)) + sq(A2(NewVel_GD, iAlt, iNorth_)) +
                                        sq(A2(NewVel_GD, iAlt, iEast_)))) *
                 (A1(c.Gamma, iAlt) - 1.0);
    A1(NewTemp, iAlt) = NewPress / (Boltzmanns_Constant * A1(NewNT, iAlt));
  }
  for (int iAlt = 1; iAlt <= nAlts; ++iAlt) {
    R NewSumRho = 0.0;
    for (int s = 1; s <= nSpecies; ++s) NewSumRho = NewSumRho + P.Mass[s] * xexp(A2(NewLogNS, iAlt, s));
    A1(NewLogRho, iAlt) = xlog(NewSumRho);
  }
  (void)VertVel;
  (void)Press;
}

// advance_vertical_1d_ausm, vertical_solver_ausm.f90:26-433
template <class R>
void advance_vertical_1d_ausm(Column<R>& c, const GitmVertParams& prm, double Dt) {
  const int G = c.G;
  const int nAlts = c.nAlts;
  auto& st = c.status;
  set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                   c.LogINS.data(), c.VertVel.data(), st);
  std::vector<R>* S[6] = {&c.LogNS, &c.LogINS, &c.LogRho, &c.Vel_GD, &c.Temp, &c.VertVel};
  const int nf[6] = {nSpecies, nIons, 1, 3, 1, nSpecies};
  std::vector<R> Stage[5][6], New[6];
  for (int v = 0; v < 6; ++v) Stage[1][v] = *S[v];
  const double dts[4] = {0.5 * Dt, 0.5 * Dt, Dt, 0.5 * Dt};
  for (int k = 0; k < 4; ++k) {
    for (int v = 0; v < 6; ++v) New[v] = *S[v];
    ausm_stage(c, prm, dts[k], c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
               New[2].data(), New[0].data(), New[3].data(), New[4].data(), c.LogINS.data(), New[1].data(),
               c.IVel.data(), c.VertVel.data(), New[5].data(), st);
    if (k < 3) {
      // Stage(k+2) = Stage1 + (New - state), then the state takes it (:167-189 ...)
      for (int v = 0; v < 6; ++v) {
        Stage[k + 2][v].resize(S[v]->size());
        for (size_t i = 0; i < S[v]->size(); ++i)
          Stage[k + 2][v][i] = Stage[1][v][i] + (New[v][i] - (*S[v])[i]);
        *S[v] = Stage[k + 2][v];
      }
      set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                       c.LogINS.data(), c.VertVel.data(), st);
    }
  }
  // :381-420: ghosts keep Stage1, cells 1..nAlts take the RK combination
  for (int v = 0; v < 6; ++v) {
    std::vector<R> Final = Stage[1][v];
    for (int k = 1; k <= nf[v]; ++k)
      for (int i = 1; i <= nAlts; ++i) {
        const size_t q = size_t((k - 1) * G + i + 1);
        Final[q] = (1.0 / 3.0) * (-1.0 * Stage[1][v][q] + Stage[2][v][q] + 2.0 * Stage[3][v][q] +
                                  Stage[4][v][q] + (New[v][q] - (*S[v])[q]));
      }
    *S[v] = Final;
  }
  set_vertical_bcs(c, prm, c.LogRho.data(), c.LogNS.data(), c.Vel_GD.data(), c.Temp.data(),
                   c.LogINS.data(), c.VertVel.data(), st);
}

#undef A1
#undef A2

}  // namespace gvo
