// vert_ausm.cuh -- the AUSM stage of the vertical step (UseAUSMSolver), run
// by vert_step_kernel when the solver is GITM_SOLVER_AUSM.
//
// advance_vertical_1stage_ausm (vertical_solver_ausm.f90:436-999) with the
// AUSM+-up fluxes of calc_all_fluxes_hydro (:1093-2070) at both faces of the
// thread's cell.  Layout of the slope buffer (L.DL, 32 fields):
//   0..5   LogRhoS   (2nd-order "kt" slopes, calc_kt_facevalues :2073-2117)
//   6..11  LogPS     (kt)
//   12..17 LogHydroPressureS (kt)
//   18..23 VertVel   (kt)
//   24,25  Vel east / north (kt)
//   26     Gamma     (kt)
//   27     Temp      (4th-order slopes, calc_facevalues_alts_ausm)
//   28,29  Vel east / north (4th order)
//   30,31  ions 1, 2 (4th order, calc_rusanov_alts_rusanov)
// Values are formed in log space where the reference multiplies and takes
// the log: LogRhoS = log m + LogNS, LogPS = LogNS + log k + log T, and the
// hydrostatic species pressure (:714-751) is
//   log HydroPressureS(i) = LogNS(0) + log k + log T(0) + m_s Q(i),
//   Q(i) = sum_{j=1..i} dAlt_F(j) MeanGravity(j) / (k MeanTemp(j)),
// because the temperature ratios of the upward recurrence telescope.
#pragma once

namespace gv {

enum AusmSlope : int {
  AS_LRHOS = 0, AS_LPS = 6, AS_LHPS = 12, AS_W = 18, AS_VE = 24, AS_VN = 25, AS_GAM = 26,
  AS_T4 = 27, AS_VE4 = 28, AS_VN4 = 29, AS_I4 = 30
};
constexpr int SC_QB = 59;  // dAlt_F(-1) * InvScaleHeight of the bulk gas below cell 0

__device__ __forceinline__ double sqr(double x) { return x * x; }

// log HydroPressureS(i) - (LogNS(0) + log k + log T(0)) for species s
__device__ __forceinline__ double hydro_q(ColCtx c, int s, int i) {
  return (i < 0) ? c.sc(SC_QB) : c_k.mass[s] * c.col[c.L.QS + i + 1];
}

// the value of AUSM slope field f at cell i
__device__ __forceinline__ double ausm_field(ColCtx c, int f, int i) {
  if (f < AS_LPS) return c.x(F_LNS + f, i);  // LogRhoS - log m
  if (f < AS_LHPS) return c.x(F_LNS + f - AS_LPS, i) + c.col[c.L.LT + i + 1];  // LogPS - log k
  if (f < AS_W) return hydro_q(c, f - AS_LHPS, i);  // LogHPS - base
  if (f < AS_VE) return c.x(F_W + f - AS_W, i);
  if (f == AS_VE || f == AS_VE4) return c.x(F_VE, i);
  if (f == AS_VN || f == AS_VN4) return c.x(F_VN, i);
  if (f == AS_GAM) return c.gm(i);
  if (f == AS_T4) return c.x(F_T, i);
  return c.x(F_I + f - AS_I4, i);
}

// Phase A1: log T on every cell, and the prefix sum Q (one warp per column).
__device__ __forceinline__ void ausm_prefix(ColCtx c, int lane) {
  const int nA = c.L.nAlts;
  double* Q = c.col + c.L.QS + 1;  // Q[i]
  double carry = 0.0;
  if (lane == 0) Q[0] = 0.0;
  for (int base = 1; base <= nA + 2; base += 32) {
    const int j = base + lane;
    double t = 0.0;
    if (j <= nA + 2) {
      const double mg = 0.5 * (c.g(GC_GRAV, j) + c.sc(SC_CENT) * c.g(GC_R, j) + c.g(GC_GRAV, j - 1) +
                               c.sc(SC_CENT) * c.g(GC_R, j - 1));
      const double mt = 0.5 * (c.x(F_T, j) + c.x(F_T, j - 1));
      t = c.dAF(j) * mg / (KB * mt);
    }
    for (int off = 1; off < 32; off <<= 1) {
      const double u = __shfl_up_sync(0xffffffffu, t, off);
      if (lane >= off) t += u;
    }
    if (j <= nA + 2) Q[j] = carry + t;
    carry += __shfl_sync(0xffffffffu, t, 31);
  }
  if (lane == 0) {
    // cell -1 from cell 0 with the mean major mass (:734-742)
    const double MeanMass = 0.5 * (c.sc(SC_MMM_M1) + c.sc(SC_MMM_0));
    const double MeanGravity = 0.5 * (c.sc(SC_EG + 1) + c.sc(SC_EG + 0));
    const double MeanTemp = 0.5 * (c.x(F_T, 0) + c.x(F_T, -1));
    const double ish = -1.0 * MeanMass * MeanGravity / (KB * MeanTemp);
    c.sc(SC_QB) = c.dAF(-1) * ish;
  }
}

// Phase A2: slope of AUSM field f at cell i (0..nAlts+1).
__device__ __forceinline__ double ausm_slope(ColCtx c, int f, int i, double beta) {
  const int nA = c.L.nAlts;
  const double vm = ausm_field(c, f, i - 1), v0 = ausm_field(c, f, i), vp = ausm_field(c, f, i + 1);
  const bool fourth = (f >= AS_T4) && i >= 1 && i <= nA;
  if (!fourth) return limiter_mc((vp - v0) * c.g(GC_IDF, i + 1), (v0 - vm) * c.g(GC_IDF, i), beta);
  const double vmm = ausm_field(c, f, i - 2), vpp = ausm_field(c, f, i + 2);
  const double up = c.g(GC_H2, i + 1) * (0.6250000 * (vp - v0) - 0.0416667 * (vpp - vm));
  const double dn = c.g(GC_H2, i) * (0.6250000 * (v0 - vm) - 0.0416667 * (vp - vmm));
  return limiter_mc(up, dn, beta);
}

// kt face values of a field at the lower (M) and upper (P) faces of cell i:
// left/right states (calc_kt_facevalues :2105-2111)
struct Faces {
  double lm, rm, lp, rp;
};
__device__ __forceinline__ Faces kt_faces(ColCtx c, int f, int i, double vm, double v0, double vp) {
  const double* d = &c.col[c.L.DL + f * (c.L.nAlts + 2)];
  // halves of the cell widths: a product with 0.5 is exact, so d * (0.5 dF)
  // rounds like (0.5 d) dF
  const double hm = 0.5 * c.dAF(i - 1), h0 = 0.5 * c.dAF(i), hp = 0.5 * c.dAF(i + 1);
  Faces r;
  r.lm = fma(d[i - 1], hm, vm);
  r.rm = fma(-d[i], h0, v0);
  r.lp = fma(d[i], h0, v0);
  r.rp = fma(-d[i + 1], hp, vp);
  return r;
}

// Rusanov gradient and dissipation from the 4th-order slopes (calc_rusanov_alts_*)
__device__ __forceinline__ void ausm_sweep(ColCtx c, int fslope, int ffield, int i, double fc0,
                                           double fc1, double& grad, double& diff) {
  const double* v = &c.col[c.xo + ffield * c.L.G + 1];
  const double* d = &c.col[c.L.DL + fslope * (c.L.nAlts + 2)];
  const double hF0 = 0.5 * c.dAF(i), hF1 = 0.5 * c.dAF(i + 1), idc = c.g(GC_IDC, i);
  const double L0 = fma(d[i - 1], hF0, v[i - 1]);
  const double R0 = fma(-d[i], hF0, v[i]);
  const double L1 = fma(d[i], hF1, v[i]);
  const double R1 = fma(-d[i + 1], hF1, v[i + 1]);
  grad = (L1 + R1 - L0 - R0) * (0.5 * idc);
  diff = (fc1 * (R1 - L1) - fc0 * (R0 - L0)) * idc;
}

// Per-species face states of cell i.
struct SpeciesFaces {
  Faces rho, ps, hps, w;
};
__device__ __forceinline__ void species_faces(ColCtx c, int s, int i, double logk, bool with_p,
                                              bool with_h, SpeciesFaces& o, bool with_rho = true) {
  const double lm = c_k.log_mass[s];
  if (with_rho) {
    const int f = AS_LRHOS + s;
    Faces t = kt_faces(c, f, i, c.x(F_LNS + s, i - 1), c.x(F_LNS + s, i), c.x(F_LNS + s, i + 1));
    o.rho.lm = exp(lm + t.lm);
    o.rho.rm = exp(lm + t.rm);
    o.rho.lp = exp(lm + t.lp);
    o.rho.rp = exp(lm + t.rp);
  }
  if (with_p) {
    const int f = AS_LPS + s;
    Faces t = kt_faces(c, f, i, ausm_field(c, f, i - 1), ausm_field(c, f, i), ausm_field(c, f, i + 1));
    o.ps.lm = exp(logk + t.lm);
    o.ps.rm = exp(logk + t.rm);
    o.ps.lp = exp(logk + t.lp);
    o.ps.rp = exp(logk + t.rp);
  }
  o.hps = Faces{0.0, 0.0, 0.0, 0.0};
  if (with_h) {
    const int f = AS_LHPS + s;
    const double base = c.x(F_LNS + s, 0) + logk + c.col[c.L.LT + 1];  // LogNS(0) + log k + log T(0)
    Faces t = kt_faces(c, f, i, hydro_q(c, s, i - 1), hydro_q(c, s, i), hydro_q(c, s, i + 1));
    o.hps.lm = exp(base + t.lm);
    o.hps.rm = exp(base + t.rm);
    o.hps.lp = exp(base + t.lp);
    o.hps.rp = exp(base + t.rp);
  }
  {
    const int f = AS_W + s;
    o.w = kt_faces(c, f, i, c.x(F_W + s, i - 1), c.x(F_W + s, i), c.x(F_W + s, i + 1));
  }
}

// AUSM+-up numerical velocity (Mach split, pressure diffusion) at one face
// and the species flux pair; (:1660-1937).
__device__ __forceinline__ void species_face_flux(double rl, double rr, double pl, double pr, double hl,
                                                  double hr, double wl, double wr, double cs, double kp,
                                                  double ku, double dzdt, bool subtract, double& nv,
                                                  double& rflux, double& mflux, double& np) {
  const double MInf = 1.0e-19;
  const double LiouBeta = 1.0 / 8.0;
  const double Ml = wl / cs, Mr = wr / cs;
  const double M2Bar = 0.5 * (sqr(Ml) + sqr(Mr));
  const double M2Zero = fmin(1.0, fmax(M2Bar, MInf));
  const double MZero = sqrt(M2Zero);
  const double FA = MZero * (2.0 - MZero);
  const double MF1P_L = 0.5 * (Ml + fabs(Ml)), MF1N_R = 0.5 * (Mr - fabs(Mr));
  const double MF2P_L = 0.25 * sqr(Ml + 1.0), MF2N_L = -0.25 * sqr(Ml - 1.0);
  const double MF2P_R = 0.25 * sqr(Mr + 1.0), MF2N_R = -0.25 * sqr(Mr - 1.0);
  const double MF4P_L = (fabs(Ml) >= 1.0) ? MF1P_L : MF2P_L * (1.0 - 16.0 * LiouBeta * MF2N_L);
  const double MF4N_R = (fabs(Mr) >= 1.0) ? MF1N_R : MF2N_R * (1.0 + 16.0 * LiouBeta * MF2P_R);
  const double meanrho = 0.5 * (rl + rr);
  const double dp = subtract ? ((pr - hr) - (pl - hl)) : (pr - pl);
  const double MPress = kp * fmax(1.0 - M2Bar, 0.0) * dp / (meanrho * cs * (FA * cs + 1.0 * dzdt));
  nv = cs * (MF4P_L + MF4N_R - MPress);
  const double meanp = 0.5 * (pl + pr);
  const double base = subtract ? (meanp - 0.5 * (hl + hr)) : meanp;
  np = base - 0.5 * ku * cs * (rr * wr - rl * wl);
  if (nv >= 0.0) {
    rflux = rl * nv;
    mflux = rl * wl * nv;
  } else {
    rflux = rr * nv;
    mflux = rr * wr * nv;
  }
}

// advance_vertical_1stage_ausm (vertical_solver_ausm.f90:436-999) at interior
// cell i with stage step dtk; emit(f, New - state) takes each new value.
// The face fluxes of calc_all_fluxes_hydro are formed at the cell's two
// faces in two passes over the species: the first sums the bulk face states
// (densities, pressures, mass-weighted vertical wind), which set the Liou
// sound speed; the second forms the species fluxes and applies them.
template <class Emit>
__device__ __forceinline__ void ausm_cell(ColCtx c, int i, const GitmVertParams& prm, double dtk,
                                          double eddy, double ivup, Emit&& emit, uint32_t* st = nullptr) {
  const int nA = c.L.nAlts;
  (void)nA;
  const double logk = c_k.log_kb;
  const double T = c.x(F_T, i), VE = c.x(F_VE, i), VN = c.x(F_VN, i), VU = c.x(F_VU, i);
  const double LR = c.x(F_LRHO, i);
  const double EG = c.g(GC_GRAV, i) + c.sc(SC_CENT) * c.g(GC_R, i);
  const double invr = c.g(GC_INVR, i);
  const double gam = c.gm(i);
  const double Rho = exp(LR);

  // Rusanov sweeps whose results the stage reads (:580-640)
  const double fc0 = 0.5 * fmax(c.cm(i - 1), c.cm(i));
  const double fc1 = 0.5 * fmax(c.cm(i), c.cm(i + 1));
  double gT, dT, gE, dE, gN, dN;
  ausm_sweep(c, AS_T4, F_T, i, fc0, fc1, gT, dT);
  ausm_sweep(c, AS_VE4, F_VE, i, fc0, fc1, gE, dE);
  ausm_sweep(c, AS_VN4, F_VN, i, fc0, fc1, gN, dN);
  (void)gE;
  (void)gN;
#pragma unroll
  for (int s = 0; s < NADV; ++s) {
    double gI, dI;
    ausm_sweep(c, AS_I4 + s, F_I + s, i, fc0, fc1, gI, dI);
    const double I = c.x(F_I + s, i);
    emit(F_I + s, (I - dtk * (ivup * gI) + dtk * dI) - I);  // :857-860
  }

  // cell values (:560-575, 752-790)
  double ns[NS];
  double NT = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    ns[s] = exp(c.x(F_LNS + s, i));
    NT = NT + ns[s];
  }
  const double Press = NT * KB * T;
  const double TotalEnergy = Press / (gam - 1.0) + 0.5 * Rho * (VU * VU + VN * VN + VE * VE);
  const double MomE = Rho * VE, MomN = Rho * VN;
  // hydrostatic species densities relative to the cell (:714-790):
  // log HydroNS(i) = LogNS(0) + log T(0) - log T(i) + m_s Q(i)
  const double lt0 = c.col[c.L.LT + 1], lti = c.col[c.L.LT + i + 1];
  unsigned sub = 0;  // SubtractHydrostatic bits
  double dev[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double RhoS = c_k.mass[s] * ns[s];
    const double HydroRhoS = c_k.mass[s] * exp(c.x(F_LNS + s, 0) + lt0 - lti + hydro_q(c, s, i));
    dev[s] = RhoS - HydroRhoS;
    const double ratio = fabs(RhoS - HydroRhoS) / RhoS;
    if (!(fabs(ratio) > 1.0)) sub |= 1u << s;
  }

  // ---- pass 1: bulk face states
  double RhoLM = 0.0, RhoRM = 0.0, RhoLP = 0.0, RhoRP = 0.0;
  double PLM = 0.0, PRM = 0.0, PLP = 0.0, PRP = 0.0;
  double WLM = 0.0, WRM = 0.0, WLP = 0.0, WRP = 0.0;  // sums of RhoS * VertVel
  // one species at a time: the fully unrolled passes made a body the
  // instruction cache could not hold (2.76 -> 3.33 M column-steps/s)
  // the density and pressure face states of each species, kept from this
  // pass for the flux pass (per-thread memory, cached)
  double fst[NS][8];
#pragma unroll 1
  for (int s = 0; s < NS; ++s) {
    SpeciesFaces f;
    species_faces(c, s, i, logk, true, false, f);
    fst[s][0] = f.rho.lm;
    fst[s][1] = f.rho.rm;
    fst[s][2] = f.rho.lp;
    fst[s][3] = f.rho.rp;
    fst[s][4] = f.ps.lm;
    fst[s][5] = f.ps.rm;
    fst[s][6] = f.ps.lp;
    fst[s][7] = f.ps.rp;
    RhoLM = RhoLM + f.rho.lm;
    RhoRM = RhoRM + f.rho.rm;
    RhoLP = RhoLP + f.rho.lp;
    RhoRP = RhoRP + f.rho.rp;
    PLM = PLM + f.ps.lm;
    PRM = PRM + f.ps.rm;
    PLP = PLP + f.ps.lp;
    PRP = PRP + f.ps.rp;
    WLM = WLM + f.rho.lm * f.w.lm;
    WRM = WRM + f.rho.rm * f.w.rm;
    WLP = WLP + f.rho.lp * f.w.lp;
    WRP = WRP + f.rho.rp * f.w.rp;
  }
  // bulk face winds (:1503-1530): the up component is the mass-weighted species wind
  const double ULM = WLM / RhoLM, URM = WRM / RhoRM, ULP = WLP / RhoLP, URP = WRP / RhoRP;
  const Faces fE = kt_faces(c, AS_VE, i, c.x(F_VE, i - 1), VE, c.x(F_VE, i + 1));
  const Faces fN = kt_faces(c, AS_VN, i, c.x(F_VN, i - 1), VN, c.x(F_VN, i + 1));
  const Faces fG = kt_faces(c, AS_GAM, i, c.gm(i - 1), gam, c.gm(i + 1));
  // energies, enthalpies (:1533-1565) and the Liou interface sound speed (:1568-1655)
  auto ke = [](double u, double e, double n) { return u * u + e * e + n * n; };
  const double KLM = ke(ULM, fE.lm, fN.lm), KRM = ke(URM, fE.rm, fN.rm);
  const double KLP = ke(ULP, fE.lp, fN.lp), KRP = ke(URP, fE.rp, fN.rp);
  auto enthalpy = [](double g, double P, double rho, double k2) { return 0.5 * k2 + (g / (g - 1.0)) * P / rho; };
  auto csound = [](double g, double H) { return sqrt(2.0 * ((g - 1.0) / (g + 1.0)) * H); };
  double CSM, CSP;
  {
    const double sl = csound(fG.lm, enthalpy(fG.lm, PLM, RhoLM, KLM));
    const double sr = csound(fG.rm, enthalpy(fG.rm, PRM, RhoRM, KRM));
    CSM = fmin(sqr(sl) / fmax(sl, ULM), sqr(sr) / fmax(sr, -1.0 * URM));
  }
  {
    const double sl = csound(fG.lp, enthalpy(fG.lp, PLP, RhoLP, KLP));
    const double sr = csound(fG.rp, enthalpy(fG.rp, PRP, RhoRP, KRP));
    CSP = fmin(sqr(sl) / fmax(sl, ULP), sqr(sr) / fmax(sr, -1.0 * URP));
  }

  // ---- pass 2: species fluxes, continuity and species momentum (:844-900)
  const double AP = c.ga(GA_AP, i), AM = c.ga(GA_AM, i), Vol = c.ga(GA_VOL, i);
  const double dAltC = c.ga(GA_DALTC, i);
  const double kp = c.ga(GA_KP, i), ku = c.ga(GA_KU, i);
  const double dzdt = dAltC / dtk;
  const double hz = dtk * (VN * VN + VE * VE) * invr;
  double BulkVM = 0.0, BulkVP = 0.0;
  double nrs[NS], wv[NS];
#pragma unroll 1
  for (int s = 0; s < NS; ++s) {
    const bool sh = (sub >> s) & 1u;
    SpeciesFaces f;
    species_faces(c, s, i, logk, false, sh, f, false);
    f.rho = Faces{fst[s][0], fst[s][1], fst[s][2], fst[s][3]};
    f.ps = Faces{fst[s][4], fst[s][5], fst[s][6], fst[s][7]};
    double nvM, rfM, mfM, npM, nvP, rfP, mfP, npP;
    species_face_flux(f.rho.lm, f.rho.rm, f.ps.lm, f.ps.rm, f.hps.lm, f.hps.rm, f.w.lm, f.w.rm, CSM, kp, ku, dzdt,
                      sh, nvM, rfM, mfM, npM);
    species_face_flux(f.rho.lp, f.rho.rp, f.ps.lp, f.ps.rp, f.hps.lp, f.hps.rp, f.w.lp, f.w.rp, CSP, kp, ku, dzdt,
                      sh, nvP, rfP, mfP, npP);
    BulkVP = BulkVP + (f.rho.lp + f.rho.rp) * nvP / (RhoLP + RhoRP);
    BulkVM = BulkVM + (f.rho.lm + f.rho.rm) * nvM / (RhoLM + RhoRM);
    const double RhoSFlux = (AP * rfP - AM * rfM) / Vol;
    double MomSFlux = (AP * mfP - AM * mfM) / Vol;
    MomSFlux = MomSFlux + (npP - npM) / dAltC;
    const double RhoS = c_k.mass[s] * ns[s];
    const double Ws = c.x(F_W + s, i);
    const double NewRhoS = RhoS - dtk * RhoSFlux;
    const double Ls = c.x(F_LNS + s, i);
    emit(F_LNS + s, log(NewRhoS / c_k.mass[s]) - Ls);
    const double MomS = RhoS * Ws;
    const double NewMomS = MomS - dtk * MomSFlux + dtk * (sh ? dev[s] : RhoS) * EG;
    double w = NewMomS / NewRhoS;
    w = w + hz;
    if (prm.use_coriolis) w = w + dtk * (c.sc(SC_CORI) * VE);
    w = w - dtk * (prm.thermal_diff_coef[s] * KB * gT) / c_k.mass[s];
    nrs[s] = NewRhoS;
    wv[s] = w;
  }
  double NewRho = 0.0, NewNT = 0.0, nns[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    nns[s] = nrs[s] / c_k.mass[s];
    NewRho = NewRho + nrs[s];
    NewNT = NewNT + nns[s];
  }
  // friction on the updated densities with the stage temperature (:902-913)
  if (prm.use_neutral_friction) {
    double glc[NS];
    grad_log_cons(c, i, glc);
    friction_solve(dtk, nns, T, eddy, glc, wv, st);
  }
  // clamp and bulk vertical wind (:916-941)
  double NewVU = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double w = fmax(-prm.max_vertical_velocity, wv[s]);
    w = fmin(prm.max_vertical_velocity, w);
    emit(F_W + s, w - c.x(F_W + s, i));
    NewVU = NewVU + w * nrs[s] / NewRho;
  }
  emit(F_VU, NewVU - VU);

  // bulk energy and horizontal momentum fluxes (:1960-2026, 2041-2068)
  double EFP, EFM, MEP, MEM, MNP, MNM;
  if (BulkVP >= 0.0) {
    EFP = ((1.0 / (fG.lp - 1.0)) * PLP + 0.5 * RhoLP * KLP + PLP) * BulkVP;
    MEP = RhoLP * fE.lp * BulkVP;
    MNP = RhoLP * fN.lp * BulkVP;
  } else {
    EFP = ((1.0 / (fG.rp - 1.0)) * PRP + 0.5 * RhoRP * KRP + PRP) * BulkVP;
    MEP = RhoRP * fE.rp * BulkVP;
    MNP = RhoRP * fN.rp * BulkVP;
  }
  if (BulkVM >= 0.0) {
    EFM = ((1.0 / (fG.lm - 1.0)) * PLM + 0.5 * RhoLM * KLM + PLM) * BulkVM;
    MEM = RhoLM * fE.lm * BulkVM;
    MNM = RhoLM * fN.lm * BulkVM;
  } else {
    EFM = ((1.0 / (fG.rm - 1.0)) * PRM + 0.5 * RhoRM * KRM + PRM) * BulkVM;
    MEM = RhoRM * fE.rm * BulkVM;
    MNM = RhoRM * fN.rm * BulkVM;
  }
  const double EnergyFlux = (AP * EFP - AM * EFM) / Vol;
  const double MomFluxE = (AP * MEP - AM * MEM) / Vol;
  const double MomFluxN = (AP * MNP - AM * MNM) / Vol;

  // horizontal winds, energy and temperature (:944-986)
  const double damp = c.ga(GA_DAMP, i);
  double NewVE = (MomE - dtk * MomFluxE) / NewRho;
  NewVE = NewVE + damp * dtk * dE;
  double NewVN = (MomN - dtk * MomFluxN) / NewRho;
  NewVN = NewVN + damp * dtk * dN;
  emit(F_VE, NewVE - VE);
  emit(F_VN, NewVN - VN);
  const double NewTotalEnergy = TotalEnergy - dtk * EnergyFlux + dtk * Rho * VU * EG;
  const double NewPress =
      (NewTotalEnergy - 0.5 * NewRho * (NewVU * NewVU + NewVN * NewVN + NewVE * NewVE)) * (gam - 1.0);
  emit(F_T, NewPress / (KB * NewNT) - T);
  // LogRho = log(sum_s Mass_s exp(NewLogNS_s)) (:993-996), from the new species densities
  emit(F_LRHO, log(NewRho) - LR);
}

}  // namespace gv
