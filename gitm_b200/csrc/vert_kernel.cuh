// vert_kernel.cuh -- fused RK4 vertical-advance kernel (Rusanov solver).
//
// One CTA holds a tile of `nc` columns of one member in shared memory for a
// whole time step (and for `n_steps` consecutive steps): the gather of
// advance_vertical (advance_vertical.f90:80-155), the four explicit stages of
// advance_vertical_1d_rusanov (vertical_solver_rusanov.f90:10-384), the five
// set_vertical_bcs passes (set_vertical_bcs.Earth.f90:8-652) and the scatter
// (advance_vertical.f90:163-217) never leave the SM.
//
// Thread mapping.  The interior cells of the tile's columns are "items": item
// t < nc * nAlts owns column t / nAlts, cell t % nAlts + 1, for the whole step
// (its RK accumulator lives in its registers).  Set_vertical_bcs runs one warp
// per column with lanes over species / ions.  Whole-column passes (load,
// store, ghost resets) stride over all threads.
//
// Arithmetic is FP64 throughout.  Results agree with the reference's
// operation order to rounding: reciprocals replace some divisions, the
// friction matrix is formed without the cancelling NDensity factors, and its
// 6x6 system (strictly diagonally dominant by rows) is solved by LU without
// pivoting instead of ludcmp's implicit partial pivoting.
#pragma once

#include "vert_common.cuh"

namespace gv {

__constant__ Consts c_k;

// DiffExp(i,j) as an index into Consts::one_minus_e; a compile-time table so
// that fully unrolled loops select the power without indexing registers.
__device__ __forceinline__ int exp_index(int r, int q) {
  constexpr int t[NS][NS] = {{0, 0, 0, 0, 1, 2}, {0, 0, 1, 0, 1, 3}, {0, 1, 0, 0, 5, 4},
                             {0, 0, 0, 0, 0, 4}, {1, 1, 5, 0, 0, 4}, {2, 3, 4, 4, 4, 0}};
  return t[r][q];
}

// ------------------------------------------------------------ smem layout
struct Layout {
  int nAlts, G;
  int nsl;  // slope fields in DL: 18 (Rusanov) or 32 (AUSM)
  int X0, XP0, X1, XP1, O, OP, OGH, DL, TU, CM, GM, SC, LT, QS, stride;
};

constexpr int NSLOPE_AUSM = 32;

constexpr int NSC = 64;  // per-column scalars
enum Scalar : int {
  SC_CENT = 0, SC_CORI = 1, SC_SZA = 2, SC_MLAT = 3, SC_MMM_M1 = 4, SC_MMM_0 = 5,
  SC_PLASMA = 6, SC_HASLBC = 7,
  SC_LBC = 8,   // 8..27: lbc[2][10]
  SC_BCC = 28,  // 28..47: mesh coefficients, lower cells 0, -1 then upper nA+1, nA+2
  SC_DAF = 48,  // 48..53: dAlt_F at -1, 0, 1, nA, nA+1, nA+2
  SC_EG = 54    // 54..58: Gravity + Centrifugal / InvR at -1, 0, nA, nA+1, nA+2
};

// Per-column shared-memory slot (doubles): the stage state twice (a stage
// reads one buffer and writes the next), Orig, the limited slopes, the
// per-cell coefficients and the column scalars.  orig_global: Orig is kept
// in the CTA's slot of global scratch instead (it is read-only during a
// step), which leaves room for more columns per SM.
__host__ __device__ inline Layout make_layout(int nAlts, int solver = GITM_SOLVER_RUSANOV,
                                              bool orig_global = false) {
  Layout L;
  L.nAlts = nAlts;
  L.G = nAlts + 4;
  L.nsl = (solver == GITM_SOLVER_AUSM) ? NSLOPE_AUSM : NSTENCIL;
  const int G = L.G;
  int o = 0;
  L.X0 = o;  o += NF * G;
  L.XP0 = o; o += NPAS * NPC;
  L.X1 = o;  o += NF * G;
  L.XP1 = o; o += NPAS * NPC;
  L.O = o;   o += orig_global ? 0 : NF * G;
  L.OP = o;  o += orig_global ? 0 : NPAS * NPC;
  // orig_global: Orig's ghost cells (f * 4 + u, u over cells -1, 0,
  // nAlts+1, nAlts+2) and passive-ion cells stay here as well, for the
  // ghost reset after every stage
  L.OGH = o; o += orig_global ? NF * 4 + NPAS * NPC : 0;
  L.DL = o;  o += L.nsl * (nAlts + 2);
  L.TU = o;  o += G;
  L.CM = o;  o += G;
  L.GM = o;  o += G;
  L.SC = o;  o += NSC;
  // AUSM only: log T and the hydrostatic prefix sum of every cell
  L.LT = o;  o += (solver == GITM_SOLVER_AUSM) ? G : 0;
  L.QS = o;  o += (solver == GITM_SOLVER_AUSM) ? G : 0;
  L.stride = o;
  return L;
}

// Bytes of dynamic shared memory a tile of nc columns needs.
__host__ __device__ inline size_t smem_bytes(int nAlts, int nc, int solver = GITM_SOLVER_RUSANOV,
                                             bool orig_global = false) {
  Layout L = make_layout(nAlts, solver, orig_global);
  return size_t(L.stride) * nc * sizeof(double) + size_t(nc) * 2 * sizeof(uint32_t);
}

// Doubles of one column's Orig (the state and its passive-ion cells).
__host__ __device__ inline int orig_doubles(int nAlts) { return NF * (nAlts + 4) + NPAS * NPC; }

// passive-ion cell slot: -1,0,1 -> 0..2; nAlts-5..nAlts+2 -> 3..10
__device__ __forceinline__ int pcell(int i, int nAlts) {
  return (i <= 1) ? i + 1 : 3 + (i - (nAlts - 5));
}
__device__ __forceinline__ bool in_pcells(int i, int nAlts) {
  return i <= 1 || i >= nAlts - 5;
}

__device__ __forceinline__ bool photochemical(int s) { return s == 3 || s == 4; }  // N(4S), NO

// ModLimiter.f90:16-36, without branches: on same-sign slopes the smallest
// magnitude of beta u, beta d and (u + d) / 2 carries the common sign (the
// reference's min of the three when both are positive and max when both are
// negative, the same values since negation is exact); 0 otherwise.  Lanes
// whose cells take different cases do not split the warp.
__device__ __forceinline__ double limiter_mc(double u, double d, double beta) {
  const double m = fmin(fmin(fabs(beta * u), fabs(beta * d)), fabs((u + d) * 0.5));
  const bool pos = (u > 0.0) && (d > 0.0);
  const bool neg = !(u > 0.0) && (d < 0.0);
  return pos ? m : (neg ? -m : 0.0);
}

struct ColCtx {
  double* col;
  Layout L;
  const double* gridc;
  int gcols;
  int gc;   // grid column (0 when the member shares one grid)
  int xo;   // offset of the current stage buffer (X0 or X1)
  int xpo;  // offset of its passive-ion cells (XP0 or XP1)

  __device__ __forceinline__ double& x(int f, int i) const { return col[xo + f * L.G + i + 1]; }
  __device__ __forceinline__ double& o(int f, int i) const { return col[L.O + f * L.G + i + 1]; }
  __device__ __forceinline__ double& dl(int f, int c) const { return col[L.DL + f * (L.nAlts + 2) + c]; }
  __device__ __forceinline__ double& sc(int k) const { return col[L.SC + k]; }
  __device__ __forceinline__ double& cm(int i) const { return col[L.CM + i + 1]; }
  __device__ __forceinline__ double& tu(int i) const { return col[L.TU + i + 1]; }
  __device__ __forceinline__ double& gm(int i) const { return col[L.GM + i + 1]; }
  __device__ __forceinline__ double& ion(int s, int i) const {
    return (s < NADV) ? col[xo + (F_I + s) * L.G + i + 1]
                      : col[xpo + (s - NADV) * NPC + pcell(i, L.nAlts)];
  }
  // grid coefficient k at Fortran cell i
  __device__ __forceinline__ double g(int k, int i) const {
    return __ldg(gridc + (size_t(k) * L.G + (i + 1)) * gcols + gc);
  }
  __device__ __forceinline__ double bcc(int j) const {
    return __ldg(gridc + (size_t(NGC) * L.G + j) * gcols + gc);
  }
  __device__ __forceinline__ double dAF(int i) const { return g(GC_DALTF, i); }
  // AUSM cell constant k at Fortran cell i
  __device__ __forceinline__ double ga(int k, int i) const {
    return __ldg(gridc + (size_t(NGC) * L.G + NBC + size_t(k) * L.G + (i + 1)) * gcols + gc);
  }
};

// Sequential sum over lanes 0..n-1 of v (same order as a Fortran DO loop
// starting from 0.0); every lane gets the result.
__device__ __forceinline__ double lane_seq_sum(double v, int n) {
  double s = 0.0;
  for (int k = 0; k < n; ++k) s = s + __shfl_sync(0xffffffffu, v, k);
  return s;
}

// ------------------------------------------------------------ boundaries
// set_vertical_bcs (Earth), set_vertical_bcs.Earth.f90:8-652, for one column.
// part 1 = the lower boundary (cells -1, 0) with the neutral densities and
// LogRho of the upper ghost cells, part 2 = the rest of the upper boundary
// (nAlts+1, nAlts+2: winds, temperature, ions), part 3 = both; the two parts
// touch disjoint cells and fields and can run on different warps.  Executed
// by a full warp, lanes over species / ions.
//
// Where the reference goes through exp and back through log with a factor
// that is exactly 1 (Temp(-1) = Temp(0) and Temp(nAlts+1:nAlts+2) =
// Temp(nAlts) make the temperature ratios 1), the hydrostatic cells are
// formed directly in log space: LogNS(-1) = LogNS(0) + dz/H, LogNS(nA+1) =
// LogNS(nA) - dz/H.  IVel ghosts and the electron slot are not set: nothing
// on the path reads them.
__device__ __forceinline__ void bc_column(ColCtx c, const GitmVertParams& prm, int lane,
                                          uint32_t* st, int part) {
  const int nA = c.L.nAlts;
  const int G = c.L.G;
  double* X = c.col + c.xo + 1;  // X[f*G + i]
  const double* sc = c.col + c.L.SC;
  const bool improved = prm.use_improved_ion_advection != 0;
  const int s = lane;
  auto x = [&](int f, int i) -> double& { return X[f * G + i]; };

  if (part & 1) {
    const bool msis = prm.use_msis_bcs && sc[SC_HASLBC] != 0.0;
    // LogNS(0) on entry: NS(0) of line 93 is formed before the MSIS values
    // overwrite cell 0
    const double l0 = (s < NS) ? x(F_LNS + s, 0) : 0.0;
    // the upper boundary's hydrostatic neutrals (lines 471-486, Temp(nA+1:nA+2)
    // = Temp(nA)) read only interior cells: formed first, so that their
    // division and exponentials overlap the lower boundary's work
    double mu1 = 0.0, mu2 = 0.0;
    if (s < NS) {
      const double T = x(F_T, nA);
      const double den = 0.5 * (T + T) * KB;
      const double ish1 = (-0.5 * (sc[SC_EG + 3] + sc[SC_EG + 2])) * c_k.mass[s] / den;
      const double ish2 = (-0.5 * (sc[SC_EG + 4] + sc[SC_EG + 3])) * c_k.mass[s] / den;
      const double l1 = x(F_LNS + s, nA) - ish1 * sc[SC_DAF + 4];
      const double l2 = l1 - ish2 * sc[SC_DAF + 5];
      x(F_LNS + s, nA + 1) = l1;
      x(F_LNS + s, nA + 2) = l2;
      mu1 = c_k.mass[s] * exp(l1);
      mu2 = c_k.mass[s] * exp(l2);
    }
    __syncwarp();
    // lines 112-148
    if (msis) {
      const double* t = sc + SC_LBC;
      if (s < NS) {
        x(F_LNS + s, -1) = t[s];
        x(F_LNS + s, 0) = t[10 + s];
      } else if (s == 6) {
        x(F_T, -1) = t[6];
        x(F_T, 0) = t[16];
      } else if (s == 7) {
        x(F_LRHO, -1) = t[7];
        x(F_LRHO, 0) = t[17];
      } else if (s == 8) {
        x(F_VE, -1) = t[8];
        x(F_VE, 0) = t[18];
      } else if (s == 9) {
        x(F_VN, -1) = t[9];
        x(F_VN, 0) = t[19];
      }
    } else {
      if (s == 8) { x(F_VE, -1) = 0.0; x(F_VE, 0) = 0.0; }
      if (s == 9) { x(F_VN, -1) = 0.0; x(F_VN, 0) = 0.0; }
    }
    if (s == 10) { x(F_VU, -1) = 0.0; x(F_VU, 0) = 0.0; }
    if (s < NS) { x(F_W + s, -1) = 0.0; x(F_W + s, 0) = 0.0; }
    __syncwarp();
    // lines 192-196
    if (s == 0) {
      x(F_T, -1) = x(F_T, 0);
      x(F_VE, -1) = x(F_VE, 0);
      x(F_VN, -1) = x(F_VN, 0);
      x(F_VU, -1) = x(F_VU, 0);
    }
    __syncwarp();
    const double* bl = sc + SC_BCC;  // lower mesh coefficients, cell 0 then -1
    if (s < NS) {
      if (!photochemical(s)) {
        // lines 205-222: hydrostatic cell -1 with the mean major mass
        const double MeanGravity = -0.5 * (sc[SC_EG + 0] + sc[SC_EG + 1]);
        const double MeanTemp = 0.5 * (x(F_T, 0) + x(F_T, -1));
        const double MeanMass = 0.5 * (sc[SC_MMM_0] + sc[SC_MMM_M1]);
        const double ish = MeanGravity * MeanMass / (MeanTemp * KB);
        x(F_LNS + s, -1) = (s == 0) ? x(F_LNS + s, 0) : l0 + ish * sc[SC_DAF + 0];
      } else {
        // lines 226-272: 3rd-order extrapolation with a gradient limit
        #pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int i = -k;
          const double* C = bl + 5 * k;
          const double d = x(F_LNS + s, i + 1) * C[0] + x(F_LNS + s, i + 2) * C[1] +
                           x(F_LNS + s, i + 3) * C[2] + x(F_LNS + s, i + 4) * C[3] +
                           x(F_LNS + s, i + 5) * C[4];
          const double up = x(F_LNS + s, i + 1);
          double v = up - sc[SC_DAF + 2 + i] * d;  // dAlt_F(i+1)
          if (d <= 0.0) v = up;
          if (s == 4 && v < up - 0.333) v = up - 0.333;
          x(F_LNS + s, i) = v;
        }
      }
      // vertical winds (lines 334-344)
      #pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int i = -k;
        const double* C = bl + 5 * k;
        const double d = x(F_W + s, i + 1) * C[0] + x(F_W + s, i + 2) * C[1] +
                         x(F_W + s, i + 3) * C[2] + x(F_W + s, i + 4) * C[3] +
                         x(F_W + s, i + 5) * C[4];
        x(F_W + s, i) = x(F_W + s, i + 1) - sc[SC_DAF + 2 + i] * d;
      }
    }
    // ions float at the lower boundary (lines 304-310)
    if (s < NI) {
      const double v = c.ion(s, 1);
      c.ion(s, 0) = v;
      c.ion(s, -1) = v;
    }
    __syncwarp();
    // lines 348-362: LogRho and bulk vertical wind at cells 0 and -1, and
    // the upper boundary's LogRho (lines 598-604) from the ghosts formed
    // above: the warp of the upper half keeps the ion chain alone.  The six
    // sums over species go through shared memory (the slope buffer is dead
    // during the boundary passes; the upper half uses its first 63 doubles):
    // lanes 0..3 add them in species order, one log serves the four cells
    {
      double* sb = c.col + c.L.DL + 64;  // [6][NS]: m0, m1, t0, t1, mu1, mu2
      if (s < NS) {
        const double m0 = c_k.mass[s] * exp(x(F_LNS + s, 0));
        const double m1 = c_k.mass[s] * exp(x(F_LNS + s, -1));
        sb[0 * NS + s] = m0;
        sb[1 * NS + s] = m1;
        sb[2 * NS + s] = m0 * x(F_W + s, 0);
        sb[3 * NS + s] = m1 * x(F_W + s, -1);
        sb[4 * NS + s] = mu1;
        sb[5 * NS + s] = mu2;
      }
      __syncwarp();
      // lanes 0..3 take cells 0, -1, nAlts+1, nAlts+2
      if (s < 4) {
        const int q = (s < 2) ? s : s + 2;
        double r = 0.0, v = 0.0;
#pragma unroll
        for (int k = 0; k < NS; ++k) r = r + sb[q * NS + k];
        if (s < 2) {
#pragma unroll
          for (int k = 0; k < NS; ++k) v = v + sb[(2 + s) * NS + k];
        }
        const int cell = (s < 2) ? -s : nA + s - 1;
        x(F_LRHO, cell) = log(r);
        if (s < 2) x(F_VU, -s) = v / r;
      }
    }
    // lines 364-376
    if (msis && (s == 8 || s == 9)) {
      const int f = (s == 8) ? F_VE : F_VN;
      const double* C = bl + 5;
      const double d = x(f, 0) * C[0] + x(f, 1) * C[1] + x(f, 2) * C[2] + x(f, 3) * C[3] + x(f, 4) * C[4];
      x(f, -1) = x(f, 0) - sc[SC_DAF + 1] * d;
    }
    __syncwarp();
    // lines 382-395
    if (s < NS && photochemical(s) && x(F_W + s, 1) > 0.0) {
      x(F_W + s, 0) = -1.0 * x(F_W + s, 1);
      x(F_W + s, -1) = -1.0 * x(F_W + s, 1);
    }
  }

  if (part & 2) {
    // lines 420-463
    if (s == 8) { x(F_VE, nA + 1) = x(F_VE, nA); x(F_VE, nA + 2) = x(F_VE, nA); }
    if (s == 9) { x(F_VN, nA + 1) = x(F_VN, nA); x(F_VN, nA + 2) = x(F_VN, nA); }
    if (s < NS) {
      const double wn = x(F_W + s, nA);
      double w1 = wn, w2 = wn;
      if (photochemical(s) && wn < 0.0) {
        w1 = -wn;
        w2 = -x(F_W + s, nA - 1);
      }
      x(F_W + s, nA + 1) = w1;
      x(F_W + s, nA + 2) = w2;
      // the hydrostatic neutrals (lines 471-486) are formed with the lower
      // boundary (part 1)
    }
    if (s == 10) {
      const double v = x(F_VU, nA);
      const double w = (v < 0.0) ? -v : v;
      x(F_VU, nA + 1) = w;
      x(F_VU, nA + 2) = w;
    }
    if (s == 11) {
      x(F_T, nA + 1) = x(F_T, nA);
      x(F_T, nA + 2) = x(F_T, nA);
    }
    // lines 497-501: TEC of the first ion; with UseImprovedIonAdvection,
    // the scan for negative values of check_for_negative_densities (lines
    // 608-649, which acts only when a value in nAlts-5 .. nAlts+2 is
    // negative) and, in the same block so that their latencies overlap, the
    // logs the extrapolation of lines 503-596 takes when no value is
    // negative: lg[7 s + j] = log(ion s at nAlts+2-j), j = 0..6 (the ghost
    // nAlts+2 and the cells nAlts+1 .. nAlts-4), 63 logs, two per lane
    double tp = 0.0;
    bool neg = false;
    double* lg = c.col + c.L.DL;  // scratch: the slopes are dead during the BCs
    if (improved) {
      for (int i = 1 + lane; i <= nA; i += 32) tp += c.dAF(i) * c.ion(0, i);
      if (s < NI)
        for (int q = nA - 5; q <= nA + 2; ++q) neg = neg || (c.ion(s, q) < 0.0);
      for (int q = lane; q < NI * 7; q += 32) {
        const int si = q / 7, j = q - si * 7;
        lg[q] = log(c.ion(si, nA + 2 - j));
      }
    } else {
      for (int i = 1 + lane; i <= nA; i += 32) tp += c.dAF(i) * exp(c.ion(0, i));
    }
    for (int off = 16; off > 0; off >>= 1) tp += __shfl_xor_sync(0xffffffffu, tp, off);
    // TEC / 1e16 < MinTEC (1e16 is exact in binary64)
    const bool hold = (tp < prm.min_tec * 1e16) && (sc[SC_PLASMA] != 0.0);
    const double* bu = sc + SC_BCC + 10;  // upper mesh coefficients, nA+1 then nA+2
    const bool anyneg = __any_sync(0xffffffffu, neg);
    __syncwarp();
    if (!improved) {
      if (s < NI && !hold) {
        #pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int iAlt = nA + 1 + k;
          const double* C = bu + 5 * k;
          double dn = C[0] * c.ion(s, iAlt - 1) + C[1] * c.ion(s, iAlt - 2) + C[2] * c.ion(s, iAlt - 3) +
                      C[3] * c.ion(s, iAlt - 4) + C[4] * c.ion(s, iAlt - 5);
          const double lim = -(0.001 * c.ion(s, iAlt) / sc[SC_DAF + 3]);
          if (dn > lim) dn = lim;
          c.ion(s, iAlt) = c.ion(s, iAlt - 1) + dn * sc[SC_DAF + 4 + k];
        }
      }
    } else if (anyneg) {
      // the reference's order, one ion per lane
      if (s < NI) {
        #pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int iAlt = nA + 1 + k;
          double mn = c.ion(s, iAlt - 5);
          for (int q = iAlt - 4; q <= iAlt; ++q) mn = fmin(mn, c.ion(s, q));
          if (mn < 0.0) {
            if (c.ion(s, iAlt - 6) < 0.0) atomicOr(st, GITM_ST_NEG_ION_TOP);
            for (int q = iAlt - 5; q <= iAlt - 1; ++q) {
              if (c.ion(s, q) < 0.0) {
                if (c.ion(s, q - 1) > 0.0 && c.ion(s, q + 1) > 0.0)
                  c.ion(s, q) = (c.ion(s, q - 1) + c.ion(s, q + 1)) / 2.0;
                else
                  c.ion(s, q) = c.ion(s, q - 1) * 0.95;
              }
            }
            if (c.ion(s, iAlt) < 0.0) c.ion(s, iAlt) = c.ion(s, iAlt - 1) * 0.95;
          }
          double n[6];
          #pragma unroll
          for (int j = 0; j < 6; ++j) n[j] = log(c.ion(s, iAlt - j));
          if (!hold) {
            const double* C = bu + 5 * k;
            double dn = C[0] * n[1] + C[1] * n[2] + C[2] * n[3] + C[3] * n[4] + C[4] * n[5];
            const double lim = -(0.001 * n[0] / sc[SC_DAF + 3]);
            if (dn > lim) dn = lim;
            c.ion(s, iAlt) = exp(n[1] + dn * sc[SC_DAF + 4 + k]);
          }
        }
      }
    } else if (!hold) {
      // no negative value: the logs taken above (the second cell reuses
      // four of the first's)
      double n1 = 0.0;
      if (s < NI) {
        const double* n = lg + s * 7 + 1;  // n[k] = log(ion at nAlts+1-k)
        const double* C = bu;
        double dn = C[0] * n[1] + C[1] * n[2] + C[2] * n[3] + C[3] * n[4] + C[4] * n[5];
        const double lim = -(0.001 * n[0] / sc[SC_DAF + 3]);
        if (dn > lim) dn = lim;
        const double y = n[1] + dn * sc[SC_DAF + 4];
        c.ion(s, nA + 1) = exp(y);
        // cell nAlts+2: the log of its own ghost, and y for the log of the
        // value just set (log(exp(y)) in the reference, y to rounding)
        const double g0 = lg[s * 7];
        n1 = y;
        const double* D = bu + 5;
        double dn2 = D[0] * n1 + D[1] * n[1] + D[2] * n[2] + D[3] * n[3] + D[4] * n[4];
        const double lim2 = -(0.001 * g0 / sc[SC_DAF + 3]);
        if (dn2 > lim2) dn2 = lim2;
        c.ion(s, nA + 2) = exp(n1 + dn2 * sc[SC_DAF + 5]);
      }
    }
    // LogRho of nAlts+1, nAlts+2 (lines 598-604) is formed with the lower
    // boundary (part 1)
  }
  __syncwarp();
}

// calc_neutral_friction (calc_neutral_friction.f90:47-106) for one cell:
// solves (I + dt C) v = w in place and adds the eddy term -Eddy GradLogConS.
// C_ij = 1e-2 k / (M_i D0_ij) n_j T^(1 - DiffExp_ij) (the NDensity factors of
// the reference cancel); LU without pivoting, the matrix being strictly
// diagonally dominant by rows for finite inputs.  ludcmp stops the run on a
// row without an element of nonzero magnitude (ludcmp.f:9-17; NaN compares
// false there, so a row of NaN counts): such a row sets GITM_ST_LU_SINGULAR
// in *st (when st is given) and the solve goes on, its results non-finite.
// A finite nonzero diagonal settles a row, so the scan of the whole row runs
// only when the diagonal fails.
__device__ __forceinline__ void friction_solve(double dt, const double (&ns)[NS], double T, double eddy,
                                               const double (&glc)[NS], double (&wv)[NS],
                                               uint32_t* st = nullptr) {
  const double lt = log(T);
  double pw[NS];
#pragma unroll
  for (int e = 0; e < NS; ++e) pw[e] = exp(c_k.one_minus_e[e] * lt);
  // dt C_ij with dt taken into the densities once per cell: the entries
  // -dt C_ij and the diagonal 1 + sum_j dt C_ij share each product
  double nd[NS];
#pragma unroll
  for (int q = 0; q < NS; ++q) nd[q] = dt * ns[q];
  double a[NS][NS];
#pragma unroll
  for (int r = 0; r < NS; ++r) {
    double rs = 0.0;
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      if (q == r) continue;
      const double dcij = c_k.kc[r][q] * nd[q] * pw[exp_index(r, q)];
      a[r][q] = -dcij;
      rs = rs + dcij;
    }
    a[r][r] = 1.0 + rs;
  }
  if (st) {
    bool diag_ok = true;
#pragma unroll
    for (int r = 0; r < NS; ++r) diag_ok = diag_ok && (fabs(a[r][r]) > 0.0);
    if (!diag_ok) {
      bool singular = false;
#pragma unroll
      for (int r = 0; r < NS; ++r) {
        double mx = 0.0;
#pragma unroll
        for (int q = 0; q < NS; ++q)
          if (fabs(a[r][q]) > mx) mx = fabs(a[r][q]);
        singular = singular || !(mx > 0.0);
      }
      if (singular) atomicOr(st, GITM_ST_LU_SINGULAR);
    }
  }
#pragma unroll
  for (int p = 0; p < NS; ++p) {
    const double ip = 1.0 / a[p][p];
    a[p][p] = ip;
#pragma unroll
    for (int r = p + 1; r < NS; ++r) {
      const double l = a[r][p] * ip;
#pragma unroll
      for (int q = p + 1; q < NS; ++q) a[r][q] -= l * a[p][q];
      wv[r] -= l * wv[p];
    }
  }
#pragma unroll
  for (int r = NS - 1; r >= 0; --r) {
    double sum = wv[r];
#pragma unroll
    for (int q = r + 1; q < NS; ++q) sum -= a[r][q] * wv[q];
    wv[r] = sum * a[r][r];
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) wv[s] = wv[s] + (-eddy * glc[s]);
}

// GradLogConS at cell i (vertical_solver_rusanov.f90:506-543,
// vertical_solver_ausm.f90:644-686): the 5-point mesh on
// LogConS = log(m_s) + LogNS - LogRho of the stage state.
__device__ __forceinline__ void grad_log_cons(ColCtx c, int i, double (&glc)[NS]) {
  double mc[5], lr5[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    mc[q] = c.g(GC_M0 + q, i);
    lr5[q] = c.x(F_LRHO, i - 2 + q);
  }
  // sum_q mc_q (log m_s + LogNS_s - LogRho) = sum_q mc_q (LogNS_s - LogRho) + log m_s sum_q mc_q:
  // the species' constant leaves the five-point sum (one fma per point)
  const double msum = ((mc[0] + mc[1]) + (mc[2] + mc[3])) + mc[4];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < 5; ++q) acc = fma(mc[q], c.x(F_LNS + s, i - 2 + q) - lr5[q], acc);
    glc[s] = fma(c_k.log_mass[s], msum, acc);
  }
}

constexpr double F1 = 0.6250000;  // Factor1, vertical_solver_rusanov.f90:739
constexpr double F2 = 0.0416667;  // Factor2, vertical_solver_rusanov.f90:740

// advance_vertical_1stage (vertical_solver_rusanov.f90:387-686) at interior
// cell i of the stage state in c, from the limited slopes in c's slope
// buffer; emit(f, New - state) takes each field's increment.  st (may be
// null) receives the column's GITM_ST_LU_SINGULAR bit.
template <class Emit>
__device__ __forceinline__ void rusanov_cell(ColCtx c, int i, const GitmVertParams& prm, double dt,
                                             double eddy, double ivup, double inv_vert_tau, Emit&& emit,
                                             uint32_t* st = nullptr) {
  const double dF0 = c.dAF(i), dF1 = c.dAF(i + 1);
  const double idc = c.g(GC_IDC, i);
  const double fc0 = 0.5 * fmax(c.cm(i - 1), c.cm(i));
  const double fc1 = 0.5 * fmax(c.cm(i), c.cm(i + 1));
  // the halves taken once per cell: a product with 0.5 is exact, so
  // d * (0.5 dF) and x * (0.5 / dAlt_C) round like (0.5 d) dF and (0.5 x) / dAlt_C
  const double hF0 = 0.5 * dF0, hF1 = 0.5 * dF1, hidc = 0.5 * idc;
  // calc_rusanov_alts_rusanov (:694-718) at cell i
  auto sweep = [&](int f, double& grad, double& diff) {
    const double* v = &c.col[c.xo + f * c.L.G + 1];
    const double* d = &c.col[c.L.DL + f * (c.L.nAlts + 2)];
    const double L0 = fma(d[i - 1], hF0, v[i - 1]);
    const double R0 = fma(-d[i], hF0, v[i]);
    const double L1 = fma(d[i], hF1, v[i]);
    const double R1 = fma(-d[i + 1], hF1, v[i + 1]);
    grad = (L1 + R1 - L0 - R0) * hidc;
    diff = (fc1 * (R1 - L1) - fc0 * (R0 - L0)) * idc;
  };
  const double invr = c.g(GC_INVR, i), rr = c.g(GC_R, i), grav = c.g(GC_GRAV, i);
  const double T = c.x(F_T, i), VE = c.x(F_VE, i), VN = c.x(F_VN, i), VU = c.x(F_VU, i);
  double gT, dT;
  sweep(F_T, gT, dT);
  {
    double gE, dE, gN, dN, gU, dU;
    sweep(F_VE, gE, dE);
    sweep(F_VN, gN, dN);
    sweep(F_VU, gU, dU);
    // :660-680
    emit(F_VE, (VE - dt * VU * gE + dt * dE) - VE);
    emit(F_VN, (VN - dt * VU * gN + dt * dN) - VN);
    const double divv = gU + 2 * VU * invr;
    emit(F_T, (T - dt * (VU * gT + (c.gm(i) - 1.0) * (T * divv)) + dt * dT) - T);
  }
  // ions 1..nIonsAdvect (:557-568)
#pragma unroll
  for (int s = 0; s < NADV; ++s) {
    double gI, dI;
    sweep(F_I + s, gI, dI);
    const double I = c.x(F_I + s, i);
    emit(F_I + s, (I - dt * (ivup * gI) + dt * dI) - I);
  }
  // species continuity and momentum (:548-617)
  const double itau = prm.use_damping ? 1.0 / (15 - (1 - exp(-1.0 * c.g(GC_ALT, i) / 1000.0 / 40.0)) * 5.0)
                                      : inv_vert_tau;
  const double hz = (VN * VN + VE * VE) * invr;
  const double cor = prm.use_coriolis ? dt * (c.sc(SC_CENT) * rr + c.sc(SC_CORI) * VE) : 0.0;
  double wv[NS];
  double sumrho = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double gL, dL, gW, dW;
    sweep(F_LNS + s, gL, dL);
    sweep(F_W + s, gW, dW);
    const double Ls = c.x(F_LNS + s, i), Ws = c.x(F_W + s, i);
    const double divw = gW + 2 * Ws * invr;
    const double nl = Ls - dt * (divw + Ws * gL) + dt * dL;
    emit(F_LNS + s, nl - Ls);
    sumrho = sumrho + c_k.mass[s] * exp(nl);
    const double km = c_k.k_over_m[s];
    double w = Ws - dt * (Ws * gW - hz + T * gL * km + gT * km - grav) + dt * dW - Ws * itau;
    w = w + cor;
    w = w - dt * (prm.thermal_diff_coef[s] * km) * gT;
    wv[s] = w;
  }
  const double LR = c.x(F_LRHO, i);
  emit(F_LRHO, log(sumrho) - LR);
  // NS = exp(LogNS), 1 / Rho (:466-467)
  double ns[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) ns[s] = exp(c.x(F_LNS + s, i));
  const double ir = exp(-LR);
  // calc_neutral_friction (calc_neutral_friction.f90:47-106)
  if (prm.use_neutral_friction) {
    // GradLogConS (:506-543), LogConS = log(m_s) + LogNS - LogRho
    double glc[NS];
    grad_log_cons(c, i, glc);
    friction_solve(dt, ns, T, eddy, glc, wv, st);
  }
  // clamp and bulk vertical wind (:643-658)
  double vu = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double w = fmax(-prm.max_vertical_velocity, wv[s]);
    w = fmin(prm.max_vertical_velocity, w);
    emit(F_W + s, w - c.x(F_W + s, i));
    vu = vu + w * (c_k.mass[s] * ns[s] * ir);
  }
  emit(F_VU, vu - VU);
}

// Limited slopes of the 18 swept fields at cell i: the 4th-order form on
// interior cells, the 2nd-order one on cells 0 and nAlts+1
// (calc_facevalues_alts_rusanov, vertical_solver_rusanov.f90:745-772),
// the choice made per field, so that a warp whose lanes hold both kinds of
// cell diverges only over the two differences (threads over cells
// 0..nAlts+1 of every column).
__device__ __forceinline__ void rusanov_slopes_cell(ColCtx c, int i, double beta) {
  const int nA = c.L.nAlts;
  const bool end = (i == 0 || i == nA + 1);
  const double cu = end ? c.g(GC_IDF, i + 1) : c.g(GC_H2, i + 1);
  const double cd = end ? c.g(GC_IDF, i) : c.g(GC_H2, i);
  // one expression for both forms: the end cells' 2nd-order differences are
  // cu * (1 * (v[i+1] - v[i]) - 0 * (...)), exactly; their outer neighbours
  // are clamped into the column (finite values the zero factor removes)
  const double a = end ? 1.0 : F1, b = end ? 0.0 : F2;
  const int ip2 = min(i + 2, nA + 2), im2 = max(i - 2, -1);
  // the state and slope regions of the column do not overlap: restrict
  // lets the loads of later fields be issued ahead of earlier stores
  const double* __restrict__ xv = c.col + c.xo + 1;
  double* __restrict__ sl = c.col + c.L.DL + i;
#pragma unroll 9
  for (int f = 0; f < NSTENCIL; ++f) {
    const double* v = xv + f * c.L.G;
    const double u = cu * (a * (v[i + 1] - v[i]) - b * (v[ip2] - v[i - 1]));
    const double d = cd * (a * (v[i] - v[i - 1]) - b * (v[i + 1] - v[im2]));
    sl[f * (nA + 2)] = limiter_mc(u, d, beta);
  }
}

}  // namespace gv

#include "vert_ausm.cuh"

namespace gv {

// ------------------------------------------------------------ the kernel
struct KParams {
  const DevMember* members;
  const Tile* tiles;
  int n_tiles;
  int n_steps;
  double dt;
  uint32_t* status;   // one word per column (member col_offset + column)
  double* scratch;    // per-CTA slots of global scratch: RK accumulators, NF * NT doubles
                      // (ACC_GLOBAL), then with OG the Orig of the tile's columns
  int64_t scratch_per_cta;  // doubles of one CTA's slot (OG kernels)
  GitmVertParams prm;
  // SAVE kernels (one step per launch): the gathered state and the
  // post-boundary stage states X0..X4 of every column, state s of global
  // column c at save[(s * save_ncols + c) * save_per], for the adjoint
  double* save;
  int64_t save_ncols;
  int save_per;
};

// IO = 0: GITM arrays (advance_vertical gather/scatter);
// IO = 1: ModVertical arrays (advance_vertical_1d_* arguments).
// ACC_GLOBAL: the RK accumulator of each item lives in a per-CTA slot of
// kp.scratch (coalesced, L2-resident under a persistent grid) instead of
// registers, which lets small CTAs share an SM.
// NA > 0: every member has exactly NA altitudes (the host checks), so the
// shared-memory layout, the item mapping and the loop bounds are
// compile-time constants; NA = 0 reads nAlts from the member.
// OG (with ACC_GLOBAL): Orig lives in the CTA's slot of global scratch after
// the accumulators (coalesced, L2-resident, read-only within a step), so a
// column needs 8 KB less shared memory and more columns share an SM.
template <int IO, int NT, int MINB, bool ACC_GLOBAL, int SOLVER, bool SAVE = false, int NA = 0, bool OG = false>
__global__ void __launch_bounds__(NT, MINB) vert_step_kernel(const KParams kp) {
  static_assert(!OG || ACC_GLOBAL, "Orig in global scratch goes with the accumulators there");
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wid = tid >> 5;
  const GitmVertParams& prm = kp.prm;
  const double dt = kp.dt;
  double* const slot = ACC_GLOBAL ? kp.scratch + size_t(blockIdx.x) * (OG ? size_t(kp.scratch_per_cta) : size_t(NF) * NT)
                                  : nullptr;
  double* accg = ACC_GLOBAL ? slot + tid : nullptr;
  double* const ogb = OG ? slot + size_t(NF) * NT : nullptr;  // Orig of column cl at ogb + cl * orig_doubles
  const double inv_vert_tau = 1.0 / prm.vert_tau;  // 1 / VertTau without damping

  for (int tix = blockIdx.x; tix < kp.n_tiles; tix += gridDim.x) {
    const Tile tile = kp.tiles[tix];
    const DevMember& M = kp.members[tile.member];
    const int nA = (NA > 0) ? NA : M.b.n_alts;
    const int nc = tile.nc;
    const Layout L = make_layout(nA, SOLVER, OG);
    const int operc = orig_doubles(nA);  // Orig doubles per column (OG)
    const int G = L.G;
    const int64_t ncols = M.b.n_cols;
    uint32_t* sst = reinterpret_cast<uint32_t*>(sm + size_t(L.stride) * nc);  // [nc] status
    uint32_t* sfrozen = sst + nc;                                             // [nc]
    const int nitems = nc * nA;
    const bool item = tid < nitems;
    const int my_cl = item ? tid / nA : 0;
    const int my_i = item ? tid % nA + 1 : 1;
    int cur = 0;  // stage buffer holding the current state

    auto ctx = [&](int cl) {
      ColCtx c;
      c.col = sm + size_t(L.stride) * cl;
      c.L = L;
      c.gridc = M.gridc;
      c.gcols = M.gcols;
      c.gc = (M.gcols == 1) ? 0 : int(tile.c0 + cl);
      c.xo = cur ? L.X1 : L.X0;
      c.xpo = cur ? L.XP1 : L.XP0;
      return c;
    };
    auto gidx = [&](int f, int g, int cl) -> int64_t {
      return (int64_t(f) * G + g) * ncols + tile.c0 + cl;
    };
    // SAVE: copies the current stage buffer (state and passive cells) of
    // every column of the tile to saved state s
    auto save_state = [&](int s) {
      if constexpr (SAVE) {
        const int per = NF * G + NPAS * NPC;
        const int xo = cur ? L.X1 : L.X0;
        for (int cl = 0; cl < nc; ++cl) {
          const double* src = sm + size_t(L.stride) * cl + xo;
          double* dst = kp.save + (int64_t(s) * kp.save_ncols + M.col_offset + tile.c0 + cl) * kp.save_per;
          for (int r = tid; r < per; r += NT) dst[r] = src[r];
        }
      }
    };
    // set_vertical_bcs for every column of the tile: the lower and upper
    // halves of a column go to different warps when there are enough
    auto boundaries = [&]() {
      constexpr int nw = NT / 32;
      if (2 * nc <= nw) {
        if (wid < 2 * nc) bc_column(ctx(wid >> 1), prm, lane, &sst[wid >> 1], 1 + (wid & 1));
      } else {
        for (int cl = wid; cl < nc; cl += nw) bc_column(ctx(cl), prm, lane, &sst[cl], 3);
      }
    };

    if (tid < nc) {
      sst[tid] = 0u;
      sfrozen[tid] = 0u;
    }
    __syncthreads();

    // ---------------------------------------------------------- load
    // per-column scalars (advance_vertical.f90:84-85,103-104)
    if (tid < nc) {
      ColCtx c = ctx(tid);
      const int64_t cc = tile.c0 + tid;
      double cent, cori, sza, mlat;
      if (IO == 0) {
        const double cl = M.b.cos_lat[cc];
        cent = (cl * prm.omega_body) * (cl * prm.omega_body);
        cori = 2 * cl * prm.omega_body;
        sza = M.b.sza[cc];
        mlat = M.b.mlat[cc];
      } else {
        cent = M.mv.centrifugal[cc];
        cori = M.mv.coriolis[cc];
        sza = M.mv.sza[cc];
        mlat = M.mv.mlat[cc];
      }
      c.sc(SC_CENT) = cent;
      c.sc(SC_CORI) = cori;
      c.sc(SC_SZA) = sza;
      c.sc(SC_MLAT) = mlat;
      // set_vertical_bcs.Earth.f90:488-495
      bool plasma = false;
      if (prm.use_nighttime_ion_bcs)
        plasma = sza > PI / 2 && ((mlat > 30.0 && mlat < 70.0) || (mlat > -60.0 && mlat < -30.0));
      c.sc(SC_PLASMA) = plasma ? 1.0 : 0.0;
      const double* lbc = (IO == 0) ? M.b.lbc : M.mv.lbc;
      c.sc(SC_HASLBC) = lbc ? 1.0 : 0.0;
      if (lbc)
        for (int k = 0; k < 2 * GITM_LBC_NVALUES; ++k)
          c.sc(SC_LBC + k) = lbc[int64_t(k) * ncols + cc];
      // boundary constants of this column's grid
      for (int j = 0; j < 20; ++j) c.sc(SC_BCC + j) = c.bcc(j);
      const int dcell[6] = {-1, 0, 1, nA, nA + 1, nA + 2};
      for (int j = 0; j < 6; ++j) c.sc(SC_DAF + j) = c.dAF(dcell[j]);
      const int ecell[5] = {-1, 0, nA, nA + 1, nA + 2};
      for (int j = 0; j < 5; ++j) c.sc(SC_EG + j) = c.g(GC_GRAV, ecell[j]) + cent * c.g(GC_R, ecell[j]);
    }
    // columns vary fastest across threads so that a warp reads whole row
    // segments of the native layout
    for (int w = tid; w < nc * G; w += NT) {
      const int g = w / nc, cl = w - g * nc, i = g - 1;
      ColCtx c = ctx(cl);
      if (IO == 0) {
        const GitmColumnBatch& b = M.b;
        double nd[NS], ww[NS];
        double mn = 1.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          nd[s] = b.ndensity_s[gidx(s, g, cl)];
          ww[s] = b.vert_vel[gidx(s, g, cl)];
          mn = fmin(mn, nd[s]);
        }
        if (!(mn > 0.0)) atomicOr(&sfrozen[cl], 1u);
        const double temperature = b.temperature[gidx(0, g, cl)];
        double gamma, mmm, tu, cmx = 0.0;
        if (prm.compute_coefficients) {
          // calc_pressure.f90:17-21,56-83; calc_rates.Earth.f90:34-50;
          // calc_timestep.f90:114-118
          double N = 0.0;
#pragma unroll
          for (int s = 0; s < NS; ++s) N = N + nd[s];
          double gg = 0.0;
#pragma unroll
          for (int s = 0; s < NS; ++s) gg = gg + nd[s] * c_k.inv_vib2[s];
          gamma = gg * 2.0 / N + 1;
          double m = 0.0;
          const double rn = 1.0 / (N + 1.0);
#pragma unroll
          for (int s = 0; s < NS; ++s) m = m + c_k.mass[s] * nd[s] * rn;
          if (m == 0) m = c_k.mass[0];
          mmm = m;
          tu = m * (1.0 / KB);
          if (g >= 1 && g <= nA + 2) {
            double mx = fabs(ww[0]);
#pragma unroll
            for (int s = 1; s < NS; ++s) mx = fmax(mx, fabs(ww[s]));
            cmx = mx + sqrt(gamma * temperature);
          }
          if (kp.n_steps == 1) {
            if (b.gamma) b.gamma[gidx(0, g, cl)] = gamma;
            if (b.mean_major_mass) b.mean_major_mass[gidx(0, g, cl)] = mmm;
            if (b.temp_unit) b.temp_unit[gidx(0, g, cl)] = tu;
            if (b.cmax && g >= 1 && g <= nA + 2) b.cmax[gidx(0, g, cl)] = cmx;
          }
        } else {
          gamma = b.gamma[gidx(0, g, cl)];
          mmm = b.mean_major_mass[gidx(0, g, cl)];
          tu = b.temp_unit[gidx(0, g, cl)];
          if (g >= 1 && g <= nA + 2) cmx = b.cmax[gidx(0, g, cl)];
        }
        c.tu(i) = tu;
        c.cm(i) = cmx;
        c.gm(i) = gamma;
        if (i == -1) c.sc(SC_MMM_M1) = mmm;
        if (i == 0) c.sc(SC_MMM_0) = mmm;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          c.x(F_LNS + s, i) = log(nd[s]);
          c.x(F_W + s, i) = ww[s];
        }
        c.x(F_T, i) = temperature * tu;
        c.x(F_VE, i) = b.velocity[gidx(0, g, cl)];
        c.x(F_VN, i) = b.velocity[gidx(1, g, cl)];
        c.x(F_VU, i) = b.velocity[gidx(2, g, cl)];
        c.x(F_LRHO, i) = log(b.rho[gidx(0, g, cl)]);
        const bool pc = in_pcells(i, nA);
#pragma unroll
        for (int s = 0; s < NI; ++s) {
          if (s >= NADV && !pc) continue;
          const double v = b.idensity_s[gidx(s, g, cl)];
          c.ion(s, i) = prm.use_improved_ion_advection ? v : log(v);
        }
      } else {
        const GitmModVerticalBatch& b = M.mv;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          c.x(F_LNS + s, i) = b.log_ns[gidx(s, g, cl)];
          c.x(F_W + s, i) = b.vert_vel[gidx(s, g, cl)];
        }
        c.x(F_T, i) = b.temp[gidx(0, g, cl)];
        c.x(F_VE, i) = b.vel_gd[gidx(0, g, cl)];
        c.x(F_VN, i) = b.vel_gd[gidx(1, g, cl)];
        c.x(F_VU, i) = b.vel_gd[gidx(2, g, cl)];
        c.x(F_LRHO, i) = b.log_rho[gidx(0, g, cl)];
        const bool pc = in_pcells(i, nA);
#pragma unroll
        for (int s = 0; s < NI; ++s) {
          if (s >= NADV && !pc) continue;
          c.ion(s, i) = b.log_ins[gidx(s, g, cl)];
        }
        c.cm(i) = (g >= 1 && g <= nA + 2) ? b.cmax[gidx(0, g, cl)] : 0.0;
        c.gm(i) = b.gamma[gidx(0, g, cl)];
        c.tu(i) = 1.0;
        if (i == -1) c.sc(SC_MMM_M1) = b.mean_major_mass[gidx(0, g, cl)];
        if (i == 0) c.sc(SC_MMM_0) = b.mean_major_mass[gidx(0, g, cl)];
      }
    }
    __syncthreads();  // @phase 0
    if constexpr (SAVE) {
      save_state(0);
      __syncthreads();  // the boundary pass rewrites what was just saved
    }

    // per-item constants for the step
    double eddy = 0.0, ivup = 0.0;
    double accr[ACC_GLOBAL ? 1 : NF];

    for (int step = 0; step < kp.n_steps; ++step) {
      if (item) {
        if (IO == 0) {
          eddy = M.b.eddy[gidx(0, my_i + 1, my_cl)];
          ivup = M.b.ivel_up[gidx(0, my_i + 1, my_cl)];
        } else {
          eddy = M.mv.eddy[gidx(0, my_i + 1, my_cl)];
          ivup = M.mv.ivel[gidx(2, my_i + 1, my_cl)];
        }
      }
      // ---------------------------------------------------- first BC pass
      boundaries();
      __syncthreads();  // @phase 1
      save_state(1);
      // Orig = state (vertical_solver_rusanov.f90:95-100); read first in
      // phase B, after the barrier that ends phase A
      {
        const int xo = cur ? L.X1 : L.X0;  // X and its passive cells are contiguous
        const int per = NF * G + NPAS * NPC;
        for (int w = tid; w < nc * per; w += NT) {
          const int cl = w / per, r = w - cl * per;
          double* col = sm + size_t(L.stride) * cl;
          if constexpr (OG) {
            const double v = col[xo + r];
            ogb[size_t(cl) * operc + r] = v;
            if (r >= NF * G) {
              col[L.OGH + NF * 4 + (r - NF * G)] = v;
            } else {
              const int f = r / G, g = r - f * G;
              if (g < 2 || g >= nA + 2) col[L.OGH + f * 4 + (g < 2 ? g : g - nA)] = v;
            }
          } else {
            col[L.O + r] = col[xo + r];
          }
        }
      }

      for (int k = 0; k < 4; ++k) {
        // -------------------------------------------------- phase A
        if constexpr (SOLVER == GITM_SOLVER_AUSM) {
          // log T and the hydrostatic prefix sum of each column, then the 32
          // limited slopes of the AUSM stage on cells 0..nAlts+1
          constexpr int nw = NT / 32;
          for (int cl = wid; cl < nc; cl += nw) {
            ColCtx c = ctx(cl);
            for (int i = lane - 1; i <= nA + 2; i += 32) c.col[L.LT + i + 1] = log(c.x(F_T, i));
            __syncwarp();
            ausm_prefix(c, lane);
          }
          __syncthreads();  // @phase 6
          // threads over cells 0..nAlts+1 of every column
          for (int j = tid; j < nc * (nA + 2); j += NT) {
            const int cl = j / (nA + 2), i = j - cl * (nA + 2);
            ColCtx c = ctx(cl);
#pragma unroll 4
            for (int f = 0; f < NSLOPE_AUSM; ++f) c.dl(f, i) = ausm_slope(c, f, i, prm.beta_limiter);
          }
        } else {
          // limited slopes of the 18 swept fields on cells 0..nAlts+1,
          // threads over the cells of every column
          for (int j = tid; j < nc * (nA + 2); j += NT) {
            const int cl = j / (nA + 2), i = j - cl * (nA + 2);
            rusanov_slopes_cell(ctx(cl), i, prm.beta_limiter);
          }
        }
        __syncthreads();  // @phase 2

        // -------------------------------------------------- phase B
        // advance_vertical_1stage (:387-686) at the item's cell; the stage
        // result goes straight into the other buffer as Orig + c_k K_k
        // (vertical_solver_rusanov.f90:120-163,190-232,261-303,350-366)
        const int nxo = cur ? L.X0 : L.X1;
        // the RK4 weights of this stage: accumulator a = prev + ca K (ca = 1,
        // 2, 2, 1), next state Orig + cx K for k < 3 (cx = 1/2, 1/2, 1) and
        // Orig + a / 6 after the last stage; a multiplication by 1 or 2 is
        // exact, so fma(ca, K, prev) rounds like prev + ca K
        const double ca = (k == 1 || k == 2) ? 2.0 : 1.0;
        const double cx = (k < 2) ? 0.5 : (k == 2) ? 1.0 : 1.0 / 6.0;
        if (item) {
          ColCtx c = ctx(my_cl);
          const int i = my_i;
          double* xn = c.col + nxo + 1;  // next buffer, xn[f*G + i]
          auto emit = [&](int f, double kval) {
            const int fa = ACC_GLOBAL ? 0 : f;
            // the first stage starts the accumulator: no read of the slot
            const double prev = (k == 0) ? 0.0 : ACC_GLOBAL ? accg[size_t(f) * NT] : accr[fa];
            const double o = OG ? ogb[size_t(my_cl) * operc + f * G + i + 1] : c.o(f, i);
            double a, x1;
            if constexpr (SOLVER == GITM_SOLVER_AUSM) {
              // Stage(k+2) = Stage1 + (New - state), and the final combination
              // (1/3)(-Stage1 + Stage2 + 2 Stage3 + Stage4 + (New - state))
              // accumulated in the reference's order (vertical_solver_ausm.f90:167-189,381-420)
              if (k < 3) {
                x1 = o + kval;
                a = (k == 0) ? -1.0 * o + x1 : (k == 1) ? prev + 2.0 * x1 : prev + x1;
              } else {
                a = prev;
                x1 = (1.0 / 3.0) * (prev + kval);
              }
            } else {
              a = fma(ca, kval, prev);
              x1 = o + cx * ((k == 3) ? a : kval);
            }
            if constexpr (ACC_GLOBAL) {
              accg[size_t(f) * NT] = a;
            } else {
              accr[fa] = a;
            }
            xn[f * G + i] = x1;
          };
          if constexpr (SOLVER == GITM_SOLVER_AUSM) {
            // advance_vertical_1stage_ausm with DtIn = Dt/2, Dt/2, Dt, Dt/2
            ausm_cell(c, i, prm, (k == 2) ? dt : 0.5 * dt, eddy, ivup, emit, &sst[my_cl]);
          } else {
            rusanov_cell(c, i, prm, dt, eddy, ivup, inv_vert_tau, emit, &sst[my_cl]);
          }
        }
        // ghost cells and passive ions of the next buffer return to Orig
        // (their K is zero)
        {
          const int per = NF * 4 + NPAS * NPC;
          const int nxpo = cur ? L.XP0 : L.XP1;
          for (int w = tid; w < nc * per; w += NT) {
            const int cl = w / per, r = w - cl * per;
            double* col = sm + size_t(L.stride) * cl;
            if (r < NF * 4) {
              const int f = r >> 2, u = r & 3;
              const int g = (u < 2) ? u : nA + u;  // cells -1,0,nA+1,nA+2
              col[nxo + f * G + g] = OG ? col[L.OGH + r] : col[L.O + f * G + g];
            } else {
              col[nxpo + r - NF * 4] = OG ? col[L.OGH + r] : col[L.OP + r - NF * 4];
            }
          }
        }
        cur ^= 1;
        __syncthreads();  // @phase 3
        // set_vertical_bcs on the updated state (:166,236,306,368)
        boundaries();
        __syncthreads();  // @phase 1
        save_state(2 + k);
      }

      // ---------------------------------------------------- store / reload
      const bool last = (step == kp.n_steps - 1);
      for (int w = tid; w < nc * G; w += NT) {
        const int g = w / nc, cl = w - g * nc, i = g - 1;
        ColCtx c = ctx(cl);
        const bool store = last && sfrozen[cl] == 0u;
        const bool pc = in_pcells(i, nA);
        if (IO == 1) {
          if (!store) continue;
          const GitmModVerticalBatch& b = M.mv;
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            b.log_ns[gidx(s, g, cl)] = c.x(F_LNS + s, i);
            b.vert_vel[gidx(s, g, cl)] = c.x(F_W + s, i);
          }
          b.temp[gidx(0, g, cl)] = c.x(F_T, i);
          b.vel_gd[gidx(0, g, cl)] = c.x(F_VE, i);
          b.vel_gd[gidx(1, g, cl)] = c.x(F_VN, i);
          b.vel_gd[gidx(2, g, cl)] = c.x(F_VU, i);
          b.log_rho[gidx(0, g, cl)] = c.x(F_LRHO, i);
#pragma unroll
          for (int s = 0; s < NI; ++s)
            if (s < NADV || pc) b.log_ins[gidx(s, g, cl)] = c.ion(s, i);
          continue;
        }
        // scatter, advance_vertical.f90:163-217
        const GitmColumnBatch& b = M.b;
        const double rho = store ? exp(c.x(F_LRHO, i)) : 1.0;
        double temperature = c.x(F_T, i) / c.tu(i);
        // add_sources' temperature line with EuvHeating its only term
        // (add_sources.f90:53-66), applied after every step
        if (IO == 0 && M.b.heating && i >= 1 && i <= nA) {
          const double hs = M.b.heating_scale ? M.b.heating_scale[tile.c0 + cl] : 1.0;
          temperature = temperature + dt * (hs * M.b.heating[gidx(0, g, cl)]);
        }
        double nd[NS], N = 0.0;
        bool finite = isfinite(rho) && isfinite(temperature);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          nd[s] = exp(c.x(F_LNS + s, i));
          N = N + nd[s];
          finite = finite && isfinite(nd[s]) && isfinite(c.x(F_W + s, i));
        }
        const bool improved = prm.use_improved_ion_advection != 0;
        const bool interior = (i >= 1 && i <= nA);
        if (prm.compute_eddy && interior && sfrozen[cl] == 0u) {
          // calc_eddy_diffusion_coefficient (Earth.f90:376-411) on Pressure =
          // Temperature * Rho (calc_pressure.f90:23) of the state this step
          // started from (Orig, with this step's TempUnit): the coefficient
          // the next step reads (calc_sources.f90:26 runs after the vertical
          // advance)
          const double* ocol = OG ? ogb + size_t(cl) * operc : c.col + L.O;
          const double pr = (ocol[F_T * G + i + 1] / c.tu(i)) * exp(ocol[F_LRHO * G + i + 1]);
          double kz = 0.0;
          if (pr > prm.eddy_pressure0)
            kz = prm.eddy_coef;
          else if (pr > prm.eddy_pressure1)
            kz = prm.eddy_coef * (pr - prm.eddy_pressure1) / (prm.eddy_pressure0 - prm.eddy_pressure1);
          b.eddy[gidx(0, g, cl)] = kz;
        }
        if (store) {
          b.rho[gidx(0, g, cl)] = rho;
          b.velocity[gidx(0, g, cl)] = c.x(F_VE, i);
          b.velocity[gidx(1, g, cl)] = c.x(F_VN, i);
          b.velocity[gidx(2, g, cl)] = c.x(F_VU, i);
          b.temperature[gidx(0, g, cl)] = temperature;
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            if (b.log_ns) b.log_ns[gidx(s, g, cl)] = c.x(F_LNS + s, i);
            b.vert_vel[gidx(s, g, cl)] = c.x(F_W + s, i);
            b.ndensity_s[gidx(s, g, cl)] = nd[s];
          }
          if (b.ndensity) b.ndensity[gidx(0, g, cl)] = N;
          if (prm.use_ion_advection) {
            double e = 0.0;
#pragma unroll
            for (int s = 0; s < NI; ++s) {
              double v;
              if (s < NADV || pc) {
                v = c.ion(s, i);
                if (!improved) v = exp(v);
              } else {
                v = b.idensity_s[gidx(s, g, cl)];  // unchanged interior value
              }
              if (improved && interior && v < 1) v = 1.0;
              finite = finite && isfinite(v);
              if (s < NADV || pc || v != b.idensity_s[gidx(s, g, cl)]) b.idensity_s[gidx(s, g, cl)] = v;
              e = e + v;
            }
            b.idensity_s[gidx(NI, g, cl)] = e;
          }
          if (!finite) atomicOr(&sst[cl], GITM_ST_NONFINITE);
        }
        if (!last) {
          // the next step's gather from the values just formed
          double gamma = c.gm(i), mmm = 0.0, tu = c.tu(i), cmx = c.cm(i);
          bool bad = false;
#pragma unroll
          for (int s = 0; s < NS; ++s) bad = bad || !(nd[s] > 0.0);
          if (bad) atomicOr(&sst[cl], GITM_ST_NEG_DENSITY);
          if (prm.compute_coefficients) {
            double gg = 0.0;
#pragma unroll
            for (int s = 0; s < NS; ++s) gg = gg + nd[s] * c_k.inv_vib2[s];
            gamma = gg * 2.0 / N + 1;
            double m = 0.0;
            const double rn = 1.0 / (N + 1.0);
#pragma unroll
            for (int s = 0; s < NS; ++s) m = m + c_k.mass[s] * nd[s] * rn;
            if (m == 0) m = c_k.mass[0];
            mmm = m;
            tu = m * (1.0 / KB);
            cmx = 0.0;
            if (g >= 1 && g <= nA + 2) {
              double mx = fabs(c.x(F_W, i));
#pragma unroll
              for (int s = 1; s < NS; ++s) mx = fmax(mx, fabs(c.x(F_W + s, i)));
              cmx = mx + sqrt(gamma * temperature);
            }
            if (step + 1 == kp.n_steps - 1) {
              if (b.gamma) b.gamma[gidx(0, g, cl)] = gamma;
              if (b.mean_major_mass) b.mean_major_mass[gidx(0, g, cl)] = mmm;
              if (b.temp_unit) b.temp_unit[gidx(0, g, cl)] = tu;
              if (b.cmax && g >= 1 && g <= nA + 2) b.cmax[gidx(0, g, cl)] = cmx;
            }
            c.gm(i) = gamma;
            c.cm(i) = cmx;
            c.tu(i) = tu;
            if (i == -1) c.sc(SC_MMM_M1) = mmm;
            if (i == 0) c.sc(SC_MMM_0) = mmm;
          }
          // LogNS = log(NDensityS) and LogRho = log(Rho) of the next gather
          // (advance_vertical.f90:105,114) give back the values in X up to a
          // rounding of exp/log, so X keeps them
          c.x(F_T, i) = temperature * tu;
          if (prm.use_ion_advection) {
#pragma unroll
            for (int s = 0; s < NI; ++s) {
              if (!(s < NADV || pc)) continue;
              double v = c.ion(s, i);
              if (!improved) v = exp(v);
              if (improved && interior && v < 1) v = 1.0;
              c.ion(s, i) = improved ? v : log(v);
            }
          }
        }
      }
      __syncthreads();  // @phase 5
    }

    if (tid < nc) {
      const int64_t gcol = M.col_offset + tile.c0 + tid;
      uint32_t w = sst[tid];
      if (sfrozen[tid]) w |= GITM_ST_NEG_DENSITY;
      if (w) kp.status[gcol] |= w;
    }
    __syncthreads();
  }
}

}  // namespace gv
