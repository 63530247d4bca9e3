// vert_adjoint.cuh -- reverse-mode derivative of one vertical step (Rusanov
// solver, GITM-array form): gitm_vert_plan_adjoint.
//
// The reference has no adjoint; this is the hand-written reverse of the
// forward kernel of vert_kernel.cuh, statement by statement, with every
// branch (limiter case, clamp, boundary switch, max of |w|) differentiated on
// the side the forward took.
//
// One CTA per tile of columns, persistent over tiles.  The CTA first re-runs
// the step forward (gather, producers, boundaries, four stages) and saves
// the six states it needs -- the gathered state, the post-boundary stage
// inputs X0..X3 and the final X4 -- to a per-CTA slot of global scratch
// (L2-resident under the persistent grid).  The reverse sweep then runs from
// the scatter back to the gather:
//   scatter^T -> bc^T(X4) -> RK combination^T -> for k = 3..0:
//     load X_k, recompute its slopes, stage_k^T at every interior cell
//     (one thread per cell writes its own cell's adjoint; the sweeps'
//     shares of the neighbouring cells go by shuffles within a warp, through
//     a small edge buffer across warps; GradLogConS's are left in shared
//     memory), the gather of those shares (one thread per cell), slopes^T
//     (one thread per field and run of cells), bc^T(X_k) and the
//     combination^T of X_k
//   -> bc^T(X0) -> gather^T and producers^T.
// Shared memory per column: the state, its adjoint, the adjoint of Orig, the
// slopes and their adjoints, the per-cell coefficients and their adjoints.
#pragma once

#include "vert_kernel.cuh"

namespace gv {

struct AdjLayout {
  Layout L;  // X0: the state; X1: its adjoint; O: the adjoint of Orig
  int DB, GU, FB, CMB, GMB, TUB, MMB, LC, stride;
};

__host__ __device__ inline AdjLayout make_adj_layout(int nAlts) {
  AdjLayout A;
  A.L = make_layout(nAlts);
  const int G = nAlts + 4;
  int o = A.L.stride;
  A.DB = o;  o += NSTENCIL * (nAlts + 2);
  // GradLogConS's -Eddy vb_s of interior cell i at [s * nAlts + i - 1], and
  // their sum (for LogRho) at s = NS: cell_gather hands them to the
  // neighbouring cells
  A.GU = o;  o += (NS + 1) * nAlts;
  // the dissipation coefficients' adjoints of interior cell i (halved): its
  // lower face at [i - 1], its upper face at [nAlts + i - 1]
  A.FB = o;  o += 2 * nAlts;
  A.CMB = o; o += G;
  A.GMB = o; o += G;
  A.TUB = o; o += G;
  A.MMB = o; o += 4;  // MeanMajorMass at cells -1, 0; the heating-factor sum
  A.LC = o;  o += (NSTENCIL * (nAlts + 2) + 7) / 8;  // limiter branch per slope, one byte each
  A.stride = o;
  return A;
}

constexpr int ADJ_NSTATE = 6;    // gathered state, X0, X1, X2, X3, X4
// threads per CTA of the adjoint kernel (2 columns of 50 cells per CTA; 64
// threads with one column measured 3 % slower) and of the saving step kernel
constexpr int ADJ_THREADS = 128;
constexpr int SAVE_THREADS = 128;
// The stage adjoint's shares that cross a warp boundary inside a column: per
// boundary (lane 31 of warp b | lane 0 of warp b+1) and swept field, the
// value and slope shares to the right cell and to the left cell.
constexpr int ADJ_EDGE_DOUBLES = (ADJ_THREADS / 32 - 1) * NSTENCIL * 4;

// The columns' slots, the edge shares, then the status words.
__host__ __device__ inline size_t adj_smem_bytes(int nAlts, int nc) {
  return (size_t(make_adj_layout(nAlts).stride) * nc + ADJ_EDGE_DOUBLES) * sizeof(double) +
         size_t(nc) * 2 * sizeof(uint32_t);
}

// Defined in vert_adjoint.cu (the kernel's own translation unit).
const void* adjoint_kernel_fn();
const void* adjoint_kernel_fn_n50();  // members of exactly 50 altitudes
cudaError_t adjoint_set_consts(const Consts& k);
cudaError_t adjoint_set_consts_n50(const Consts& k);
__host__ __device__ inline int adj_state_doubles(int nAlts) { return NF * (nAlts + 4) + NPAS * NPC; }

constexpr int ADJ_INLINE_BARS = 4;  // members whose descriptors travel in the kernel parameters

struct AParams {
  const DevMember* members;
  const GitmColumnAdjoint* bars;      // device array (more members than fit inline)
  GitmColumnAdjoint bars_inline[ADJ_INLINE_BARS];
  int n_inline;                       // > 0: use bars_inline
  const Tile* tiles;
  int n_tiles;
  int nc_max;
  int per_max;             // adj_state_doubles of the largest member
  double dt;
  uint32_t* status;
  double* scratch;
  size_t scratch_per_cta;  // doubles
  GitmVertParams prm;
  // states saved by the SAVE step kernel (gitm_vert_plan_advance_saving),
  // state s of global column c at saved[(s * saved_ncols + c) * per_max];
  // NULL: the kernel recomputes them
  const double* saved;
  int64_t saved_ncols;
};

// ---------------------------------------------------------------- helpers
// The branch of limiter_mc (ModLimiter.f90:16-36) at (u, d) that its
// derivative follows: 0 a zero slope, 1 the slope is beta u, 2 it is beta d,
// 3 it is the mean (u + d) / 2 (ties go to the first candidate of the
// forward's min / max).  The slope's adjoint ob then gives u the adjoint
// beta ob (1) or ob / 2 (3), and d beta ob (2) or ob / 2 (3).
__device__ __forceinline__ int limiter_mc_branch(double u, double d, double beta) {
  const double bu = beta * u, bd = beta * d, av = (u + d) * 0.5;
  const bool pos = (u > 0.0) && (d > 0.0);
  const bool neg = !(u > 0.0) && (d < 0.0);
  const int cp = (fmin(bu, bd) <= av) ? ((bu <= bd) ? 1 : 2) : 3;
  const int cn = (fmax(bu, bd) >= av) ? ((bu >= bd) ? 1 : 2) : 3;
  return pos ? cp : (neg ? cn : 0);
}

// Where a cell's neighbour is held in the stage adjoint: the next lane of
// the same warp, a ghost cell (no thread; only this cell gives it shares
// there), or a cell of the neighbouring warp.
enum NbKind : int { NB_LANE = 0, NB_GHOST = 1, NB_WARP = 2 };

// Per-column view of the adjoint arrays in shared memory.
struct ColAdj {
  double* xb;    // adjoint of the state, [f*G + cell+1]
  double* xbp;   // its passive-ion cells
  double* ob;    // adjoint of Orig
  double* obp;
  double* db;    // slope adjoints [f*(nAlts+2) + cell]
  double* gu;    // GradLogConS's -Eddy vb_s [s*nAlts + i-1]; their sum at s = NS
  double* fb;    // the dissipation coefficients' adjoints, halved [i-1], [nAlts + i-1]
  double* cmb;   // cMax adjoint [cell+1]
  double* gmb;   // Gamma adjoint
  double* tub;   // TempUnit adjoint
  double* mmb;   // MeanMajorMass(-1), MeanMajorMass(0), heating-factor sum
  uint8_t* lc;   // limiter branch of each slope [f*(nAlts+2) + cell] (limiter_mc_branch)
  int G, nA;
  // the stage adjoint of interior cells (one thread per cell): the warp's
  // lanes holding cells, where this cell's neighbours are, the CTA's edge
  // shares and this thread's warp
  unsigned mask;
  int nbl, nbr;
  double* eb;
  int wid;

  __device__ __forceinline__ double& x(int f, int i) const { return xb[f * G + i + 1]; }
  __device__ __forceinline__ double& ion(int s, int i) const {
    return (s < NADV) ? xb[(F_I + s) * G + i + 1] : xbp[(s - NADV) * NPC + pcell(i, nA)];
  }
  // In the stage adjoint the value and slope adjoints of interior cell i
  // are written by its own thread alone (the neighbours' shares reach it by
  // shuffles, or later through cell_gather), those of the ghost cells by
  // the end cells' threads alone.
  __device__ __forceinline__ void own(int f, int i, double v) const { xb[f * G + i + 1] += v; }
  // a sweep's value share xv and slope share dv for neighbour cell j of kind
  // nb (not NB_LANE); side 0: j = i+1, side 1: j = i-1
  __device__ __forceinline__ void give(int f, int j, double xv, double dv, int nb, int side) const {
    if (nb == NB_GHOST) {
      own(f, j, xv);
      db[f * (nA + 2) + j] += dv;
    } else {
      double* e = eb + ((wid - side) * NSTENCIL + f) * 4 + 2 * side;
      e[0] += xv;
      e[1] += dv;
    }
  }
};

// ---------------------------------------------------------------- boundaries^T
// Reverse of bc_column for one column, by a full warp with lanes over
// species and ions as in bc_column.  part 1 = lower half, 2 = upper half,
// 3 = both.  c: the post-boundary state; a: its adjoint, replaced by the
// adjoint of the pre-boundary state (ghost cells the boundary overwrites get
// 0, ghost cells it reads before overwriting get their contribution);
// pre / prep: the pre-boundary state's cells and passive-ion cells (the
// values of the ion ghosts the top boundary reads).  Follows
// set_vertical_bcs.Earth.f90:8-652 as bc_column does, in reverse.  The
// lower half writes the adjoints of cells <= 5, the upper one of cells
// >= nAlts-4.
__device__ inline void bc_column_adjoint(const ColCtx& c, const ColAdj& a, const double* pre,
                                         const double* prep, const GitmVertParams& prm, int lane,
                                         uint32_t* st, int part) {
  const int nA = c.L.nAlts;
  const int G = c.L.G;
  const double* sc = c.col + c.L.SC;
  const int s = lane;
  auto X = [&](int f, int i) -> double { return c.x(f, i); };
  auto XI = [&](int q, int i) -> double { return c.ion(q, i); };
  auto PI = [&](int q, int i) -> double {
    return (q < NADV) ? pre[(F_I + q) * G + i + 1] : prep[(q - NADV) * NPC + pcell(i, nA)];
  };
  const double* bl = sc + SC_BCC;       // lower mesh coefficients: cell 0 then -1
  const double* bu = sc + SC_BCC + 10;  // upper: nA+1 then nA+2
  auto dAF = [&](int i) { return c.dAF(i); };

  if (part & 2) {
    // the pre-boundary ion ghosts (global memory) read first, so that their
    // latency overlaps the LogRho pass
    double pg1 = 0.0, pg2 = 0.0;
    if (s < NI) {
      pg1 = PI(s, nA + 1);
      pg2 = PI(s, nA + 2);
    }
    // lines 598-604: LogRho of the two top ghosts (both cells' sums first)
    {
      double ms1 = 0.0, ms2 = 0.0;
      if (s < NS) {
        ms1 = c_k.mass[s] * exp(X(F_LNS + s, nA + 1));
        ms2 = c_k.mass[s] * exp(X(F_LNS + s, nA + 2));
      }
      const double r1 = lane_seq_sum(ms1, NS);
      const double r2 = lane_seq_sum(ms2, NS);
      const double lb1 = a.x(F_LRHO, nA + 1), lb2 = a.x(F_LRHO, nA + 2);
      __syncwarp();
      if (s < NS) {
        a.x(F_LNS + s, nA + 1) += lb1 * ms1 / r1;
        a.x(F_LNS + s, nA + 2) += lb2 * ms2 / r2;
      }
      if (s == 0) {
        a.x(F_LRHO, nA + 1) = 0.0;
        a.x(F_LRHO, nA + 2) = 0.0;
      }
    }
    __syncwarp();
    // lines 488-596: ions, one per lane.  With UseImprovedIonAdvection the
    // logs of the extrapolation are taken lane-parallel first, as bc_column
    // takes them: lg[7 s + j] = log(pre-boundary ion s at nAlts+2-j), j =
    // 0..6; the ghost values the forward set (exp of its extrapolations) are
    // read from the post-boundary state, and the log of the first one is its
    // exponent y, as bc_column uses it.
    {
      const bool improved = prm.use_improved_ion_advection != 0;
      double tp = 0.0;
      bool neg = false;
      double* lg = c.col + c.L.DL;  // scratch: the slopes are dead during the boundary adjoint
      static_assert(NI * 9 <= NSTENCIL * (8 + 2), "the ion logs and ghosts fit the slope region at nAlts >= 8");
      if (improved) {
        for (int i = 1 + lane; i <= nA; i += 32) tp += c.dAF(i) * XI(0, i);
        if (s < NI) {
          neg = (pg1 < 0.0) || (pg2 < 0.0);
          for (int q = nA - 5; q <= nA; ++q) neg = neg || (XI(s, q) < 0.0);
          lg[NI * 7 + s] = pg2;
          lg[NI * 8 + s] = pg1;
        }
        __syncwarp();
        for (int q = lane; q < NI * 7; q += 32) {
          const int si = q / 7, j = q - si * 7;
          const int cell = nA + 2 - j;
          lg[q] = log((j < 2) ? lg[NI * (7 + j) + si] : XI(si, cell));
        }
      } else {
        for (int i = 1 + lane; i <= nA; i += 32) tp += c.dAF(i) * exp(XI(0, i));
      }
      for (int off = 16; off > 0; off >>= 1) tp += __shfl_xor_sync(0xffffffffu, tp, off);
      // the forward's test (bc_column): TEC < MinTEC * 1e16
      const bool hold = (tp < prm.min_tec * 1e16) && (sc[SC_PLASMA] != 0.0);
      const bool anyneg = __any_sync(0xffffffffu, neg);
      __syncwarp();
      const double dT = dAF(nA);
      if (anyneg) {
        if (lane == 0) atomicOr(st, GITM_ST_ADJ_BRANCH);
      } else if (!hold && s < NI) {
        const double* C = bu;
        const double* D = bu + 5;
        if (improved) {
          const double* n = lg + s * 7 + 1;  // n[k] = log(ion at nAlts+1-k), k = 0..5
          const double g0 = lg[s * 7];
          const double dnr = C[0] * n[1] + C[1] * n[2] + C[2] * n[3] + C[3] * n[4] + C[4] * n[5];
          const double lim = -(0.001 * n[0] / dT);
          const bool t1 = dnr > lim;
          const double dn = t1 ? lim : dnr;
          const double y = n[1] + dn * dAF(nA + 1);
          const double v1 = XI(s, nA + 1);  // exp(y)
          const double dn2r = D[0] * y + D[1] * n[1] + D[2] * n[2] + D[3] * n[3] + D[4] * n[4];
          const double lim2 = -(0.001 * g0 / dT);
          const bool t2 = dn2r > lim2;
          const double v2 = XI(s, nA + 2);  // exp(y + dn2 dAF(nAlts+2))
          double nb[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
          const double v2b = a.ion(s, nA + 2);
          a.ion(s, nA + 2) = 0.0;
          const double e2 = v2b * v2;
          double yb = e2;
          const double dn2b = e2 * dAF(nA + 2);
          if (t2) {
            a.ion(s, nA + 2) += (dn2b * (-0.001 / dT)) / pg2;
          } else {
            yb += D[0] * dn2b;
            for (int q = 1; q < 5; ++q) nb[q] += D[q] * dn2b;
          }
          const double e1 = a.ion(s, nA + 1) * v1 + yb;
          a.ion(s, nA + 1) = 0.0;
          nb[1] += e1;
          const double dnb = e1 * dAF(nA + 1);
          if (t1) {
            a.ion(s, nA + 1) += (dnb * (-0.001 / dT)) / pg1;
          } else {
            for (int q = 0; q < 5; ++q) nb[q + 1] += C[q] * dnb;
          }
          for (int j = 1; j < 6; ++j) a.ion(s, nA + 1 - j) += nb[j] / XI(s, nA + 1 - j);
        } else {
          const double dn1r = C[0] * XI(s, nA) + C[1] * XI(s, nA - 1) + C[2] * XI(s, nA - 2) +
                              C[3] * XI(s, nA - 3) + C[4] * XI(s, nA - 4);
          const bool t1 = dn1r > -(0.001 * pg1 / dT);
          const double v1 = XI(s, nA + 1);
          const double dn2r = D[0] * v1 + D[1] * XI(s, nA) + D[2] * XI(s, nA - 1) + D[3] * XI(s, nA - 2) +
                              D[4] * XI(s, nA - 3);
          const bool t2 = dn2r > -(0.001 * pg2 / dT);
          const double v2b = a.ion(s, nA + 2);
          a.ion(s, nA + 2) = 0.0;
          double v1b = a.ion(s, nA + 1) + v2b;
          a.ion(s, nA + 1) = 0.0;
          const double dn2b = v2b * dAF(nA + 2);
          if (t2) {
            a.ion(s, nA + 2) += dn2b * (-0.001 / dT);
          } else {
            v1b += D[0] * dn2b;
            for (int q = 1; q < 5; ++q) a.ion(s, nA + 1 - q) += D[q] * dn2b;
          }
          a.ion(s, nA) += v1b;
          const double dn1b = v1b * dAF(nA + 1);
          if (t1) {
            a.ion(s, nA + 1) += dn1b * (-0.001 / dT);
          } else {
            for (int q = 0; q < 5; ++q) a.ion(s, nA - q) += C[q] * dn1b;
          }
        }
      }
    }
    __syncwarp();
    // lines 420-486: species winds and hydrostatic densities, one per lane
    double tb = 0.0;
    if (s < NS) {
      const double T = X(F_T, nA);
      const double wn = X(F_W + s, nA);
      const double w1b = a.x(F_W + s, nA + 1), w2b = a.x(F_W + s, nA + 2);
      a.x(F_W + s, nA + 1) = 0.0;
      a.x(F_W + s, nA + 2) = 0.0;
      if (photochemical(s) && wn < 0.0) {
        a.x(F_W + s, nA) -= w1b;
        a.x(F_W + s, nA - 1) -= w2b;
      } else {
        a.x(F_W + s, nA) += w1b + w2b;
      }
      const double ish1 = (-0.5 * (sc[SC_EG + 3] + sc[SC_EG + 2])) * c_k.mass[s] / (0.5 * (T + T) * KB);
      const double ish2 = (-0.5 * (sc[SC_EG + 4] + sc[SC_EG + 3])) * c_k.mass[s] / (0.5 * (T + T) * KB);
      const double lb2 = a.x(F_LNS + s, nA + 2);
      a.x(F_LNS + s, nA + 2) = 0.0;
      const double l1b = lb2 + a.x(F_LNS + s, nA + 1);
      a.x(F_LNS + s, nA + 1) = 0.0;
      const double ish2b = -sc[SC_DAF + 5] * lb2;
      a.x(F_LNS + s, nA) += l1b;
      const double ish1b = -sc[SC_DAF + 4] * l1b;
      tb = -(ish1b * ish1 + ish2b * ish2) / T;
    }
    tb = lane_seq_sum(tb, NS);
    if (s == 0) {
      // lines 466-469: Temp(nA+1:nA+2) = Temp(nA)
      a.x(F_T, nA) += tb + a.x(F_T, nA + 1) + a.x(F_T, nA + 2);
      a.x(F_T, nA + 1) = 0.0;
      a.x(F_T, nA + 2) = 0.0;
      // lines 455-463: Vel_GD up = |Vel_GD up (nA)|
      const double v = X(F_VU, nA);
      const double sg = (v < 0.0) ? -1.0 : (v > 0.0 ? 1.0 : 0.0);
      a.x(F_VU, nA) += sg * (a.x(F_VU, nA + 1) + a.x(F_VU, nA + 2));
      a.x(F_VU, nA + 1) = 0.0;
      a.x(F_VU, nA + 2) = 0.0;
      // lines 420-430: horizontal winds
      for (int f = F_VE; f <= F_VN; ++f) {
        a.x(f, nA) += a.x(f, nA + 1) + a.x(f, nA + 2);
        a.x(f, nA + 1) = 0.0;
        a.x(f, nA + 2) = 0.0;
      }
    }
    __syncwarp();
  }

  if (part & 1) {
    const bool msis = prm.use_msis_bcs && sc[SC_HASLBC] != 0.0;
    const double* C0 = bl;
    const double* C1 = bl + 5;
    // this lane's species winds of cells 0 and -1 as the extrapolation of
    // lines 334-344 left them (lines 382-395 may flip them afterwards)
    double w0e = 0.0, wm1e = 0.0;
    if (s < NS) {
      const double d0 = X(F_W + s, 1) * C0[0] + X(F_W + s, 2) * C0[1] + X(F_W + s, 3) * C0[2] +
                        X(F_W + s, 4) * C0[3] + X(F_W + s, 5) * C0[4];
      w0e = X(F_W + s, 1) - sc[SC_DAF + 2] * d0;
      const double d1 = w0e * C1[0] + X(F_W + s, 1) * C1[1] + X(F_W + s, 2) * C1[2] + X(F_W + s, 3) * C1[3] +
                        X(F_W + s, 4) * C1[4];
      wm1e = w0e - sc[SC_DAF + 1] * d1;
      // lines 382-395: photochemical sign flip
      if (photochemical(s) && X(F_W + s, 1) > 0.0) {
        a.x(F_W + s, 1) -= a.x(F_W + s, 0) + a.x(F_W + s, -1);
        a.x(F_W + s, 0) = 0.0;
        a.x(F_W + s, -1) = 0.0;
      }
    }
    // lines 364-376: MSIS winds of cell -1
    if (msis && s == 0) {
      for (int f = F_VE; f <= F_VN; ++f) {
        const double b = a.x(f, -1);
        a.x(f, -1) = 0.0;
        a.x(f, 0) += b;
        for (int q = 0; q < 5; ++q) a.x(f, q) += -sc[SC_DAF + 1] * C1[q] * b;
      }
    }
    __syncwarp();
    // lines 348-362: LogRho and bulk vertical wind of cells 0 and -1 (both
    // cells' sums first)
    {
      double ms0 = 0.0, msm = 0.0;
      if (s < NS) {
        ms0 = c_k.mass[s] * exp(X(F_LNS + s, 0));
        msm = c_k.mass[s] * exp(X(F_LNS + s, -1));
      }
      const double r0 = lane_seq_sum(ms0, NS);
      const double mw0 = lane_seq_sum(ms0 * w0e, NS);
      const double rm = lane_seq_sum(msm, NS);
      const double mwm = lane_seq_sum(msm * wm1e, NS);
      const double lrb0 = a.x(F_LRHO, 0), vub0 = a.x(F_VU, 0);
      const double lrbm = a.x(F_LRHO, -1), vubm = a.x(F_VU, -1);
      __syncwarp();
      const double rb0 = lrb0 / r0 - vub0 * mw0 / (r0 * r0);
      const double mwb0 = vub0 / r0;
      const double rbm = lrbm / rm - vubm * mwm / (rm * rm);
      const double mwbm = vubm / rm;
      if (s < NS) {
        a.x(F_W + s, 0) += mwb0 * ms0;
        a.x(F_LNS + s, 0) += (rb0 + mwb0 * w0e) * ms0;
        a.x(F_W + s, -1) += mwbm * msm;
        a.x(F_LNS + s, -1) += (rbm + mwbm * wm1e) * msm;
      }
      if (s == 0) {
        a.x(F_LRHO, 0) = 0.0;
        a.x(F_VU, 0) = 0.0;
        a.x(F_LRHO, -1) = 0.0;
        a.x(F_VU, -1) = 0.0;
      }
      __syncwarp();
    }
    // lines 304-310: ions float
    if (s < NI) {
      a.ion(s, 1) += a.ion(s, 0) + a.ion(s, -1);
      a.ion(s, 0) = 0.0;
      a.ion(s, -1) = 0.0;
    }
    // lines 205-272 and 334-344, one species per lane
    double l0b = 0.0, tb = 0.0, mb = 0.0;
    if (s < NS) {
      {  // winds: cell -1 from cell 0 (new), then cell 0 from the interior
        const double b = a.x(F_W + s, -1);
        a.x(F_W + s, -1) = 0.0;
        a.x(F_W + s, 0) += b * (1.0 - sc[SC_DAF + 1] * C1[0]);
        for (int q = 1; q < 5; ++q) a.x(F_W + s, q) += -sc[SC_DAF + 1] * C1[q] * b;
        const double b0 = a.x(F_W + s, 0);
        a.x(F_W + s, 0) = 0.0;
        a.x(F_W + s, 1) += b0 * (1.0 - sc[SC_DAF + 2] * C0[0]);
        for (int q = 1; q < 5; ++q) a.x(F_W + s, 1 + q) += -sc[SC_DAF + 2] * C0[q] * b0;
      }
      if (!photochemical(s)) {
        const double b = a.x(F_LNS + s, -1);
        a.x(F_LNS + s, -1) = 0.0;
        if (s == 0) {
          a.x(F_LNS + s, 0) += b;
        } else {
          l0b = b;
          const double ishb = b * sc[SC_DAF + 0];
          const double mg = -0.5 * (sc[SC_EG + 0] + sc[SC_EG + 1]);
          const double mt = 0.5 * (X(F_T, 0) + X(F_T, -1));
          const double mm = 0.5 * (sc[SC_MMM_0] + sc[SC_MMM_M1]);
          const double ish = mg * mm / (mt * KB);
          mb = ishb * mg / (mt * KB);
          tb = 0.5 * (-ishb * ish / mt);
        }
      } else {
        for (int k = 1; k >= 0; --k) {
          const int i = -k;
          const double* C = bl + 5 * k;
          const double d = X(F_LNS + s, i + 1) * C[0] + X(F_LNS + s, i + 2) * C[1] + X(F_LNS + s, i + 3) * C[2] +
                           X(F_LNS + s, i + 4) * C[3] + X(F_LNS + s, i + 5) * C[4];
          const double up = X(F_LNS + s, i + 1);
          const double dF = sc[SC_DAF + 2 + i];
          double v = up - dF * d;
          const bool flat = d <= 0.0;
          if (flat) v = up;
          const bool floor = (s == 4) && (v < up - 0.333);
          const double b = a.x(F_LNS + s, i);
          a.x(F_LNS + s, i) = 0.0;
          a.x(F_LNS + s, i + 1) += b;
          if (!flat && !floor) {
            const double dbv = -dF * b;
            for (int q = 0; q < 5; ++q) a.x(F_LNS + s, i + 1 + q) += C[q] * dbv;
          }
        }
      }
    }
    mb = lane_seq_sum(mb, NS);
    tb = lane_seq_sum(tb, NS);
    if (s == 0) {
      a.mmb[0] += 0.5 * mb;
      a.mmb[1] += 0.5 * mb;
      a.x(F_T, 0) += tb;
      a.x(F_T, -1) += tb;
      // lines 192-196
      for (int f : {F_T, F_VE, F_VN, F_VU}) {
        a.x(f, 0) += a.x(f, -1);
        a.x(f, -1) = 0.0;
      }
      // lines 112-148
      a.x(F_VU, 0) = 0.0;
      a.x(F_VE, 0) = 0.0;
      a.x(F_VN, 0) = 0.0;
      if (msis) {
        a.x(F_T, 0) = 0.0;
        a.x(F_LRHO, 0) = 0.0;
        a.x(F_LRHO, -1) = 0.0;
      }
    }
    if (s < NS) {
      a.x(F_W + s, 0) = 0.0;
      a.x(F_W + s, -1) = 0.0;
      if (msis) {
        a.x(F_LNS + s, -1) = 0.0;
        a.x(F_LNS + s, 0) = l0b;
      } else {
        a.x(F_LNS + s, 0) += l0b;
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- stage^T
// Reverse of rusanov_cell at interior cell i, in two passes that each hold
// only their own part of the cell's values (one pass over everything held
// the friction matrix, the species terms and all field adjoints at once and
// spilled): cell_adjoint_species (continuity and momentum of the species,
// the friction solve, LogRho) and cell_adjoint_rest (temperature, the
// horizontal winds, the bulk vertical wind's own terms, the ions).  kb(f)
// is the adjoint of New for field f (the caller applies K = New - state);
// contributions go to the state adjoint (this cell and its neighbours), the
// slope adjoints, the cMax and Gamma adjoints.  Every sweep adjoint is
// linear in its inputs, so the two passes' shares of the temperature
// sweep add up.

// The face geometry of cell i and its sweep (calc_rusanov_alts_rusanov,
// vertical_solver_rusanov.f90:694-718), forward and reverse.
struct CellFaces {
  double dF0, dF1, idc, fc0, fc1;
  double hF0, hF1, hidc;  // the halves of dF0, dF1, idc (a product with 0.5 is exact)
  double fc0b, fc1b;  // adjoints of the two dissipation coefficients

  __device__ __forceinline__ CellFaces(const ColCtx& c, int i) {
    dF0 = c.dAF(i);
    dF1 = c.dAF(i + 1);
    idc = c.g(GC_IDC, i);
    hF0 = 0.5 * dF0;
    hF1 = 0.5 * dF1;
    hidc = 0.5 * idc;
    fc0 = 0.5 * fmax(c.cm(i - 1), c.cm(i));
    fc1 = 0.5 * fmax(c.cm(i), c.cm(i + 1));
    fc0b = 0.0;
    fc1b = 0.0;
  }
  __device__ __forceinline__ void sweep(const ColCtx& c, int f, int i, double& grad, double& diff) const {
    const double* v = &c.col[c.xo + f * c.L.G + 1];
    const double* d = &c.col[c.L.DL + f * (c.L.nAlts + 2)];
    const double L0 = fma(d[i - 1], hF0, v[i - 1]);
    const double R0 = fma(-d[i], hF0, v[i]);
    const double L1 = fma(d[i], hF1, v[i]);
    const double R1 = fma(-d[i + 1], hF1, v[i + 1]);
    grad = (L1 + R1 - L0 - R0) * hidc;
    diff = (fc1 * (R1 - L1) - fc0 * (R0 - L0)) * idc;
  }
  // (gb, dbv) -> faces -> values and slopes; returns this cell's value
  // share, with what the neighbouring cells of the same warp give it (by
  // shuffles), and adds its slope share with theirs; the shares of ghost
  // cells and of cells in the neighbouring warp go by give().
  __device__ __forceinline__ double sweep_adj(const ColCtx& c, const ColAdj& a, int f, int i, double gb,
                                              double dbv) {
    const double* v = &c.col[c.xo + f * c.L.G + 1];
    const double* d = &c.col[c.L.DL + f * (c.L.nAlts + 2)];
    const double L0 = fma(d[i - 1], hF0, v[i - 1]);
    const double R0 = fma(-d[i], hF0, v[i]);
    const double L1 = fma(d[i], hF1, v[i]);
    const double R1 = fma(-d[i + 1], hF1, v[i + 1]);
    const double hg = hidc * gb;
    const double L1b = hg - fc1 * idc * dbv, R1b = hg + fc1 * idc * dbv;
    const double L0b = -hg + fc0 * idc * dbv, R0b = -hg - fc0 * idc * dbv;
    fc1b += idc * (R1 - L1) * dbv;
    fc0b += -idc * (R0 - L0) * dbv;
    const double dl = hF0 * L0b;               // to the slope of cell i-1
    const double dm = -hF0 * R0b + hF1 * L1b;  // this cell's slope
    const double dr = -hF1 * R1b;              // the slope of cell i+1
    const double xr = __shfl_down_sync(a.mask, L0b, 1);  // cell i+1's share of this cell
    const double drr = __shfl_down_sync(a.mask, dl, 1);
    const double xl = __shfl_up_sync(a.mask, R1b, 1);    // cell i-1's
    const double dll = __shfl_up_sync(a.mask, dr, 1);
    double own = R0b + L1b, down = dm;
    if (a.nbl == NB_LANE) {
      own += xl;
      down += dll;
    } else {
      a.give(f, i - 1, L0b, dl, a.nbl, 1);
    }
    if (a.nbr == NB_LANE) {
      own += xr;
      down += drr;
    } else {
      a.give(f, i + 1, R1b, dr, a.nbr, 0);
    }
    a.db[f * (a.nA + 2) + i] += down;
    return own;
  }
  // the dissipation coefficients' adjoints (fc = 0.5 max(cMax, cMax') at
  // each face), kept for cell_gather, which hands them to the cMax of the
  // side each max took; acc: add to what the cell's other pass kept
  __device__ __forceinline__ void keep_fc(const ColAdj& a, int i, bool acc) const {
    double& b0 = a.fb[i - 1];
    double& b1 = a.fb[a.nA + i - 1];
    b0 = acc ? b0 + 0.5 * fc0b : 0.5 * fc0b;
    b1 = acc ? b1 + 0.5 * fc1b : 0.5 * fc1b;
  }
};

// Species continuity and momentum (:548-617), the friction solve
// (calc_neutral_friction.f90:47-106), the clamp and LogRho / the bulk wind's
// species terms (:643-658) in reverse.  kb(f) = kbp[f * kstride].  Returns
// the KappaEddyDiffusion adjoint of the cell.
__device__ inline double cell_adjoint_species(const ColCtx& c, const ColAdj& a, int i, const GitmVertParams& prm,
                                              double dt, double eddy, const double* kbp, int kstride) {
  auto kb = [&](int f) { return kbp[size_t(f) * kstride]; };
  CellFaces fa(c, i);
  // ---- forward recompute
  const double invr = c.g(GC_INVR, i), rr = c.g(GC_R, i), grav = c.g(GC_GRAV, i);
  const double T = c.x(F_T, i), VE = c.x(F_VE, i), VN = c.x(F_VN, i);
  const double LR = c.x(F_LRHO, i);
  double gT, dT;
  fa.sweep(c, F_T, i, gT, dT);
  const double itau = 1.0 / (prm.use_damping ? 15 - (1 - exp(-1.0 * c.g(GC_ALT, i) / 1000.0 / 40.0)) * 5.0
                                             : prm.vert_tau);
  const double hz = (VN * VN + VE * VE) * invr;
  const double cor = prm.use_coriolis ? dt * (c.sc(SC_CENT) * rr + c.sc(SC_CORI) * VE) : 0.0;
  double wv[NS], menl[NS];
  double sumrho = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double gL, dL, gW, dW;
    fa.sweep(c, F_LNS + s, i, gL, dL);
    fa.sweep(c, F_W + s, i, gW, dW);
    const double Ls = c.x(F_LNS + s, i), Ws = c.x(F_W + s, i);
    const double divw = gW + 2 * Ws * invr;
    const double nl = Ls - dt * (divw + Ws * gL) + dt * dL;
    menl[s] = c_k.mass[s] * exp(nl);
    sumrho = sumrho + menl[s];
    const double km = c_k.k_over_m[s];
    double w = Ws - dt * (Ws * gW - hz + T * gL * km + gT * km - grav) + dt * dW - Ws * itau;
    w = w + cor;
    w = w - dt * (prm.thermal_diff_coef[s] * km) * gT;
    wv[s] = w;
  }
  double ns[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) ns[s] = exp(c.x(F_LNS + s, i));
  const double ir = exp(-LR);
  // reverse of New LogRho = log(sumrho): the continuity adjoints, with
  // New LogNS's own adjoint
  double nlb[NS];
  {
    const double srb = kb(F_LRHO) / sumrho;
#pragma unroll
    for (int s = 0; s < NS; ++s) nlb[s] = srb * menl[s] + kb(F_LNS + s);
  }
  double Tb = 0.0, VEb = 0.0, VNb = 0.0, LRb = 0.0, irb = 0.0;
  double nsb[NS], wb[NS], lself[NS];  // lself: GradLogConS's share of this cell's LogNS adjoint
  double eddyb = 0.0;
  // New VU = sum_s w_s m_s ns_s / Rho; New VertVel = the clamped w
  const double kvu = kb(F_VU);
  if (prm.use_neutral_friction) {
    double glc[NS], lu[NS][NS], vsol[NS], pw[NS];
    grad_log_cons(c, i, glc);
    const double lt = log(T);
#pragma unroll
    for (int e = 0; e < NS; ++e) pw[e] = exp(c_k.one_minus_e[e] * lt);
#pragma unroll
    for (int r = 0; r < NS; ++r) {
      double rs = 0.0;
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        if (q == r) continue;
        const double cij = c_k.kc[r][q] * ns[q] * pw[exp_index(r, q)];
        lu[r][q] = -dt * cij;
        rs = rs + cij;
      }
      lu[r][r] = 1.0 + dt * rs;
    }
    // LU without pivoting: multipliers below the diagonal, pivot
    // reciprocals on it (as friction_solve)
#pragma unroll
    for (int p = 0; p < NS; ++p) {
      const double ip = 1.0 / lu[p][p];
      lu[p][p] = ip;
#pragma unroll
      for (int r = p + 1; r < NS; ++r) {
        const double l = lu[r][p] * ip;
        lu[r][p] = l;
#pragma unroll
        for (int q = p + 1; q < NS; ++q) lu[r][q] -= l * lu[p][q];
      }
    }
#pragma unroll
    for (int r = 0; r < NS; ++r) {
      double sum = wv[r];
#pragma unroll
      for (int q = 0; q < r; ++q) sum -= lu[r][q] * vsol[q];
      vsol[r] = sum;
    }
#pragma unroll
    for (int r = NS - 1; r >= 0; --r) {
      double sum = vsol[r];
#pragma unroll
      for (int q = r + 1; q < NS; ++q) sum -= lu[r][q] * vsol[q];
      vsol[r] = sum * lu[r][r];
    }
    // clamp, bulk wind and their reverse
    double vb[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double v = vsol[s] + (-eddy * glc[s]);
      const bool inside = !(v < -prm.max_vertical_velocity) && !(v > prm.max_vertical_velocity);
      double wc = fmax(-prm.max_vertical_velocity, v);
      wc = fmin(prm.max_vertical_velocity, wc);
      const double m = c_k.mass[s];
      const double wcb = kvu * (m * ns[s] * ir) + kb(F_W + s);
      nsb[s] = kvu * wc * m * ir;
      irb += kvu * wc * m * ns[s];
      vb[s] = inside ? wcb : 0.0;
      eddyb -= vb[s] * glc[s];
    }
    // GradLogConS: 5-point mesh on log(m_s) + LogNS - LogRho.  This
    // cell's own share here; u_s = -Eddy vb_s (and their sum, for LogRho)
    // left for cell_gather, which gives cells i-2, i-1, i+1, i+2 theirs
    {
      const double mc = c.g(GC_M0 + 2, i);
      double lrb = 0.0, ul = 0.0;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const double u = -eddy * vb[s];
        a.gu[s * a.nA + i - 1] = u;
        ul += u;
        const double v = u * mc;
        lrb -= v;
        lself[s] = v;
      }
      a.gu[NS * a.nA + i - 1] = ul;
      LRb += lrb;
    }
    // wb = M^-T vb with M = L U: U^T z = vb, then L^T wb = z
#pragma unroll
    for (int r = 0; r < NS; ++r) {
      double sum = vb[r];
#pragma unroll
      for (int q = 0; q < r; ++q) sum -= lu[q][r] * wb[q];
      wb[r] = sum * lu[r][r];
    }
#pragma unroll
    for (int r = NS - 1; r >= 0; --r) {
      double sum = wb[r];
#pragma unroll
      for (int q = r + 1; q < NS; ++q) sum -= lu[q][r] * wb[q];
      wb[r] = sum;
    }
    // M_rq = -dt C_rq (q != r), M_rr = 1 + dt sum_q C_rq:  Cb_rq = dt wb_r (vsol_q - vsol_r)
    double pwb[NS];
#pragma unroll
    for (int e = 0; e < NS; ++e) pwb[e] = 0.0;
#pragma unroll
    for (int r = 0; r < NS; ++r)
#pragma unroll
      for (int q = 0; q < NS; ++q) {
        if (q == r) continue;
        const double cb = dt * wb[r] * (vsol[q] - vsol[r]);
        const double k = c_k.kc[r][q];
        nsb[q] += cb * k * pw[exp_index(r, q)];
        pwb[exp_index(r, q)] += cb * k * ns[q];
      }
    double ltb = 0.0;
#pragma unroll
    for (int e = 0; e < NS; ++e) ltb += pwb[e] * pw[e] * c_k.one_minus_e[e];
    Tb += ltb / T;
  } else {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double v = wv[s];
      const bool inside = !(v < -prm.max_vertical_velocity) && !(v > prm.max_vertical_velocity);
      double wc = fmax(-prm.max_vertical_velocity, v);
      wc = fmin(prm.max_vertical_velocity, wc);
      const double m = c_k.mass[s];
      const double wcb = kvu * (m * ns[s] * ir) + kb(F_W + s);
      nsb[s] = kvu * wc * m * ir;
      irb += kvu * wc * m * ns[s];
      wb[s] = inside ? wcb : 0.0;
      lself[s] = 0.0;
      a.gu[s * a.nA + i - 1] = 0.0;
    }
    a.gu[NS * a.nA + i - 1] = 0.0;
  }
  // species momentum, continuity and their sweeps
  double gTb = 0.0, hzb = 0.0, corb = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double gL, dL, gW, dW;
    fa.sweep(c, F_LNS + s, i, gL, dL);
    fa.sweep(c, F_W + s, i, gW, dW);
    const double Ws = c.x(F_W + s, i);
    const double km = c_k.k_over_m[s];
    const double w = wb[s];
    double Wb = w * (1.0 - dt * gW - itau);
    double gWb = -dt * Ws * w;
    hzb += dt * w;
    Tb += -dt * gL * km * w;
    double gLb = -dt * T * km * w;
    gTb += -dt * km * w - dt * (prm.thermal_diff_coef[s] * km) * w;
    const double dWb = dt * w;
    corb += w;
    // New LogNS = nl = Ls - dt (divw + Ws gL) + dt dL
    const double n = nlb[s];
    double Lb = lself[s] + n;
    const double divwb = -dt * n;
    Wb += -dt * gL * n + 2 * invr * divwb;
    gLb += -dt * Ws * n;
    const double dLb = dt * n;
    gWb += divwb;
    Lb += fa.sweep_adj(c, a, F_LNS + s, i, gLb, dLb);
    Wb += fa.sweep_adj(c, a, F_W + s, i, gWb, dWb);
    Lb += nsb[s] * ns[s];
    a.own(F_LNS + s, i, Lb);
    a.own(F_W + s, i, Wb);
  }
  LRb -= irb * ir;
  if (prm.use_coriolis) VEb += corb * dt * c.sc(SC_CORI);
  VNb += hzb * 2 * VN * invr;
  VEb += hzb * 2 * VE * invr;
  // the species' share of the temperature sweep
  Tb += fa.sweep_adj(c, a, F_T, i, gTb, 0.0);
  fa.keep_fc(a, i, false);
  a.own(F_T, i, Tb);
  a.own(F_VE, i, VEb);
  a.own(F_VN, i, VNb);
  a.own(F_LRHO, i, LRb);
  return eddyb;
}

// Temperature, horizontal winds, the bulk vertical wind's own terms and the
// ions (:557-568, :660-680) in reverse.
__device__ inline void cell_adjoint_rest(const ColCtx& c, const ColAdj& a, int i, double dt, double ivup,
                                         const double* kbp, int kstride) {
  auto kb = [&](int f) { return kbp[size_t(f) * kstride]; };
  // the New adjoints this pass reads
  double ki[NADV];
#pragma unroll
  for (int s = 0; s < NADV; ++s) ki[s] = kb(F_I + s);
  const double kE = kb(F_VE), kN = kb(F_VN), kT = kb(F_T);
  CellFaces fa(c, i);
  const double invr = c.g(GC_INVR, i);
  const double T = c.x(F_T, i), VU = c.x(F_VU, i);
  const double gm = c.gm(i);
  double gT, dT, gE, dE, gN, dN, gU, dU;
  fa.sweep(c, F_T, i, gT, dT);
  fa.sweep(c, F_VE, i, gE, dE);
  fa.sweep(c, F_VN, i, gN, dN);
  fa.sweep(c, F_VU, i, gU, dU);
  const double divv = gU + 2 * VU * invr;
  // ions: New = I - dt (IVel gI) + dt dI
#pragma unroll
  for (int s = 0; s < NADV; ++s) {
    const double k = ki[s];
    const double own = fa.sweep_adj(c, a, F_I + s, i, -dt * ivup * k, dt * k);
    a.own(F_I + s, i, k + own);
  }
  // horizontal winds: New = V - dt VU gV + dt dV
  double VEb = kE + fa.sweep_adj(c, a, F_VE, i, -dt * VU * kE, dt * kE);
  double VNb = kN + fa.sweep_adj(c, a, F_VN, i, -dt * VU * kN, dt * kN);
  double VUb = -dt * gE * kE - dt * gN * kN;
  // temperature: New = T - dt (VU gT + (Gamma - 1) T divv) + dt dT
  double Tb = kT;
  VUb += -dt * gT * kT;
  const double gTb = -dt * VU * kT;
  const double gmb = -dt * T * divv * kT;
  Tb += -dt * (gm - 1.0) * divv * kT;
  const double divvb = -dt * (gm - 1.0) * T * kT;
  VUb += 2 * invr * divvb;
  Tb += fa.sweep_adj(c, a, F_T, i, gTb, dt * kT);
  VUb += fa.sweep_adj(c, a, F_VU, i, divvb, 0.0);
  fa.keep_fc(a, i, true);
  a.gmb[i + 1] += gmb;
  a.own(F_T, i, Tb);
  a.own(F_VE, i, VEb);
  a.own(F_VN, i, VNb);
  a.own(F_VU, i, VUb);
}

// The limited slopes of cell i (interior: 4th-order form; cells 0 and
// nAlts+1: 2nd-order form), as rusanov_slopes_cell forms them, with each
// slope's limiter branch recorded for slopes_adjoint_window.
__device__ inline void slopes_with_branches(const ColCtx& c, const ColAdj& a, int i, double beta) {
  const int nA = c.L.nAlts;
  const bool end = (i == 0 || i == nA + 1);
  const double cu = end ? c.g(GC_IDF, i + 1) : c.g(GC_H2, i + 1);
  const double cd = end ? c.g(GC_IDF, i) : c.g(GC_H2, i);
  // both forms in one expression, as rusanov_slopes_cell
  const double fa = end ? 1.0 : F1, fb = end ? 0.0 : F2;
  const int ip2 = min(i + 2, nA + 2), im2 = max(i - 2, -1);
  // state, slopes and branch bytes are disjoint regions (restrict: the
  // loads of later fields may be issued ahead of earlier stores)
  const double* __restrict__ xv = c.col + c.xo + 1;
  double* __restrict__ sl = c.col + c.L.DL + i;
  uint8_t* __restrict__ br = a.lc + i;
#pragma unroll 3
  for (int f = 0; f < NSTENCIL; ++f) {
    const double* v = xv + f * c.L.G;
    const double u = cu * (fa * (v[i + 1] - v[i]) - fb * (v[ip2] - v[i - 1]));
    const double d = cd * (fa * (v[i] - v[i - 1]) - fb * (v[i + 1] - v[im2]));
    sl[f * (nA + 2)] = limiter_mc(u, d, beta);
    br[f * (nA + 2)] = uint8_t(limiter_mc_branch(u, d, beta));
  }
}

// Adjoint of the limited slopes into the state adjoint, on the branches
// slopes_with_branches recorded.  The slope of cell i is limiter_mc(u, d)
// with u = cu (fa (v[i+1] - v[i]) - fb (v[i+2] - v[i-1])) and d = cd (fa
// (v[i] - v[i-1]) - fb (v[i+1] - v[i-2])) (fa = 1, fb = 0 at the end
// cells); its adjoint ob gives u the adjoint ub and d the adjoint dbv by
// the branch, and those go to cells i-2..i+2.  One thread walks the slopes
// of field f along cells j0-2..j1+2 and owns the state cells j0..j1
// (within -1..nAlts+2): each slope is read once, its five shares are kept
// in a window of partial sums, and a cell is written once it is complete
// (no atomics).
__device__ inline void slopes_adjoint_window(const ColCtx& c, const ColAdj& a, int f, int j0, int j1,
                                             double beta) {
  const int nA = c.L.nAlts;
  const double* __restrict__ dbp = a.db + f * (nA + 2);
  const uint8_t* __restrict__ lcp = a.lc + f * (nA + 2);
  // the state adjoint of field f (a region apart from the inputs: the loads
  // of later cells may go ahead of the stores)
  double* __restrict__ xo = a.xb + f * a.G + 1;
  double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0, w4 = 0.0;  // partial sums of cells i-2 .. i+2
#pragma unroll 2
  for (int i = j0 - 2; i <= j1 + 2; ++i) {
    const bool ok = (i >= 0 && i <= nA + 1);  // slopes exist at cells 0..nAlts+1
    const int ic = min(max(i, 0), nA + 1);
    const bool end = (ic == 0 || ic == nA + 1);
    const double cu = end ? c.g(GC_IDF, ic + 1) : c.g(GC_H2, ic + 1);
    const double cd = end ? c.g(GC_IDF, ic) : c.g(GC_H2, ic);
    const double fa = end ? 1.0 : F1, fb = end ? 0.0 : F2;
    const double ob = ok ? dbp[ic] : 0.0;
    const int br = lcp[ic];
    const double ub = (br == 1) ? beta * ob : (br == 3) ? 0.5 * ob : 0.0;
    const double dbv = (br == 2) ? beta * ob : (br == 3) ? 0.5 * ob : 0.0;
    w4 += -cu * fb * ub;                   // cell i+2
    w3 += cu * fa * ub - cd * fb * dbv;    // cell i+1
    w2 += -cu * fa * ub + cd * fa * dbv;   // cell i
    w1 += cu * fb * ub - cd * fa * dbv;    // cell i-1
    w0 += cd * fb * dbv;                   // cell i-2: complete
    if (i - 2 >= j0) xo[i - 2] += w0;
    w0 = w1;
    w1 = w2;
    w2 = w3;
    w3 = w4;
    w4 = 0.0;
  }
}

// What reaches state cell m (-1..nAlts+2) of one column from the other
// cells after the stage adjoint: GradLogConS's shares (u_s mc_q of interior
// cell j = m - q + 2, q != 2, to LogNS_s; -sum_s u_s mc_q to LogRho) and,
// when cell m and its neighbour sit on the two sides of a warp boundary,
// the sweeps' shares the edge buffer holds.  One thread per cell: every
// value and slope adjoint of the cell is written by that thread alone.
// t0: the thread of the column's cell 1; nitems: threads holding cells.
__device__ inline void cell_gather(const ColCtx& c, const ColAdj& a, int m, int t0, int nitems) {
  const int nA = c.L.nAlts;
  double mc[4];
  int jj[4];
  bool ok[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int d = (k < 2) ? k - 2 : k - 1;  // source cell m + d, d = -2, -1, 1, 2
    const int j = m + d;
    ok[k] = (j >= 1 && j <= nA);
    jj[k] = ok[k] ? j : 1;
    mc[k] = ok[k] ? c.g(GC_M0 + 2 - d, j) : 0.0;
  }
#pragma unroll
  for (int s = 0; s <= NS; ++s) {
    const double* u = a.gu + s * nA - 1;
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) v += ok[k] ? u[jj[k]] * mc[k] : 0.0;
    a.x((s < NS) ? F_LNS + s : F_LRHO, m) += (s < NS) ? v : -v;
  }
  // cMax of cell m: the dissipation coefficients of the faces whose max
  // took it (cells m and m+1 at their lower faces, cells m-1 and m at their
  // upper faces), in that order
  {
    double cb = 0.0;
    const double cmm = c.cm(m - (m > -1 ? 1 : 0)), cm0 = c.cm(m), cmp = c.cm(m + (m < nA + 2 ? 1 : 0));
    if (m + 1 >= 1 && m + 1 <= nA && cm0 >= cmp) cb += a.fb[m];              // cell m+1, lower face
    if (m >= 1 && m <= nA && !(cmm >= cm0)) cb += a.fb[m - 1];               // cell m, lower face
    if (m >= 1 && m <= nA && cm0 >= cmp) cb += a.fb[nA + m - 1];             // cell m, upper face
    if (m - 1 >= 1 && m - 1 <= nA && !(cmm >= cm0)) cb += a.fb[nA + m - 2];  // cell m-1, upper face
    a.cmb[m + 1] += cb;
  }
  // the edge shares (interior cells): t = this cell's thread
  if (m >= 1 && m <= nA) {
    const int t = t0 + m - 1;
    const int lane = t & 31;
    int bnd = -1, side = 0;
    if (lane == 0 && m > 1) {
      bnd = (t >> 5) - 1;  // the right cell of boundary bnd: what lane 31 gave it
      side = 0;
    } else if (lane == 31 && m < nA && t + 1 < nitems) {
      bnd = t >> 5;  // the left cell: what lane 0 of the next warp gave it
      side = 1;
    }
    if (bnd >= 0) {
#pragma unroll 2
      for (int f = 0; f < NSTENCIL; ++f) {
        const double* e = a.eb + (bnd * NSTENCIL + f) * 4 + 2 * side;
        a.x(f, m) += e[0];
        a.db[f * (nA + 2) + m] += e[1];
      }
    }
  }
}

// 8-byte asynchronous global -> shared copy (cp.async: no register round
// trip, every copy of a thread in flight at once); cp_async_wait_all waits
// for the calling thread's copies.
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------- the kernel
// NA > 0: every member has exactly NA altitudes (the host checks), so the
// layout offsets and loop bounds are compile-time constants; NA = 0 reads
// nAlts from the member.
template <int NT, int NA = 0>
__global__ void __launch_bounds__(NT, 1) vert_adjoint_kernel(const AParams kp) {
  static_assert(NT == ADJ_THREADS, "the edge-share buffer is sized for ADJ_THREADS");
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int wid = tid >> 5;
  constexpr int nw = NT / 32;
  const GitmVertParams& prm = kp.prm;
  const double dt = kp.dt;
  double* cta = kp.scratch + size_t(blockIdx.x) * kp.scratch_per_cta;
  double* acc = cta + size_t(ADJ_NSTATE) * kp.nc_max * kp.per_max + tid;  // [NF] stride NT
  double* kbs = acc + size_t(NF) * NT;                                     // [NF] stride NT

  for (int tix = blockIdx.x; tix < kp.n_tiles; tix += gridDim.x) {
    const Tile tile = kp.tiles[tix];
    const DevMember& M = kp.members[tile.member];
    const GitmColumnAdjoint B = (kp.n_inline > 0) ? kp.bars_inline[tile.member] : kp.bars[tile.member];
    const GitmColumnBatch& b = M.b;
    const int nA = (NA > 0) ? NA : b.n_alts;
    const int nc = tile.nc;
    const AdjLayout A = make_adj_layout(nA);
    const Layout& L = A.L;
    const int G = L.G;
    const int per = adj_state_doubles(nA);
    const int64_t ncols = b.n_cols;
    double* const eb = sm + size_t(A.stride) * nc;  // [ADJ_EDGE_DOUBLES]
    uint32_t* sst = reinterpret_cast<uint32_t*>(eb + ADJ_EDGE_DOUBLES);
    uint32_t* sfrozen = sst + nc;
    const int nitems = nc * nA;
    const bool item = tid < nitems;
    const int my_cl = item ? tid / nA : 0;
    const int my_i = item ? tid % nA + 1 : 1;
    // the stage adjoint's neighbours of this thread's cell (cells of a
    // column are consecutive threads)
    const unsigned imask = __ballot_sync(0xffffffffu, item);
    const int nbl = (my_i == 1) ? NB_GHOST : (lane == 0) ? NB_WARP : NB_LANE;
    const int nbr = (my_i == nA) ? NB_GHOST : (lane == 31) ? NB_WARP : NB_LANE;
    int cur = 0;

    auto ctx = [&](int cl) {
      ColCtx c;
      c.col = sm + size_t(A.stride) * cl;
      c.L = L;
      c.gridc = M.gridc;
      c.gcols = M.gcols;
      c.gc = (M.gcols == 1) ? 0 : int(tile.c0 + cl);
      c.xo = cur ? L.X1 : L.X0;
      c.xpo = cur ? L.XP1 : L.XP0;
      return c;
    };
    auto adj = [&](int cl) {
      ColAdj a;
      double* col = sm + size_t(A.stride) * cl;
      a.xb = col + L.X1;
      a.xbp = col + L.XP1;
      a.ob = col + L.O;
      a.obp = col + L.OP;
      a.db = col + A.DB;
      a.gu = col + A.GU;
      a.fb = col + A.FB;
      a.cmb = col + A.CMB;
      a.gmb = col + A.GMB;
      a.tub = col + A.TUB;
      a.mmb = col + A.MMB;
      a.lc = reinterpret_cast<uint8_t*>(col + A.LC);
      a.G = G;
      a.nA = nA;
      a.mask = imask;
      a.nbl = nbl;
      a.nbr = nbr;
      a.eb = eb;
      a.wid = wid;
      return a;
    };
    auto gidx = [&](int f, int g, int cl) -> int64_t { return (int64_t(f) * G + g) * ncols + tile.c0 + cl; };
    auto state = [&](int s, int cl) -> double* {
      if (kp.saved)
        return const_cast<double*>(kp.saved) +
               (int64_t(s) * kp.saved_ncols + M.col_offset + tile.c0 + cl) * kp.per_max;
      return cta + (size_t(s) * kp.nc_max + cl) * kp.per_max;
    };
    auto save = [&](int s, int off) {
      for (int cl = 0; cl < nc; ++cl) {
        const double* src = sm + size_t(A.stride) * cl + off;
        double* dst = state(s, cl);
        for (int r = tid; r < per; r += NT) dst[r] = src[r];
      }
    };
    // (the caller's barrier publishes the copies)
    auto load = [&](int s, int off) {
      for (int cl = 0; cl < nc; ++cl) {
        const double* src = state(s, cl);
        double* dst = sm + size_t(A.stride) * cl + off;
        for (int r = tid; r < per; r += NT) cp_async8(dst + r, src + r);
      }
      cp_async_wait_all();
    };
    // dst[r] += src[r], src[r] = 0 over the state-sized slots of every column
    auto fold = [&](int dst_off, int src_off) {
      for (int cl = 0; cl < nc; ++cl) {
        double* col = sm + size_t(A.stride) * cl;
        for (int r = tid; r < per; r += NT) {
          col[dst_off + r] += col[src_off + r];
          col[src_off + r] = 0.0;
        }
      }
    };
    auto boundaries = [&]() {
      if (2 * nc <= nw) {
        if (wid < 2 * nc) bc_column(ctx(wid >> 1), prm, lane, &sst[wid >> 1], 1 + (wid & 1));
      } else {
        for (int cl = wid; cl < nc; cl += nw) bc_column(ctx(cl), prm, lane, &sst[cl], 3);
      }
    };
    // bc^T of every column on the state in X0 with the pre-boundary ghost
    // values of saved state s_pre; a warp per column, or per column half
    // when the halves' interior cells are disjoint
    auto boundaries_adjoint = [&](int s_pre) {
      if (2 * nc <= nw && nA >= 10) {
        if (wid < 2 * nc) {
          const int cl = wid >> 1;
          const double* pre = state(s_pre, cl);
          bc_column_adjoint(ctx(cl), adj(cl), pre, pre + NF * G, prm, lane, &sst[cl], 1 + (wid & 1));
        }
      } else {
        for (int cl = wid; cl < nc; cl += nw) {
          const double* pre = state(s_pre, cl);
          bc_column_adjoint(ctx(cl), adj(cl), pre, pre + NF * G, prm, lane, &sst[cl], 3);
        }
      }
    };

    if (tid < nc) {
      sst[tid] = 0u;
      sfrozen[tid] = 0u;
    }
    __syncthreads();

    // ------------------------------------------------------------ gather
    // as the forward kernel's load (IO = 0), into X0
    if (tid < nc) {
      ColCtx c = ctx(tid);
      const int64_t cc = tile.c0 + tid;
      const double cl = b.cos_lat[cc];
      const double cent = (cl * prm.omega_body) * (cl * prm.omega_body);
      c.sc(SC_CENT) = cent;
      c.sc(SC_CORI) = 2 * cl * prm.omega_body;
      const double sza = b.sza[cc], mlat = b.mlat[cc];
      c.sc(SC_SZA) = sza;
      c.sc(SC_MLAT) = mlat;
      bool plasma = false;
      if (prm.use_nighttime_ion_bcs)
        plasma = sza > PI / 2 && ((mlat > 30.0 && mlat < 70.0) || (mlat > -60.0 && mlat < -30.0));
      c.sc(SC_PLASMA) = plasma ? 1.0 : 0.0;
      c.sc(SC_HASLBC) = b.lbc ? 1.0 : 0.0;
      if (b.lbc)
        for (int k = 0; k < 2 * GITM_LBC_NVALUES; ++k) c.sc(SC_LBC + k) = b.lbc[int64_t(k) * ncols + cc];
      for (int j = 0; j < 20; ++j) c.sc(SC_BCC + j) = c.bcc(j);
      const int dcell[6] = {-1, 0, 1, nA, nA + 1, nA + 2};
      for (int j = 0; j < 6; ++j) c.sc(SC_DAF + j) = c.dAF(dcell[j]);
      const int ecell[5] = {-1, 0, nA, nA + 1, nA + 2};
      for (int j = 0; j < 5; ++j) c.sc(SC_EG + j) = c.g(GC_GRAV, ecell[j]) + cent * c.g(GC_R, ecell[j]);
    }
    for (int w = tid; w < nc * G; w += NT) {
      const int g = w / nc, cl = w - g * nc, i = g - 1;
      ColCtx c = ctx(cl);
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
      // with saved stage states the state itself comes from them
      if (kp.saved) continue;
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
    }
    __syncthreads();  // @phase 0
    double eddy = 0.0, ivup = 0.0;
    if (item) {
      eddy = b.eddy[gidx(0, my_i + 1, my_cl)];
      ivup = b.ivel_up[gidx(0, my_i + 1, my_cl)];
    }
    if (kp.saved) {
      // the step's states come from the saving forward: X4 into X0
      load(5, L.X0);
      __syncthreads();
    } else {
      save(0, L.X0);
      __syncthreads();  // @phase 0
      boundaries();
      __syncthreads();  // @phase 1
      save(1, L.X0);
      // Orig := X0
      for (int cl = 0; cl < nc; ++cl) {
        double* col = sm + size_t(A.stride) * cl;
        for (int r = tid; r < per; r += NT) col[L.O + r] = col[L.X0 + r];
      }
      __syncthreads();  // @phase 1

      // ------------------------------------------------------------ forward
      for (int k = 0; k < 4; ++k) {
        for (int j = tid; j < nc * (nA + 2); j += NT) {
          const int cl = j / (nA + 2), i = j - cl * (nA + 2);
          rusanov_slopes_cell(ctx(cl), i, prm.beta_limiter);
        }
        __syncthreads();  // @phase 2
        const int nxo = cur ? L.X0 : L.X1;
        if (item) {
          ColCtx c = ctx(my_cl);
          const int i = my_i;
          double* xn = c.col + nxo + 1;
          auto emit = [&](int f, double kval) {
            double& ag = acc[size_t(f) * NT];
            const double a = (k == 0) ? kval : (k < 3) ? ag + 2.0 * kval : ag + kval;
            ag = a;
            const double o = c.o(f, i);
            xn[f * G + i] = (k < 2) ? o + 0.5 * kval : (k == 2) ? o + kval : o + (1.0 / 6.0) * a;
          };
          rusanov_cell(c, i, prm, dt, eddy, ivup, 1.0 / prm.vert_tau, emit);
        }
        {
          const int pr = NF * 4 + NPAS * NPC;
          const int nxpo = cur ? L.XP0 : L.XP1;
          for (int w = tid; w < nc * pr; w += NT) {
            const int cl = w / pr, r = w - cl * pr;
            double* col = sm + size_t(A.stride) * cl;
            if (r < NF * 4) {
              const int f = r >> 2, u = r & 3;
              const int g = (u < 2) ? u : nA + u;
              col[nxo + f * G + g] = col[L.O + f * G + g];
            } else {
              col[nxpo + r - NF * 4] = col[L.OP + r - NF * 4];
            }
          }
        }
        cur ^= 1;
        __syncthreads();  // @phase 3
        boundaries();
        __syncthreads();  // @phase 4
        save(2 + k, cur ? L.X1 : L.X0);
        __syncthreads();  // @phase 1
      }
    }
    // cur == 0: X4 is in X0

    // ------------------------------------------------------------ reverse
    for (int cl = 0; cl < nc; ++cl) {
      double* col = sm + size_t(A.stride) * cl;
      for (int r = tid; r < per; r += NT) {
        col[L.X1 + r] = 0.0;
        col[L.O + r] = 0.0;
      }
      for (int r = A.DB + tid; r < A.stride; r += NT) col[r] = 0.0;
    }
    __syncthreads();  // @phase 0
    // scatter^T (advance_vertical.f90:163-217 and the heating line).  The
    // cell's output adjoints are read into registers first: read between
    // the shared-memory updates, each load would wait for the one before.
    for (int w = tid; w < nc * G; w += NT) {
      const int g = w / nc, cl = w - g * nc, i = g - 1;
      if (sfrozen[cl]) continue;
      const bool ions = prm.use_ion_advection != 0;
      const bool pc = in_pcells(i, nA);
      const bool interior = (i >= 1 && i <= nA);
      const double y_rho = B.rho[gidx(0, g, cl)];
      const double y_ve = B.velocity[gidx(0, g, cl)];
      const double y_vn = B.velocity[gidx(1, g, cl)];
      const double y_vu = B.velocity[gidx(2, g, cl)];
      const double ytemp = B.temperature[gidx(0, g, cl)];
      const bool heat = b.heating && interior && B.heating_scale;
      const double hq = heat ? b.heating[gidx(0, g, cl)] : 0.0;
      const double yN = B.ndensity ? B.ndensity[gidx(0, g, cl)] : 0.0;
      double y_w[NS], y_nd[NS], y_ln[NS], y_ion[NI];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        y_w[s] = B.vert_vel[gidx(s, g, cl)];
        y_nd[s] = B.ndensity_s[gidx(s, g, cl)];
        y_ln[s] = B.log_ns ? B.log_ns[gidx(s, g, cl)] : 0.0;
      }
      const double ye = ions ? B.idensity_s[gidx(NI, g, cl)] : 0.0;
#pragma unroll
      for (int s = 0; s < NI; ++s) y_ion[s] = (ions && (s < NADV || pc)) ? B.idensity_s[gidx(s, g, cl)] : 0.0;
      ColCtx c = ctx(cl);
      ColAdj a = adj(cl);
      const double tu = c.tu(i);
      const double LR4 = c.x(F_LRHO, i), T4 = c.x(F_T, i);
      a.x(F_LRHO, i) += y_rho * exp(LR4);
      a.x(F_VE, i) += y_ve;
      a.x(F_VN, i) += y_vn;
      a.x(F_VU, i) += y_vu;
      a.x(F_T, i) += ytemp / tu;
      a.tub[i + 1] += -(ytemp * T4 / tu) / tu;
      // the heating factor's adjoint of each interior cell, summed in cell
      // order below (GradLogConS's buffer is free until the stage adjoints)
      if (interior && b.heating && B.heating_scale) a.gu[i - 1] = heat ? ytemp * dt * hq : 0.0;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        a.x(F_W + s, i) += y_w[s];
        const double L4 = c.x(F_LNS + s, i);
        double v = (y_nd[s] + yN) * exp(L4);
        if (B.log_ns) v += y_ln[s];
        a.x(F_LNS + s, i) += v;
      }
      if (ions) {
        const bool improved = prm.use_improved_ion_advection != 0;
#pragma unroll
        for (int s = 0; s < NI; ++s) {
          if (!(s < NADV || pc)) continue;
          const double I4 = c.ion(s, i);
          const double v = improved ? I4 : exp(I4);
          const bool floored = improved && interior && v < 1;
          const double yb = y_ion[s] + ye;
          a.ion(s, i) += floored ? 0.0 : (improved ? yb : yb * v);
        }
      }
    }
    __syncthreads();  // @phase 5
    boundaries_adjoint(1);  // X4's boundaries: pre-boundary ghosts are Orig's
    if (tid < nc && !sfrozen[tid] && b.heating && B.heating_scale) {
      const double* hv = sm + size_t(A.stride) * tid + A.GU;
      double sum = 0.0;
      for (int i = 0; i < nA; ++i) sum += hv[i];
      sm[size_t(A.stride) * tid + A.MMB + 2] += sum;
    }
    __syncthreads();  // @phase 6
    // combination^T of the final: X4pre = Orig + (K0 + 2K1 + 2K2 + K3) / 6
    if (item) {
      ColAdj a = adj(my_cl);
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double ab = (1.0 / 6.0) * a.x(f, my_i);
        acc[size_t(f) * NT] = ab;
        kbs[size_t(f) * NT] = ab;  // K3bar = Abar
      }
    }
    __syncthreads();  // @phase 7
    fold(L.O, L.X1);
    __syncthreads();  // @phase 7

    const double wk[4] = {1.0, 2.0, 2.0, 1.0};
    const double ck[3] = {0.5, 0.5, 1.0};
    double eddy_bar = 0.0;  // the four stages' KappaEddyDiffusion adjoints of this thread's cell
    for (int k = 3; k >= 0; --k) {
      load(1 + k, L.X0);
      for (int cl = 0; cl < nc; ++cl) {
        double* db = sm + size_t(A.stride) * cl + A.DB;
        for (int r = tid; r < NSTENCIL * (nA + 2); r += NT) db[r] = 0.0;
      }
      for (int r = tid; r < ADJ_EDGE_DOUBLES; r += NT) eb[r] = 0.0;
      __syncthreads();  // @phase 8
      for (int j = tid; j < nc * (nA + 2); j += NT) {
        const int cl = j / (nA + 2), i = j - cl * (nA + 2);
        slopes_with_branches(ctx(cl), adj(cl), i, prm.beta_limiter);
      }
      __syncthreads();  // @phase 8
      if (item) {
        ColCtx c = ctx(my_cl);
        ColAdj a = adj(my_cl);
        eddy_bar += cell_adjoint_species(c, a, my_i, prm, dt, eddy, kbs, NT);
        cell_adjoint_rest(c, a, my_i, dt, ivup, kbs, NT);
        // K = New - state: the state's own -K
#pragma unroll
        for (int f = 0; f < NF; ++f) a.own(f, my_i, -kbs[size_t(f) * NT]);
      }
      __syncthreads();  // @phase 9
      // GradLogConS's shares of the neighbouring cells and the sweeps'
      // shares that crossed a warp boundary, one thread per cell
      for (int w = tid; w < nc * G; w += NT) {
        const int cl = w / G, m = w - cl * G - 1;
        cell_gather(ctx(cl), adj(cl), m, cl * nA, nitems);
      }
      __syncthreads();  // @phase 9
      {
        // (column, field, run of cells) per thread
        const int nseg = max(1, NT / (nc * NSTENCIL));
        const int seg = (G + nseg - 1) / nseg;
        for (int w = tid; w < nc * NSTENCIL * nseg; w += NT) {
          const int sg = w % nseg, r = w / nseg, f = r % NSTENCIL, cl = r / NSTENCIL;
          const int j0 = -1 + sg * seg, j1 = min(j0 + seg - 1, nA + 2);
          if (j0 <= j1) slopes_adjoint_window(ctx(cl), adj(cl), f, j0, j1, prm.beta_limiter);
        }
      }
      __syncthreads();  // @phase 10
      if (k > 0) {
        boundaries_adjoint(1);
        __syncthreads();  // @phase 6
        if (item) {
          ColAdj a = adj(my_cl);
#pragma unroll
          for (int f = 0; f < NF; ++f)
            kbs[size_t(f) * NT] = wk[k - 1] * acc[size_t(f) * NT] + ck[k - 1] * a.x(f, my_i);
        }
        __syncthreads();  // @phase 7
        fold(L.O, L.X1);
        __syncthreads();  // @phase 7
      } else {
        // X0 is also Orig
        for (int cl = 0; cl < nc; ++cl) {
          double* col = sm + size_t(A.stride) * cl;
          for (int r = tid; r < per; r += NT) col[L.X1 + r] += col[L.O + r];
        }
        __syncthreads();  // @phase 7
        boundaries_adjoint(0);  // the first boundary pass: pre-boundary values are the gathered ones
        __syncthreads();  // @phase 6
      }
    }

    if (item && B.eddy && !sfrozen[my_cl]) B.eddy[gidx(0, my_i + 1, my_cl)] += eddy_bar;

    // ------------------------------------------------------------ gather^T
    for (int w = tid; w < nc * G; w += NT) {
      const int g = w / nc, cl = w - g * nc, i = g - 1;
      if (sfrozen[cl]) continue;
      // every global value of the cell is read before its first global
      // store (a store could alias a later load, which would then wait)
      const bool ions = prm.use_ion_advection != 0;
      const bool pc = in_pcells(i, nA);
      double nd[NS], ww[NS], ndb[NS], wwb[NS], iv[NI];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        nd[s] = b.ndensity_s[gidx(s, g, cl)];
        ww[s] = b.vert_vel[gidx(s, g, cl)];
      }
      const double temperature = b.temperature[gidx(0, g, cl)];
      const double rho_in = b.rho[gidx(0, g, cl)];
      const double ye = ions ? B.idensity_s[gidx(NI, g, cl)] : 0.0;
#pragma unroll
      for (int s = 0; s < NI; ++s)
        iv[s] = !ions ? 0.0 : (s < NADV || pc) ? b.idensity_s[gidx(s, g, cl)] : B.idensity_s[gidx(s, g, cl)];
      ColCtx c = ctx(cl);
      ColAdj a = adj(cl);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        ndb[s] = a.x(F_LNS + s, i) / nd[s];
        wwb[s] = a.x(F_W + s, i);
      }
      const double tu = c.tu(i);
      double tb = a.x(F_T, i) * tu;
      double tub = a.tub[i + 1] + a.x(F_T, i) * temperature;
      if (prm.compute_coefficients) {
        double N = 0.0, gg = 0.0, ms = 0.0;
#pragma unroll
        for (int s = 0; s < NS; ++s) N = N + nd[s];
#pragma unroll
        for (int s = 0; s < NS; ++s) gg = gg + nd[s] * c_k.inv_vib2[s];
        const double gamma = gg * 2.0 / N + 1;
        const double rn = 1.0 / (N + 1.0);
#pragma unroll
        for (int s = 0; s < NS; ++s) ms = ms + c_k.mass[s] * nd[s];
        double gammab = a.gmb[i + 1];
        if (g >= 1 && g <= nA + 2) {
          const double cb = a.cmb[i + 1];
          int am = 0;
          double mx = fabs(ww[0]);
#pragma unroll
          for (int s = 1; s < NS; ++s)
            if (fabs(ww[s]) > mx) {
              mx = fabs(ww[s]);
              am = s;
            }
          wwb[am] += cb * ((ww[am] < 0.0) ? -1.0 : (ww[am] > 0.0 ? 1.0 : 0.0));
          const double sq = sqrt(gamma * temperature);
          gammab += cb * temperature / (2.0 * sq);
          tb += cb * gamma / (2.0 * sq);
        }
        double mb = tub * (1.0 / KB);
        if (i == -1) mb += a.mmb[0];
        if (i == 0) mb += a.mmb[1];
        const double rnb = mb * ms;
        double Nb = rnb * (-rn * rn);
        const double ggb = gammab * 2.0 / N;
        Nb += -gammab * gg * 2.0 / (N * N);
#pragma unroll
        for (int s = 0; s < NS; ++s) ndb[s] += mb * c_k.mass[s] * rn + ggb * c_k.inv_vib2[s] + Nb;
      }
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        B.ndensity_s[gidx(s, g, cl)] = ndb[s];
        B.vert_vel[gidx(s, g, cl)] = wwb[s];
      }
      B.temperature[gidx(0, g, cl)] = tb;
      B.velocity[gidx(0, g, cl)] = a.x(F_VE, i);
      B.velocity[gidx(1, g, cl)] = a.x(F_VN, i);
      B.velocity[gidx(2, g, cl)] = a.x(F_VU, i);
      B.rho[gidx(0, g, cl)] = a.x(F_LRHO, i) / rho_in;
      if (ions) {
        const bool improved = prm.use_improved_ion_advection != 0;
#pragma unroll
        for (int s = 0; s < NI; ++s) {
          // advected ions: the state value iv; the others: their own
          // output adjoint iv, unchanged by the step, summed into e-
          if (s < NADV || pc)
            B.idensity_s[gidx(s, g, cl)] = improved ? a.ion(s, i) : a.ion(s, i) / iv[s];
          else
            B.idensity_s[gidx(s, g, cl)] = iv[s] + ye;
        }
        B.idensity_s[gidx(NI, g, cl)] = 0.0;
      }
    }
    if (tid < nc && !sfrozen[tid] && b.heating && B.heating_scale)
      B.heating_scale[tile.c0 + tid] += sm[size_t(A.stride) * tid + A.MMB + 2];
    if (tid < nc) {
      const int64_t gcol = M.col_offset + tile.c0 + tid;
      uint32_t wv = sst[tid];
      if (sfrozen[tid]) wv |= GITM_ST_NEG_DENSITY;
      if (wv) kp.status[gcol] |= wv;
    }
    __syncthreads();  // @phase 11
  }
}

}  // namespace gv
