// hz_kernel.cu -- the horizontal advance (advance_horizontal.f90:58-1034) on
// the GPU: gitm_hz_advance's kernel, in its own translation unit.
//
// One CTA per (block, altitude) plane.  The plane's swept fields (Rho,
// Temperature, Velocity, the six NDensityS and VerticalVelocity, the advected
// IDensityS: 19 fields) and its grid metrics are loaded with their two ghost
// rings from GITM's own Fortran-layout arrays (a plane of one field is
// contiguous there, longitude fastest) into shared memory; one thread per
// interior cell runs the four RK stages of :168-345, each stage the whole
// horizontal_solver (:535-818) at the thread's cell: for every field the
// limited slopes of calc_facevalues_lons / _lats (:928-1034) at the cell and
// its two neighbours, the face values, the Rusanov gradient and diffusion
// (calc_rusanov_lons / _lats, :821-922), then the cell's equations.  The
// ghost rings keep their values through the stages, as in the reference.
// The store phase writes the interior cells back with the stores of
// :346-421 and, with UseImprovedIonAdvection, the parallel ion-velocity
// divergence of :423-517 (UAM_Gradient, gradient.f90:4-104) at the cell,
// which reads only IVelocityPar and the grid; the CTA of the first and last
// altitude also rewrite the electron sum of the ghost planes.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/gitm_hz.h"
#include "vert_common.cuh"
#include "vert_hz.cuh"

namespace gv {

namespace {

constexpr int HZ_NSW = 5 + 2 * NS + NADV;  // swept fields
constexpr int NI_ALL = GITM_NIONS - 1;     // ions without the electrons
constexpr int HF_R = 0, HF_T = 1, HF_V = 2, HF_N = 5, HF_W = 5 + NS, HF_I = 5 + 2 * NS;
constexpr int HZ_NGP = 6;   // metric planes with ghost rings: IFB, DFB lon; IFB, DFB lat; cMax E, N
constexpr int HZ_NGC = 7;   // metric values at interior cells: InvD*Dist_GB lon, lat; Gamma; InvR; R; IVel E, N
constexpr double F1 = 0.6250000;  // Factor1, advance_horizontal.f90:939
constexpr double F2 = 0.0416667;  // Factor2, advance_horizontal.f90:940

// Shared-memory plan of one plane: P cells with ghosts, C interior cells.
struct HzLayout {
  int P, C;
  int S, K, G, GC, stride;
};

__host__ __device__ inline HzLayout hz_layout(int nLons, int nLats) {
  HzLayout L;
  L.P = (nLons + 4) * (nLats + 4);
  L.C = nLons * nLats;
  int o = 0;
  L.S = o;  o += HZ_NSW * L.P;
  L.K = o;  o += HZ_NSW * L.C;  // the stage's New - state of every field
  L.G = o;  o += HZ_NGP * L.P;
  L.GC = o; o += HZ_NGC * L.C;
  L.stride = o;
  return L;
}

// Limiter_mc (ModLimiter.f90:16-36) without branches: both candidates are
// formed and the signs select one, so lanes of different cases do not split
// the warp
__device__ __forceinline__ double hz_limiter(double u, double d, double beta) {
  const double bu = beta * u, bd = beta * d, av = (u + d) * 0.5;
  const double lo = fmin(fmin(bu, bd), av), hi = fmax(fmax(bu, bd), av);
  const bool pos = (u > 0.0) && (d > 0.0);
  const bool neg = !(u > 0.0) && (d < 0.0);
  return pos ? lo : (neg ? hi : 0.0);
}

// The limited slope of line cell q (0 .. n+1) as calc_facevalues_lons /
// _lats form it: the 4th-order differences, with the 2nd-order one on the
// outer side of cells 0 and n+1.  V(q) = V[(q+1)*s], IF(q) = IF[(q+1)*s].
__device__ __forceinline__ double hz_slope(const double* V, const double* IF, int s, int q, int n,
                                           double beta) {
  auto v = [&](int x) { return V[(x + 1) * s]; };
  auto f = [&](int x) { return IF[(x + 1) * s]; };
  // both forms in one expression: the 2nd-order side is h * (1 * (...) -
  // 0 * (...)) with h = IF, exactly; the outer neighbours are clamped into
  // the line (finite values the zero factor removes)
  const bool eu = (q == n + 1), ed = (q == 0);
  const double hu = eu ? f(q + 1) : f(q + 1) * 2, hd = ed ? f(q) : f(q) * 2;
  const double au = eu ? 1.0 : F1, bu = eu ? 0.0 : F2, ad = ed ? 1.0 : F1, bd = ed ? 0.0 : F2;
  const double up = hu * (au * (v(q + 1) - v(q)) - bu * (v(min(q + 2, n + 2)) - v(q - 1)));
  const double dn = hd * (ad * (v(q) - v(q - 1)) - bd * (v(q + 1) - v(max(q - 2, -1))));
  return hz_limiter(up, dn, beta);
}

// calc_rusanov_lons / _lats at line cell p (1..n): the gradient and the
// Rusanov diffusion from the face values of faces p and p+1.
__device__ __forceinline__ void hz_line(const double* V, const double* IF, const double* DF, const double* CM,
                                        int s, int p, int n, double invd, double beta, double& grad,
                                        double& diff) {
  const double sm = hz_slope(V, IF, s, p - 1, n, beta);
  const double s0 = hz_slope(V, IF, s, p, n, beta);
  const double sp = hz_slope(V, IF, s, p + 1, n, beta);
  const double vm = V[p * s], v0 = V[(p + 1) * s], vp = V[(p + 2) * s];
  const double d0 = DF[(p + 1) * s], d1 = DF[(p + 2) * s];
  const double W0 = vm + 0.5 * sm * d0;  // VarLeft(p)
  const double E0 = v0 - 0.5 * s0 * d0;  // VarRight(p)
  const double W1 = v0 + 0.5 * s0 * d1;  // VarLeft(p+1)
  const double E1 = vp - 0.5 * sp * d1;  // VarRight(p+1)
  grad = 0.5 * (W1 + E1 - W0 - E0) * invd;
  const double c0 = 0.5 * fmax(CM[p * s], CM[(p + 1) * s]) * (E0 - W0);
  const double c1 = 0.5 * fmax(CM[(p + 1) * s], CM[(p + 2) * s]) * (E1 - W1);
  diff = (c1 - c0) * invd;
}

struct HzArgs {
  GitmHzParams prm;
  GitmHzBlocks b;
  double dt;
  uint32_t* status;  // one word per block
};

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) hz_step_kernel(const HzArgs A) {
  extern __shared__ double sm[];
  const GitmHzBlocks& B = A.b;
  const GitmHzParams& prm = A.prm;
  const int nl = B.n_lons, nt = B.n_lats, na = B.n_alts;
  const int NI = nl + 4, NJ = nt + 4, NK = na + 4;
  const int64_t P = int64_t(NI) * NJ, V = P * NK;
  const int k = blockIdx.x % na + 1;  // Fortran altitude of this plane
  const int b = blockIdx.x / na;
  const int tid = threadIdx.x;
  const HzLayout L = hz_layout(nl, nt);
  const double dt = A.dt;
  // first element of plane k of field f of a block array with nf fields
  auto plane = [&](const double* a, int f, int nf) -> const double* {
    return a + ((int64_t(b) * nf + f) * NK + (k + 1)) * P;
  };
  auto lat1 = [&](const double* a, int j) { return a[int64_t(b) * NJ + (j + 1)]; };

  // ---------------------------------------------------------------- load
  double* S = sm + L.S;
  double* Kc = sm + L.K;
  double* GP = sm + L.G;
  double* GC = sm + L.GC;
  auto src_of = [&](int f) -> const double* {
    if (f == HF_R) return plane(B.rho, 0, 1);
    if (f == HF_T) return plane(B.temperature, 0, 1);
    if (f < HF_N) return plane(B.velocity, f - HF_V, 3);
    if (f < HF_W) return plane(B.ndensity_s, f - HF_N, GITM_NSPECIES_TOTAL);
    if (f < HF_I) return plane(B.vert_vel, f - HF_W, NS);
    return plane(B.idensity_s, f - HF_I, GITM_NIONS);
  };
  for (int f = 0; f < HZ_NSW; ++f) {
    const double* src = src_of(f);
    for (int c = tid; c < P; c += NT) S[f * P + c] = src[c];
  }
  {
    const double* gsrc[4] = {plane(B.inv_dlon_dist_fb, 0, 1), plane(B.dlon_dist_fb, 0, 1),
                             plane(B.inv_dlat_dist_fb, 0, 1), plane(B.dlat_dist_fb, 0, 1)};
    for (int g = 0; g < 4; ++g)
      for (int c = tid; c < P; c += NT) GP[g * P + c] = gsrc[g][c];
    // cMax_GDB(0:nLons+1, 0:nLats+1, 0:nAlts+1, 3, nBlocks): east and north
    // components of this altitude into planes with the outer ghost ring
    // (never read) zeroed
    const int ci2 = nl + 2, cj2 = nt + 2;
    for (int d = 0; d < 2; ++d) {
      const double* cm = B.cmax + (((int64_t(b) * 3 + d) * (na + 2) + k) * cj2) * ci2;
      for (int c = tid; c < P; c += NT) {
        const int i = c % NI - 1, j = c / NI - 1;  // Fortran indices
        const bool in = (i >= 0 && i <= nl + 1 && j >= 0 && j <= nt + 1);
        GP[(4 + d) * P + c] = in ? cm[j * ci2 + i] : 0.0;
      }
    }
  }
  const bool cell = tid < L.C;
  const int ci = cell ? tid % nl + 1 : 1, cj = cell ? tid / nl + 1 : 1;  // Fortran (iLon, iLat)
  const int pc = (cj + 1) * NI + (ci + 1);                                // plane index of the cell
  if (cell) {
    GC[0 * L.C + tid] = plane(B.inv_dlon_dist_gb, 0, 1)[pc];
    GC[1 * L.C + tid] = plane(B.inv_dlat_dist_gb, 0, 1)[pc];
    GC[2 * L.C + tid] = plane(B.gamma, 0, 1)[pc];
    GC[3 * L.C + tid] = plane(B.inv_radial_distance, 0, 1)[pc];
    GC[4 * L.C + tid] = plane(B.radial_distance, 0, 1)[pc];
    GC[5 * L.C + tid] = plane(B.ivelocity, 0, 3)[pc];
    GC[6 * L.C + tid] = plane(B.ivelocity, 1, 3)[pc];
  }
  // Orig (:181-186) stays in the input arrays: they are written only by the
  // store phase, after the last stage

  // per-cell constants of the equations (:680-686)
  double SinLat = 0.0, CosLat = 0.0, TanLat = 0.0;
  if (cell) {
    SinLat = sin(lat1(B.latitude, cj));
    CosLat = lat1(B.cos_latitude, cj);
    TanLat = lat1(B.tan_latitude, cj);
  }
  const double CoriolisSin = SinLat * 2 * prm.omega_body;
  const double CoriolisCos = CosLat * 2 * prm.omega_body;
  const double CentrifugalParameter = (prm.omega_body * prm.omega_body) * CosLat * SinLat;
  const double beta = prm.beta_limiter;
  const double* IFlo = GP + 0 * P;
  const double* DFlo = GP + 1 * P;
  const double* IFla = GP + 2 * P;
  const double* DFla = GP + 3 * P;
  const double* CMe = GP + 4 * P;
  const double* CMn = GP + 5 * P;

  // the Rusanov gradient / diffusion of field f at the cell along lon, lat
  auto lon_of = [&](int f, double& g, double& d) {
    const int row = (cj + 1) * NI;
    hz_line(S + f * P + row, IFlo + row, DFlo + row, CMe + row, 1, ci, nl, GC[0 * L.C + tid], beta, g, d);
  };
  auto lat_of = [&](int f, double& g, double& d) {
    const int col = ci + 1;
    hz_line(S + f * P + col, IFla + col, DFla + col, CMn + col, NI, cj, nt, GC[1 * L.C + tid], beta, g, d);
  };

  double acc[HZ_NSW];
  __syncthreads();

  // ---------------------------------------------------------------- RK4
  for (int st = 0; st < 4; ++st) {
    auto kv = [&](int f) -> double& { return Kc[f * L.C + tid]; };
    if (cell) {
      const double InvR = GC[3 * L.C + tid];
      const double R = S[HF_R * P + pc], T = S[HF_T * P + pc];
      const double VE = S[(HF_V + 0) * P + pc], VN = S[(HF_V + 1) * P + pc], VU = S[(HF_V + 2) * P + pc];
      double gLoR, dLoR, gLaR, dLaR, gLoT, dLoT, gLaT, dLaT;
      double gLoE, dLoE, gLaE, dLaE, gLoN, dLoN, gLaN, dLaN, gLoU, dLoU, gLaU, dLaU;
      lon_of(HF_R, gLoR, dLoR);
      lat_of(HF_R, gLaR, dLaR);
      lon_of(HF_T, gLoT, dLoT);
      lat_of(HF_T, gLaT, dLaT);
      lon_of(HF_V + 0, gLoE, dLoE);
      lat_of(HF_V + 0, gLaE, dLaE);
      lon_of(HF_V + 1, gLoN, dLoN);
      lat_of(HF_V + 1, gLaN, dLaN);
      lon_of(HF_V + 2, gLoU, dLoU);
      lat_of(HF_V + 2, gLaU, dLaU);
      // DivVel_C (:614-617)
      const double DivVel = gLaN + gLoE - TanLat * VN * InvR;
      // :688-694
      kv(HF_R) = (R - dt * (R * DivVel + gLaR * VN + gLoR * VE) + dt * (dLoR + dLaR)) - R;
      // :749-759, :765-777, :785-790 and the Coriolis terms of :803-813
      double nE = VE - dt * (VN * gLaE + VE * gLoE + VE * (VU - TanLat * VN) * InvR + gLoT + gLoR * T / R) +
                  dt * (dLoE + dLaE);
      double nN = VN - dt * (VN * gLaN + VE * gLoN + (VN * VU + TanLat * (VE * VE)) * InvR + gLaT + gLaR * T / R) +
                  dt * (dLoN + dLaN);
      const double nU = VU - dt * (VN * gLaU + VE * gLoU) + dt * (dLoU + dLaU);
      if (prm.use_coriolis) {
        nE = nE + dt * (+CoriolisSin * VN - CoriolisCos * VU);
        nN = nN - dt * (CentrifugalParameter * GC[4 * L.C + tid] + CoriolisSin * VE);
      }
      kv(HF_V + 0) = nE - VE;
      kv(HF_V + 1) = nN - VN;
      kv(HF_V + 2) = nU - VU;
      // :817-823
      kv(HF_T) = (T - dt * ((GC[2 * L.C + tid] - 1) * T * DivVel + gLaT * VN + gLoT * VE) + dt * (dLoT + dLaT)) - T;
      // species continuity (:696-703) and vertical winds (:794-801)
#pragma unroll 1
      for (int s = 0; s < NS; ++s) {
        double gLo, dLo, gLa, dLa;
        lon_of(HF_N + s, gLo, dLo);
        lat_of(HF_N + s, gLa, dLa);
        const double x = S[(HF_N + s) * P + pc];
        kv(HF_N + s) = (x - dt * (x * DivVel + gLa * VN + gLo * VE) + dt * (dLo + dLa)) - x;
        lon_of(HF_W + s, gLo, dLo);
        lat_of(HF_W + s, gLa, dLa);
        const double w = S[(HF_W + s) * P + pc];
        kv(HF_W + s) = (w - dt * (VN * gLa + VE * gLo) + dt * (dLa + dLo)) - w;
      }
      // advected ions (:719-736)
#pragma unroll 1
      for (int s = 0; s < NADV; ++s) {
        double gLo, dLo, gLa, dLa;
        lon_of(HF_I + s, gLo, dLo);
        lat_of(HF_I + s, gLa, dLa);
        const double x = S[(HF_I + s) * P + pc];
        kv(HF_I + s) =
            (x - dt * (+gLa * GC[6 * L.C + tid] + gLo * GC[5 * L.C + tid]) + dt * (dLo + dLa)) - x;
      }
    }
    __syncthreads();  // every read of this stage's state is done
    if (cell) {
#pragma unroll
      for (int f = 0; f < HZ_NSW; ++f) {
        const double o = src_of(f)[pc];
        const double kf = Kc[f * L.C + tid];
        double nx;
        if (st == 0) {
          acc[f] = kf;
          nx = 0.5 * kf + o;
        } else if (st == 1) {
          acc[f] = acc[f] + 2.0 * kf;
          nx = 0.5 * kf + o;
        } else if (st == 2) {
          acc[f] = acc[f] + 2.0 * kf;
          nx = kf + o;
        } else {
          acc[f] = acc[f] + kf;
          nx = o + (1.0 / 6.0) * acc[f];
        }
        S[f * P + pc] = nx;
      }
    }
    __syncthreads();
  }

  // ---------------------------------------------------------------- store
  auto out = [&](double* a, int f, int nf) { return a + ((int64_t(b) * nf + f) * NK + (k + 1)) * P + pc; };
  if (cell) {
    *out(B.rho, 0, 1) = S[HF_R * P + pc];
    for (int d = 0; d < 3; ++d) *out(B.velocity, d, 3) = S[(HF_V + d) * P + pc];
    const double Tn = S[HF_T * P + pc];
    if (B.temp_source)
      B.temp_source[((int64_t(b) * na + (k - 1)) * nt + (cj - 1)) * nl + (ci - 1)] = Tn - src_of(HF_T)[pc];
    *out(B.temperature, 0, 1) = Tn;
    bool neg = false;
    for (int s = 0; s < NS; ++s) {
      *out(B.vert_vel, s, NS) = S[(HF_W + s) * P + pc];
      const double nd = S[(HF_N + s) * P + pc];
      neg = neg || nd < 0.0;
      *out(B.ndensity_s, s, GITM_NSPECIES_TOTAL) = nd;
    }
    if (neg) atomicOr(&A.status[b], GITM_ST_NEG_DENSITY);  // the reference stops (:359-372)
    if (prm.use_ion_advection) {
      const bool div = prm.use_improved_ion_advection != 0;
      double change = 0.0;
      if (div) {
        // DivIVelocityLocal at the cell (:423-509): UAM_Gradient's component
        // iDir of IVelocityPar(iDir) plus the latitude and radial terms
        const double* VI = prm.non_magnetic ? B.ivelocity : B.ivelocity_par;
        auto vi = [&](int d, int i, int j, int kk) {
          return VI[((int64_t(b) * 3 + d) * NK + (kk + 1)) * P + int64_t(j + 1) * NI + (i + 1)];
        };
        const double InvR = GC[3 * L.C + tid];
        double D = 0.0;
        double g = 0.0;
        if (nl > 1) {
          const double InvCosLat = 1. / fmax(CosLat, 0.17);
          const int64_t o = int64_t(b) * nl + (ci - 1);
          g = (B.grad_lon_m[o] * vi(0, ci - 1, cj, k) + B.grad_lon_0[o] * vi(0, ci, cj, k) +
               B.grad_lon_p[o] * vi(0, ci + 1, cj, k)) * InvR * InvCosLat;
        }
        D = D + g;
        g = 0.0;
        if (nt > 1) {
          const int64_t o = int64_t(b) * nt + (cj - 1);
          g = (B.grad_lat_m[o] * vi(1, ci, cj - 1, k) + B.grad_lat_0[o] * vi(1, ci, cj, k) +
               B.grad_lat_p[o] * vi(1, ci, cj + 1, k)) * InvR;
        }
        D = D + g;
        double tl = TanLat;
        if (tl > 5.0) tl = 5.0;
        if (tl < -5.0) tl = -5.0;
        D = D - tl * vi(1, ci, cj, k) * InvR;
        g = 0.0;
        if (na > 1) {
          const double* Rg = B.radial_distance + int64_t(b) * V + int64_t(cj + 1) * NI + (ci + 1);
          const double Drp = Rg[(k + 2) * P] - Rg[(k + 1) * P];
          const double Drm = Rg[(k + 1) * P] - Rg[k * P];
          const double DrmOverDrp = Drm / Drp;
          const double Drr2 = DrmOverDrp * DrmOverDrp;
          const double Bottom = Drm * (1 + DrmOverDrp);
          g = (Drr2 * vi(2, ci, cj, k + 1) - vi(2, ci, cj, k - 1) - (Drr2 - 1) * vi(2, ci, cj, k)) / Bottom;
        }
        D = D + g;
        D = D + 2 * vi(2, ci, cj, k) * InvR;
        D = D * CosLat;
        change = dt * D;
      }
      double e = 0.0;
      for (int s = 0; s < NI_ALL; ++s) {
        double v;
        if (s < NADV) {
          v = S[(HF_I + s) * P + pc];
          if (v < 1.0e2) v = 1.0e2;  // :400-412
          if (div) v = v / (1 + change);
          *out(B.idensity_s, s, GITM_NIONS) = v;
        } else {
          v = *out(B.idensity_s, s, GITM_NIONS);
        }
        e = e + v;
      }
      *out(B.idensity_s, GITM_NIONS - 1, GITM_NIONS) = e;
    }
  }
  // with the divergence term the reference sums the electrons on every cell
  // (:512-515): this plane's ghost ring, and the ghost planes of the block
  if (prm.use_ion_advection && prm.use_improved_ion_advection) {
    auto esum = [&](int64_t off) {  // off: index of a cell in field 0's block array
      double e = 0.0;
      for (int s = 0; s < NI_ALL; ++s) e = e + B.idensity_s[off + int64_t(s) * V];
      B.idensity_s[off + int64_t(GITM_NIONS - 1) * V] = e;
    };
    const int64_t base = int64_t(b) * GITM_NIONS * V;
    for (int c = tid; c < P; c += NT) {
      const int i = c % NI - 1, j = c / NI - 1;
      if (i >= 1 && i <= nl && j >= 1 && j <= nt) continue;
      esum(base + (k + 1) * P + c);
    }
    if (k == 1)
      for (int64_t c = tid; c < 2 * P; c += NT) esum(base + c);  // altitudes -1, 0
    if (k == na)
      for (int64_t c = tid; c < 2 * P; c += NT) esum(base + (na + 2) * P + c);  // nAlts+1, nAlts+2
  }
}

// exchange_messages_sphere (exchange_messages_sphere.f90:4-95) for one
// (block, altitude) plane: the ghost ring takes the interior cells it
// covers (longitude periodic; across a connected pole the cell mirrored in
// latitude, n_blocks_lon / 2 blocks away -- the neighbours of
// AB_SPH_module.f90:180-370 and the packing of AB_XFER_array_util.f90),
// then the polar ghost rows' horizontal winds and ion velocities change sign
// (:35-76, on every altitude: the CTAs of the first and last altitude also
// take the ghost altitudes), then the checks of :78-88.
__global__ void __launch_bounds__(128) hz_exchange_kernel(const GitmHzExchange X, uint32_t* status) {
  const int nl = X.n_lons, nt = X.n_lats, na = X.n_alts;
  const int NI = nl + 4, NJ = nt + 4, NK = na + 4;
  const int64_t P = int64_t(NI) * NJ;
  const int k = blockIdx.x % na + 1;
  const int b = blockIdx.x / na;
  const int bx = b % X.n_blocks_lon, by = b / X.n_blocks_lon;
  const int64_t NLON = int64_t(nl) * X.n_blocks_lon, NLAT = int64_t(nt) * X.n_blocks_lat;
  const int64_t half = int64_t(X.n_blocks_lon / 2) * nl;
  double* VIw = X.non_magnetic ? X.ivelocity : X.ivelocity_par;
  auto at = [&](double* a, int blk, int f, int nf, int kk, int64_t c) -> double& {
    return a[((int64_t(blk) * nf + f) * NK + (kk + 1)) * P + c];
  };
  for (int c = threadIdx.x; c < P; c += blockDim.x) {
    const int i = c % NI - 1, j = c / NI - 1;  // Fortran (iLon, iLat)
    if (i >= 1 && i <= nl && j >= 1 && j <= nt) continue;
    int64_t G = int64_t(bx) * nl + i, GJ = int64_t(by) * nt + j;  // global 1-based
    if (GJ < 1) {
      if (!X.south_pole) continue;
      GJ = 1 - GJ;
      G += half;
    } else if (GJ > NLAT) {
      if (!X.north_pole) continue;
      GJ = 2 * NLAT + 1 - GJ;
      G += half;
    }
    G = ((G - 1) % NLON + NLON) % NLON + 1;
    const int sbx = int((G - 1) / nl), sby = int((GJ - 1) / nt);
    const int si = int(G - int64_t(sbx) * nl), sj = int(GJ - int64_t(sby) * nt);
    const int sb = sby * X.n_blocks_lon + sbx;
    const int64_t sc = int64_t(sj + 1) * NI + (si + 1);
    // the moved fields in pack_vars_nblk's order (ModSphereInterface.f90:
    // 395-447); every load is issued before the first store (source and
    // destination share arrays, so interleaved pairs would serialise)
    constexpr int NX = 1 + 3 + NS + NS + 3 + GITM_NIONS + 3;
    auto field = [&](int q, int& f, int& nf) -> double* {
      if (q == 0) { f = 0; nf = 1; return X.rho; }
      if (q < 4) { f = q - 1; nf = 3; return X.velocity; }
      if (q < 4 + NS) { f = q - 4; nf = NS; return X.vert_vel; }
      if (q < 4 + 2 * NS) { f = q - 4 - NS; nf = GITM_NSPECIES_TOTAL; return X.ndensity_s; }
      if (q == 4 + 2 * NS) { f = 0; nf = 1; return X.temperature; }
      if (q == 5 + 2 * NS) { f = 0; nf = 1; return X.itemperature; }
      if (q == 6 + 2 * NS) { f = 0; nf = 1; return X.etemperature; }
      if (q < 7 + 2 * NS + GITM_NIONS) { f = q - 7 - 2 * NS; nf = GITM_NIONS; return X.use_ion_advection ? X.idensity_s : nullptr; }
      f = q - 7 - 2 * NS - GITM_NIONS; nf = 3;
      return X.use_ion_advection ? VIw : nullptr;
    };
    double v[NX];
#pragma unroll
    for (int q = 0; q < NX; ++q) {
      int f, nf;
      double* a = field(q, f, nf);
      v[q] = a ? at(a, sb, f, nf, k, sc) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < NX; ++q) {
      int f, nf;
      double* a = field(q, f, nf);
      if (a) at(a, b, f, nf, k, c) = v[q];
    }
  }
  __syncthreads();
  // :35-76 -- Latitude(0) < -pi/2: rows -1:0; Latitude(nLats+1) > pi/2:
  // rows nLats+1:nLats+2; every longitude, every altitude
  const double lat0 = X.latitude[int64_t(b) * NJ + 1];
  const double latn = X.latitude[int64_t(b) * NJ + nt + 2];
  auto flip_plane = [&](int kk, int j0) {
    for (int c = threadIdx.x; c < 2 * NI; c += blockDim.x) {
      const int64_t cc = int64_t(j0 + 1 + c / NI) * NI + c % NI;
      for (int d = 0; d < 2; ++d) {
        at(X.velocity, b, d, 3, kk, cc) = -at(X.velocity, b, d, 3, kk, cc);
        at(VIw, b, d, 3, kk, cc) = -at(VIw, b, d, 3, kk, cc);
      }
    }
  };
  const double PI_ = 3.141592653589793;
  for (int side = 0; side < 2; ++side) {
    const bool polar = side == 0 ? (lat0 < -PI_ / 2.0) : (latn > PI_ / 2.0);
    if (!polar) continue;
    const int j0 = side == 0 ? -1 : nt + 1;
    flip_plane(k, j0);
    if (k == 1) {
      flip_plane(-1, j0);
      flip_plane(0, j0);
    }
    if (k == na) {
      flip_plane(na + 1, j0);
      flip_plane(na + 2, j0);
    }
  }
  // :78-88 on this altitude's interior
  uint32_t w = 0;
  for (int c = threadIdx.x; c < nl * nt; c += blockDim.x) {
    const int64_t cc = int64_t(c / nl + 2) * NI + (c % nl + 2);
    if (at(X.temperature, b, 0, 1, k, cc) < 100.0) w |= GITM_ST_LOW_TEMPERATURE;
    if (at(X.rho, b, 0, 1, k, cc) < 0.0) w |= GITM_ST_NEG_DENSITY;
  }
  if (w) atomicOr(&status[b], w);
}

}  // namespace

cudaError_t hz_exchange_launch(const GitmHzExchange& x, uint32_t* status, cudaStream_t stream) {
  hz_exchange_kernel<<<unsigned(int64_t(x.n_blocks_lon) * x.n_blocks_lat * x.n_alts), 128, 0, stream>>>(x, status);
  return cudaGetLastError();
}

size_t hz_smem_bytes(int n_lons, int n_lats) { return size_t(hz_layout(n_lons, n_lats).stride) * sizeof(double); }

int hz_threads(int n_lons, int n_lats) {
  const int c = n_lons * n_lats;
  return c <= 96 ? 96 : (c <= 128 ? 128 : (c <= 256 ? 256 : 0));
}

cudaError_t hz_launch(const GitmHzParams& prm, const GitmHzBlocks& b, double dt, uint32_t* status,
                      cudaStream_t stream) {
  HzArgs a;
  a.prm = prm;
  a.b = b;
  a.dt = dt;
  a.status = status;
  const int nt = hz_threads(b.n_lons, b.n_lats);
  const size_t smem = hz_smem_bytes(b.n_lons, b.n_lats);
  // 96 threads: 9 x 9 blocks (GITM's usual size) at 4 CTAs per SM
  const void* fn = (nt == 96) ? (const void*)hz_step_kernel<96, 4>
                 : (nt == 128) ? (const void*)hz_step_kernel<128, 3> : (const void*)hz_step_kernel<256, 1>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  if (e != cudaSuccess) return e;
  void* args[] = {&a};
  return cudaLaunchKernel(fn, dim3(unsigned(int64_t(b.n_blocks) * b.n_alts)), dim3(nt), args, smem, stream);
}

}  // namespace gv
