// oracle_capi.cpp -- extern "C" entry points of the CPU oracle (liboracle.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU legs of bench.py to check and time the CUDA library; never linked into
// it.  The per-column work follows advance_vertical (advance_vertical.f90:
// 45-219) around advance_vertical_1d_rusanov, with the coefficient producers
// of the GITM main loop (main.f90:56-73) in front when
// params.compute_coefficients is set, and calc_sources' eddy coefficient
// behind it when params.compute_eddy is set.  Columns are independent, so
// they are split over host threads.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "gitm_vert_oracle.hpp"
#include "oracle_ausm.hpp"
#include "oracle_hz.hpp"
#include "flop_counter.hpp"

using namespace gvo;

namespace {

inline int64_t nat(int f, int g, int64_t c, int G, int64_t n) { return (int64_t(f) * G + g) * n + c; }

inline double grid_at(const double* p, int g, int64_t c, const GitmColumnBatch& m) {
  return m.grid_per_column ? p[int64_t(g) * m.n_cols + c] : p[g];
}

// calc_eddy_diffusion_coefficient (Earth.f90:376-411) at one cell:
// EddyDiffusionCoef above EddyDiffusionPressure0, a linear taper down to
// EddyDiffusionPressure1, 0 below.
double eddy_coefficient(double pressure, const GitmVertParams& prm) {
  if (pressure > prm.eddy_pressure0) return prm.eddy_coef;
  if (pressure > prm.eddy_pressure1)
    return prm.eddy_coef * (pressure - prm.eddy_pressure1) / (prm.eddy_pressure0 - prm.eddy_pressure1);
  return 0.0;
}

template <class R>
void run_solver(Column<R>& col, const GitmVertParams& prm, double dt) {
  if (prm.solver == GITM_SOLVER_AUSM)
    advance_vertical_1d_ausm(col, prm, dt);
  else
    advance_vertical_1d_rusanov(col, prm, dt);
}

// One column of one member through n_steps steps (producers, gather, RK4,
// scatter per step).  Returns the status word.
uint32_t step_gitm_column(const GitmVertParams& prm, const GitmColumnBatch& m, int64_t c,
                          double dt, int n_steps) {
  const int nAlts = m.n_alts;
  const int G = nAlts + 4;
  const int64_t n = m.n_cols;
  const Planet& P = planet();
  uint32_t status = 0;
  Column<double> col;
  col.resize(nAlts);
  for (int g = 0; g < G; ++g) {
    col.Altitude[g] = grid_at(m.altitude, g, c, m);
    col.Gravity[g] = grid_at(m.gravity, g, c, m);
    col.dAlt_C[g] = grid_at(m.dalt_c, g, c, m);
    col.InvR[g] = grid_at(m.inv_r, g, c, m);
  }
  derive_faces(col);
  col.SZA = m.sza[c];
  col.MLat = m.mlat[c];
  // advance_vertical.f90:103-104
  const double cl = m.cos_lat[c];
  col.Centrifugal = (cl * prm.omega_body) * (cl * prm.omega_body);
  col.Coriolis = 2 * cl * prm.omega_body;
  col.has_lbc = (m.lbc != nullptr);
  if (m.lbc)
    for (int k = 0; k < 2; ++k)
      for (int v = 0; v < GITM_LBC_NVALUES; ++v) col.lbc[k][v] = m.lbc[nat(k, v, c, GITM_LBC_NVALUES, n)];

  std::vector<double> nden(nSpecies * G), ww(nSpecies * G), tt(G);
  for (int step = 0; step < n_steps; ++step) {
    // ---- producers (calc_pressure, calc_timestep_vertical, calc_rates)
    std::vector<double> gamma(G), mmm(G), tu(G), cmax(G, 0.0);
    for (int s = 0; s < nSpecies; ++s)
      for (int g = 0; g < G; ++g) {
        nden[s * G + g] = m.ndensity_s[nat(s, g, c, G, n)];
        ww[s * G + g] = m.vert_vel[nat(s, g, c, G, n)];
      }
    for (int g = 0; g < G; ++g) tt[g] = m.temperature[nat(0, g, c, G, n)];
    // Pressure = Temperature * Rho (calc_pressure.f90:23) of the state the
    // step starts from, for calc_sources' eddy coefficient after the step
    std::vector<double> pressure(G);
    for (int g = 0; g < G; ++g) pressure[g] = tt[g] * m.rho[nat(0, g, c, G, n)];
    if (prm.compute_coefficients) {
      Producers pr;
      produce_coefficients(nAlts, nden.data(), tt.data(), ww.data(), pr);
      gamma = pr.Gamma;
      mmm = pr.MeanMajorMass;
      tu = pr.TempUnit;
      cmax = pr.cMax;
      for (int g = 0; g < G; ++g) {
        if (m.gamma) m.gamma[nat(0, g, c, G, n)] = gamma[g];
        if (m.mean_major_mass) m.mean_major_mass[nat(0, g, c, G, n)] = mmm[g];
        if (m.temp_unit) m.temp_unit[nat(0, g, c, G, n)] = tu[g];
        if (m.cmax && g >= 1 && g <= nAlts + 2) m.cmax[nat(0, g, c, G, n)] = cmax[g];
      }
    } else {
      for (int g = 0; g < G; ++g) {
        gamma[g] = m.gamma[nat(0, g, c, G, n)];
        mmm[g] = m.mean_major_mass[nat(0, g, c, G, n)];
        tu[g] = m.temp_unit[nat(0, g, c, G, n)];
        cmax[g] = (g >= 1 && g <= nAlts + 2) ? m.cmax[nat(0, g, c, G, n)] : 0.0;
      }
    }

    // ---- gather, advance_vertical.f90:90-133
    double mn = nden[0];
    for (double v : nden) mn = std::min(mn, v);
    if (mn <= 0.0) return status | GITM_ST_NEG_DENSITY;  // :96-100
    for (int g = 0; g < G; ++g) {
      col.EddyCoef[g] = m.eddy[nat(0, g, c, G, n)];
      col.LogRho[g] = std::log(m.rho[nat(0, g, c, G, n)]);
      for (int d = 0; d < 3; ++d) col.Vel_GD[d * G + g] = m.velocity[nat(d, g, c, G, n)];
      col.Temp[g] = tt[g] * tu[g];
      for (int s = 0; s < nSpecies; ++s) {
        col.LogNS[s * G + g] = std::log(nden[s * G + g]);
        col.VertVel[s * G + g] = ww[s * G + g];
      }
      col.cMax[g] = cmax[g];
      col.IVel[0 * G + g] = 0.0;
      col.IVel[1 * G + g] = 0.0;
      col.IVel[2 * G + g] = m.ivel_up[nat(0, g, c, G, n)];
      for (int s = 0; s < nIons - 1; ++s) {
        double v = m.idensity_s[nat(s, g, c, G, n)];
        col.LogINS[s * G + g] = prm.use_improved_ion_advection ? v : std::log(v);
      }
      col.LogINS[(nIons - 1) * G + g] = 0.0;
      col.MeanMajorMass[g] = mmm[g];
      col.Gamma[g] = gamma[g];
    }

    col.status = 0;
    run_solver(col, prm, dt);
    status |= col.status;

    // ---- scatter, advance_vertical.f90:163-212
    bool finite = true;
    for (int g = 0; g < G; ++g) {
      double rho = std::exp(col.LogRho[g]);
      m.rho[nat(0, g, c, G, n)] = rho;
      for (int d = 0; d < 3; ++d) m.velocity[nat(d, g, c, G, n)] = col.Vel_GD[d * G + g];
      double T = col.Temp[g] / tu[g];
      // add_sources.f90:53-66 with EuvHeating its only nonzero term
      if (m.heating && g - 1 >= 1 && g - 1 <= nAlts)
        T = T + dt * ((m.heating_scale ? m.heating_scale[c] : 1.0) * m.heating[nat(0, g, c, G, n)]);
      m.temperature[nat(0, g, c, G, n)] = T;
      finite = finite && std::isfinite(rho) && std::isfinite(T);
      double N = 0.0;
      for (int s = 0; s < nSpecies; ++s) {
        if (m.log_ns) m.log_ns[nat(s, g, c, G, n)] = col.LogNS[s * G + g];
        m.vert_vel[nat(s, g, c, G, n)] = col.VertVel[s * G + g];
        double ns = std::exp(col.LogNS[s * G + g]);
        m.ndensity_s[nat(s, g, c, G, n)] = ns;
        N = N + ns;
        finite = finite && std::isfinite(ns) && std::isfinite(col.VertVel[s * G + g]);
      }
      if (m.ndensity) m.ndensity[nat(0, g, c, G, n)] = N;
      if (prm.use_ion_advection) {
        const int iAlt = g - 1;
        double e = 0.0;
        for (int s = 0; s < nIons - 1; ++s) {
          double v = prm.use_improved_ion_advection ? col.LogINS[s * G + g]
                                                    : std::exp(col.LogINS[s * G + g]);
          if (prm.use_improved_ion_advection && iAlt >= 1 && iAlt <= nAlts && v < 1) v = 1.0;
          m.idensity_s[nat(s, g, c, G, n)] = v;
          e = e + v;
          finite = finite && std::isfinite(v);
        }
        m.idensity_s[nat(nIons - 1, g, c, G, n)] = e;
      }
    }
    if (!finite) status |= GITM_ST_NONFINITE;
    // calc_sources.f90:26 after the vertical advance: the next step's
    // KappaEddyDiffusion (cells 1..nAlts, the ones the solver reads)
    if (prm.compute_eddy)
      for (int g = 2; g <= nAlts + 1; ++g) m.eddy[nat(0, g, c, G, n)] = eddy_coefficient(pressure[g], prm);
  }
  return status;
}

uint32_t step_1d_column(const GitmVertParams& prm, const GitmModVerticalBatch& b, int64_t c,
                        double dt) {
  const int nAlts = b.n_alts;
  const int G = nAlts + 4;
  const int64_t n = b.n_cols;
  Column<double> col;
  col.resize(nAlts);
  auto grid = [&](const double* p, int g) {
    return b.grid_per_column ? p[int64_t(g) * n + c] : p[g];
  };
  for (int g = 0; g < G; ++g) {
    col.Altitude[g] = grid(b.altitude, g);
    col.Gravity[g] = grid(b.gravity, g);
    col.dAlt_C[g] = grid(b.dalt_c, g);
    col.InvR[g] = grid(b.inv_r, g);
    col.LogRho[g] = b.log_rho[nat(0, g, c, G, n)];
    col.Temp[g] = b.temp[nat(0, g, c, G, n)];
    col.cMax[g] = b.cmax[nat(0, g, c, G, n)];
    col.MeanMajorMass[g] = b.mean_major_mass[nat(0, g, c, G, n)];
    col.Gamma[g] = b.gamma[nat(0, g, c, G, n)];
    col.EddyCoef[g] = b.eddy[nat(0, g, c, G, n)];
    for (int d = 0; d < 3; ++d) {
      col.Vel_GD[d * G + g] = b.vel_gd[nat(d, g, c, G, n)];
      col.IVel[d * G + g] = b.ivel[nat(d, g, c, G, n)];
    }
    for (int s = 0; s < nSpecies; ++s) {
      col.LogNS[s * G + g] = b.log_ns[nat(s, g, c, G, n)];
      col.VertVel[s * G + g] = b.vert_vel[nat(s, g, c, G, n)];
    }
    for (int s = 0; s < nIons; ++s) col.LogINS[s * G + g] = b.log_ins[nat(s, g, c, G, n)];
  }
  derive_faces(col);
  col.Centrifugal = b.centrifugal[c];
  col.Coriolis = b.coriolis[c];
  col.SZA = b.sza[c];
  col.MLat = b.mlat[c];
  col.has_lbc = (b.lbc != nullptr);
  if (b.lbc)
    for (int k = 0; k < 2; ++k)
      for (int v = 0; v < GITM_LBC_NVALUES; ++v) col.lbc[k][v] = b.lbc[nat(k, v, c, GITM_LBC_NVALUES, n)];
  col.status = 0;
  run_solver(col, prm, dt);
  for (int g = 0; g < G; ++g) {
    b.log_rho[nat(0, g, c, G, n)] = col.LogRho[g];
    b.temp[nat(0, g, c, G, n)] = col.Temp[g];
    for (int d = 0; d < 3; ++d) b.vel_gd[nat(d, g, c, G, n)] = col.Vel_GD[d * G + g];
    for (int s = 0; s < nSpecies; ++s) {
      b.log_ns[nat(s, g, c, G, n)] = col.LogNS[s * G + g];
      b.vert_vel[nat(s, g, c, G, n)] = col.VertVel[s * G + g];
    }
    for (int s = 0; s < nIons - 1; ++s) b.log_ins[nat(s, g, c, G, n)] = col.LogINS[s * G + g];
  }
  return col.status;
}

template <class F>
void parallel_for(int64_t n, int nthreads, F&& f) {
  if (nthreads <= 1 || n < 2) {
    for (int64_t i = 0; i < n; ++i) f(i);
    return;
  }
  nthreads = int(std::min<int64_t>(nthreads, n));
  std::atomic<int64_t> next{0};
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t)
    th.emplace_back([&] {
      for (;;) {
        int64_t i = next.fetch_add(16);
        if (i >= n) break;
        for (int64_t j = i; j < std::min(n, i + 16); ++j) f(j);
      }
    });
  for (auto& t : th) t.join();
}

}  // namespace

extern "C" {

// Advances every column of every member n_steps steps.  status: one word per
// column, members concatenated (may be NULL).  Returns the OR of all words.
uint32_t oracle_advance_native(const GitmVertParams* prm, const GitmColumnBatch* members,
                               int n_members, double dt, int n_steps, uint32_t* status,
                               int nthreads) {
  std::vector<int64_t> off(n_members + 1, 0);
  for (int k = 0; k < n_members; ++k) off[k + 1] = off[k] + members[k].n_cols;
  std::atomic<uint32_t> acc{0};
  parallel_for(off[n_members], nthreads, [&](int64_t i) {
    int k = int(std::upper_bound(off.begin(), off.end(), i) - off.begin()) - 1;
    uint32_t st = step_gitm_column(*prm, members[k], i - off[k], dt, n_steps);
    if (status) status[i] = st;
    acc.fetch_or(st);
  });
  return acc.load();
}

// One RK4 step of advance_vertical_1d_* on ModVertical-form columns.
uint32_t oracle_advance_1d(const GitmVertParams* prm, const GitmModVerticalBatch* b, double dt,
                           uint32_t* status, int nthreads) {
  std::atomic<uint32_t> acc{0};
  parallel_for(b->n_cols, nthreads, [&](int64_t c) {
    uint32_t st = step_1d_column(*prm, *b, c, dt);
    if (status) status[c] = st;
    acc.fetch_or(st);
  });
  return acc.load();
}

// advance_horizontal (advance_horizontal.f90:58-924) for every block; blocks
// are independent and split over host threads.  status: one word per block
// (may be NULL).  Returns the OR of all words.
uint32_t oracle_hz_advance(const GitmHzParams* prm, const GitmHzBlocks* b, double dt, uint32_t* status,
                           int nthreads) {
  std::atomic<uint32_t> acc{0};
  parallel_for(b->n_blocks, nthreads, [&](int64_t k) {
    const uint32_t st = gvo_hz::advance_horizontal_block(*prm, *b, int(k), dt);
    if (status) status[k] = st;
    acc.fetch_or(st);
  });
  return acc.load();
}

// calc_timestep_vertical (calc_timestep.f90:85-157) for one member: cMax for
// cells 0..nAlts+1 is written to cmax (native layout) and the local CFL time
// step min over columns is returned (the caller takes the min with Dt and
// DtEnd, as the reference does after the MPI_Allreduce).
double oracle_cfl_dt(const GitmVertParams* prm, const GitmColumnBatch* m, double cfl) {
  const int nAlts = m->n_alts, G = nAlts + 4;
  const int64_t n = m->n_cols;
  double dtl = 1.0e32;
  for (int64_t c = 0; c < n; ++c) {
    std::vector<double> cm(G, 0.0);
    for (int g = 1; g <= nAlts + 2; ++g) {
      double mx = std::fabs(m->vert_vel[nat(0, g, c, G, n)]);
      for (int s = 1; s < nSpecies; ++s) mx = std::max(mx, std::fabs(m->vert_vel[nat(s, g, c, G, n)]));
      cm[g] = mx + std::sqrt(m->gamma[nat(0, g, c, G, n)] * m->temperature[nat(0, g, c, G, n)]);
      if (m->cmax) m->cmax[nat(0, g, c, G, n)] = cm[g];
    }
    double mx = -1e300;
    for (int g = 2; g <= nAlts + 1; ++g)
      mx = std::max(mx, cm[g] / grid_at(m->dalt_c, g, c, *m));
    dtl = std::min(dtl, cfl / mx);
    if (prm->use_ion_advection) {
      double mi = -1e300;
      for (int g = 2; g <= nAlts + 1; ++g) {
        double v = std::fabs(m->ivel_up[nat(0, g, c, G, n)]) +
                   std::sqrt(m->gamma[nat(0, g, c, G, n)] * m->temperature[nat(0, g, c, G, n)]);
        mi = std::max(mi, v / grid_at(m->dalt_c, g, c, *m));
      }
      dtl = std::min(dtl, cfl / mi);
    }
  }
  return dtl;
}

// Operation counts of one column step of the given member column (solver per
// params): adds, muls, divs, sqrts, transcendentals (exp/log/pow/tanh/cos),
// compares.  Uses the instrumented scalar type.
void oracle_count_ops(const GitmVertParams* prm, const GitmModVerticalBatch* b, double dt,
                      double out[6]) {
  const int nAlts = b->n_alts, G = nAlts + 4;
  const int64_t n = b->n_cols, c = 0;
  Column<CD> col;
  col.resize(nAlts);
  auto grid = [&](const double* p, int g) { return b->grid_per_column ? p[int64_t(g) * n + c] : p[g]; };
  for (int g = 0; g < G; ++g) {
    col.Altitude[g] = grid(b->altitude, g);
    col.Gravity[g] = grid(b->gravity, g);
    col.dAlt_C[g] = grid(b->dalt_c, g);
    col.InvR[g] = grid(b->inv_r, g);
    col.LogRho[g] = b->log_rho[nat(0, g, c, G, n)];
    col.Temp[g] = b->temp[nat(0, g, c, G, n)];
    col.cMax[g] = b->cmax[nat(0, g, c, G, n)];
    col.MeanMajorMass[g] = b->mean_major_mass[nat(0, g, c, G, n)];
    col.Gamma[g] = b->gamma[nat(0, g, c, G, n)];
    col.EddyCoef[g] = b->eddy[nat(0, g, c, G, n)];
    for (int d = 0; d < 3; ++d) {
      col.Vel_GD[d * G + g] = b->vel_gd[nat(d, g, c, G, n)];
      col.IVel[d * G + g] = b->ivel[nat(d, g, c, G, n)];
    }
    for (int s = 0; s < nSpecies; ++s) {
      col.LogNS[s * G + g] = b->log_ns[nat(s, g, c, G, n)];
      col.VertVel[s * G + g] = b->vert_vel[nat(s, g, c, G, n)];
    }
    for (int s = 0; s < nIons; ++s) col.LogINS[s * G + g] = b->log_ins[nat(s, g, c, G, n)];
  }
  col.Centrifugal = b->centrifugal[c];
  col.Coriolis = b->coriolis[c];
  col.SZA = b->sza[c];
  col.MLat = b->mlat[c];
  CD::reset();
  derive_faces(col);
  run_solver(col, *prm, dt);
  out[0] = double(CD::n_add);
  out[1] = double(CD::n_mul);
  out[2] = double(CD::n_div);
  out[3] = double(CD::n_sqrt);
  out[4] = double(CD::n_trans);
  out[5] = double(CD::n_cmp);
}

}  // extern "C"

// ---------------------------------------------------------------- unit hooks
extern "C" {

double oracle_limiter_mc(double u, double d, double beta) { return Limiter_mc(u, d, beta); }

// ludcmp + lubksb on a 6x6 system; a row-major, b overwritten by x.
// Returns 0 for a singular matrix (ludcmp's stop), else 1.
int oracle_lu_solve(const double* a, double* b) {
  double m[7][7];
  double v[7];
  int indx[7];
  double d;
  for (int i = 1; i <= 6; ++i) {
    for (int j = 1; j <= 6; ++j) m[i][j] = a[(i - 1) * 6 + (j - 1)];
    v[i] = b[i - 1];
  }
  if (!ludcmp(m, 6, indx, d)) return 0;
  lubksb(m, 6, indx, v);
  for (int i = 1; i <= 6; ++i) b[i - 1] = v[i];
  return 1;
}

// Mesh coefficients of a column with altitudes alt[G]: out[0 .. 5*nAlts) the
// GradLogConS stencil of cells 1..nAlts, then 10 lower (cells 0, -1) and 10
// upper (nAlts+1, nAlts+2) extrapolation coefficients.
void oracle_mesh_coefs(int nAlts, const double* alt, double* out) {
  Column<double> c;
  c.resize(nAlts);
  for (int g = 0; g < nAlts + 4; ++g) c.Altitude[g] = alt[g];
  derive_faces(c);
  for (int i = 1; i <= nAlts; ++i) gradlogcons_coefs(c, i, out + 5 * (i - 1));
  double* bc = out + 5 * nAlts;
  lower_mesh_coefs(c, 0, bc);
  lower_mesh_coefs(c, -1, bc + 5);
  upper_mesh_coefs(c, nAlts + 1, bc + 10);
  upper_mesh_coefs(c, nAlts + 2, bc + 15);
}

// sizeof of the ABI structs as the C compiler lays them out.
void oracle_abi_sizes(int64_t out[9]) {
  out[0] = sizeof(GitmVertParams);
  out[1] = sizeof(GitmColumnBatch);
  out[2] = sizeof(GitmModVerticalBatch);
  out[3] = sizeof(GitmLaunchConfig);
  out[4] = sizeof(GitmFArray);
  out[5] = sizeof(GitmFortranState);
  out[6] = sizeof(GitmColumnAdjoint);
  out[7] = sizeof(GitmHzParams);
  out[8] = sizeof(GitmHzBlocks);
}

}  // extern "C"
