// gitm_vert.cu -- host side of libgitmvert: the C ABI of include/gitm_vert.h.
//
// The reference drives the path from Fortran modules (ModGITM, ModVertical,
// ModInputs); this file turns explicit arguments into device descriptors,
// precomputes the altitude-grid coefficients once per plan and launches the
// fused step kernel of vert_kernel.cuh.  No entry point falls back to the
// CPU: every compute call either launches a kernel or returns an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "vert_common.cuh"
#include "vert_kernel.cuh"
#include "vert_adjoint.cuh"
#include "vert_instances.h"
#include "vert_hz.cuh"

using namespace gv;

// ------------------------------------------------------------------ context
struct GitmVertCtx {
  int device = 0;
  int num_sms = 0;
  size_t max_smem = 0;
  GitmVertParams params;
  std::string err;
  // device staging for the host-pointer and Fortran-layout entry points,
  // grown on demand and reused across calls
  char* arena = nullptr;
  size_t arena_bytes = 0;
  double* d_scalar = nullptr;  // one double for reductions
  cudaStream_t streams[3] = {nullptr, nullptr, nullptr};
  // the host-pointer path keeps its plan while the calls' chunking, staging
  // arena and altitude grids stay the same
  GitmVertPlan* host_plan = nullptr;
  std::vector<uint64_t> host_plan_key;
  std::vector<cudaEvent_t> events;  // chunk hand-offs between the host path's streams
  // gitm_hz_advance: one status word per block, the stream of the last call
  uint32_t* hz_status = nullptr;
  int64_t hz_status_n = 0;
  int64_t hz_blocks = 0;
  cudaStream_t hz_stream = nullptr;
  // device address of the no-allocation entry point's file-scope scratch on
  // this context's device, looked up when the context is created
  double* noalloc_scratch = nullptr;
};

static int arena_reserve(GitmVertCtx* ctx, size_t bytes);
static cudaError_t noalloc_scratch_address(double** out);
struct GitmVertPlan;
static void plan_free(GitmVertPlan* P);

struct GitmVertPlan {
  GitmVertCtx* ctx = nullptr;
  std::vector<GitmColumnBatch> host_members;
  std::vector<DevMember> dev_members_host;
  DevMember* d_members = nullptr;
  double* d_grid = nullptr;
  uint32_t* d_status = nullptr;
  int64_t n_cols_total = 0;
  int n_members = 0;
  int io = 0;  // 0 GITM arrays, 1 ModVertical arrays
  int solver = GITM_SOLVER_RUSANOV;  // the context's solver when the plan was made
  GitmLaunchConfig cfg{256, 0, 1, 0};
  // tiles for the current cfg
  std::vector<Tile> tiles;
  Tile* d_tiles = nullptr;
  size_t smem = 0;
  int grid = 0;                 // CTAs per launch for the current cfg
  double* d_scratch = nullptr;  // RK accumulators (and Orig) of persistent CTAs
  size_t scratch_doubles = 0;
  int64_t scratch_per_cta = 0;  // doubles of one CTA's scratch slot
  int max_nalts = 0, min_nalts = 1 << 30;
  // adjoint launch (built on the first gitm_vert_plan_adjoint)
  bool adj_ready = false;
  std::vector<Tile> adj_tiles;
  Tile* d_adj_tiles = nullptr;
  size_t adj_smem = 0;
  int adj_grid = 0, adj_nc_max = 0, adj_per_max = 0;
  size_t adj_scratch_per_cta = 0;
  double* d_adj_scratch = nullptr;
  GitmColumnAdjoint* d_bars = nullptr;
  // the saving step kernel (its own tiles and persistent grid)
  std::vector<Tile> save_tiles;
  Tile* d_save_tiles = nullptr;
  int save_grid = 0;
  size_t save_smem = 0;
  double* d_save_scratch = nullptr;
};

static int set_err(GitmVertCtx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}

#define CUDA_TRY(ctx, call)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return set_err((ctx), GITM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

// ------------------------------------------------------------------ constants
static void fill_consts(Consts& k) {
  // ModConstants.f90:11,15; ModEarth.f90:237-281,307-312
  const double AMU = 1.6726e-27;
  const double mN = 14.0 * AMU, mO = 16.0 * AMU;
  const double mass[NS] = {mO, 2 * mO, 2 * mN, mN, mN + mO, 4.0 * AMU};
  const double vib[NS] = {5.0, 7.0, 7.0, 5.0, 7.0, 5.0};
  static const double d0[NS][NS] = {{0.000, 0.969, 0.969, 0.969, 0.715, 3.440},
                                    {0.969, 0.000, 0.715, 0.969, 0.715, 3.208},
                                    {0.969, 0.715, 0.000, 0.969, 0.527, 2.939},
                                    {0.969, 0.969, 0.969, 0.000, 0.969, 2.939},
                                    {0.715, 0.715, 0.527, 0.969, 0.000, 2.939},
                                    {3.440, 3.208, 2.939, 2.939, 2.939, 0.000}};
  // the six distinct DiffExp values; exp_index() in vert_kernel.cuh maps
  // each (i, j) of the DiffExp table to one of them
  const double distinct[NS] = {0.774, 0.750, 0.749, 0.710, 0.718, 0.810};
  for (int s = 0; s < NS; ++s) {
    k.mass[s] = mass[s];
    k.log_mass[s] = std::log(mass[s]);
    k.log_kb = std::log(KB);
    k.k_over_m[s] = KB / mass[s];
    k.inv_vib2[s] = 1.0 / (vib[s] - 2);
    k.one_minus_e[s] = 1.0 - distinct[s];
  }
  for (int i = 0; i < NS; ++i)
    for (int j = 0; j < NS; ++j) {
      k.kc[i][j] = 0.0;
      if (i == j) continue;
      // C_ij = (k T / M_i)(n_j / N) / (1e-4 D0_ij T^e / (N 1e-6))
      //      = 1e-2 k / (M_i D0_ij) * n_j * T^(1-e)   (calc_neutral_friction.f90:66-72)
      k.kc[i][j] = 1.0e-2 * KB / (mass[i] * (1.0e17 * d0[i][j]));
    }
}

// ------------------------------------------------------------------ grid
// Grid coefficients of one column, in the reference's operation order:
// dAlt_F / InvDAlt_F (advance_vertical.f90:149-151), the 5-point GradLogConS
// mesh (vertical_solver_rusanov.f90:515-533) and the one-sided boundary
// meshes (set_vertical_bcs.Earth.f90:279-297, 505-525).
static size_t grid_rows(int G) { return size_t(NGC) * G + NBC + size_t(NGA) * G; }

static void grid_coefs(int nA, const double* alt, const double* grav, const double* dalt_c,
                       const double* inv_r, double* out /* [grid_rows(G)] */) {
  const int G = nA + 4;
  std::vector<double> dAF(G), IDF(G);
  auto A = [&](int i) { return alt[i + 1]; };
  for (int i = 0; i <= nA + 2; ++i) dAF[i + 1] = A(i) - A(i - 1);
  dAF[0] = dAF[1];
  for (int g = 0; g < G; ++g) IDF[g] = 1.0 / dAF[g];
  auto F = [&](int i) { return dAF[i + 1]; };
  std::fill(out, out + grid_rows(G), 0.0);
  for (int g = 0; g < G; ++g) {
    out[GC_DALTF * G + g] = dAF[g];
    out[GC_H2 * G + g] = IDF[g] * 2.0;
    out[GC_IDF * G + g] = IDF[g];
    out[GC_IDC * G + g] = 1.0 / dalt_c[g];
    out[GC_GRAV * G + g] = grav[g];
    out[GC_INVR * G + g] = inv_r[g];
    out[GC_R * G + g] = 1.0 / inv_r[g];
    out[GC_ALT * G + g] = alt[g];
  }
  for (int i = 1; i <= nA; ++i) {
    const double h1 = F(i - 1), h2 = F(i), h3 = F(i + 1), h4 = F(i + 2);
    const double H2 = h2 + h1, H3 = h3 + h2 + h1, H4 = h4 + h3 + h2 + h1;
    const double c0 = (h2 * h3 * (h3 + h4)) / (h1 * H2 * H3 * H4);
    const double c1 = -1.0 * (H2 * h3 * (h3 + h4)) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
    const double c3 = H2 * h2 * (h4 + h3) / (H3 * (h2 + h3) * h3 * h4);
    const double c4 = -1.0 * H2 * h2 * h3 / (H4 * (h2 + h3 + h4) * (h3 + h4) * h4);
    const double c2 = (h2 * h3 * (h3 + h4) + H2 * h3 * (h3 + h4) - H2 * h2 * (h3 + h4) - H2 * h2 * h3) /
                      (H2 * h2 * h3 * (h3 + h4));
    const double cs[5] = {c0, c1, c2, c3, c4};
    for (int k = 0; k < 5; ++k) out[(GC_M0 + k) * G + i + 1] = cs[k];
  }
  double* bc = out + NGC * G;
  for (int k = 0; k < 2; ++k) {  // lower: cells 0, -1
    const int iAlt = -k;
    const double h1 = F(iAlt + 2), h2 = F(iAlt + 3), h3 = F(iAlt + 4), h4 = F(iAlt + 5);
    const double M1 = h1, M2 = h1 + h2, M3 = h1 + h2 + h3, M4 = h1 + h2 + h3 + h4;
    bc[5 * k + 0] = -1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4);
    bc[5 * k + 1] = 1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
    bc[5 * k + 2] = -1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4));
    bc[5 * k + 3] = 1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4);
    bc[5 * k + 4] = -1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4);
  }
  for (int k = 0; k < 2; ++k) {  // upper: cells nA+1, nA+2
    const int iAlt = nA + 1 + k;
    const double h1 = F(iAlt - 1), h2 = F(iAlt - 2), h3 = F(iAlt - 3), h4 = F(iAlt - 4);
    const double M1 = h1, M2 = h1 + h2, M3 = h1 + h2 + h3, M4 = h1 + h2 + h3 + h4;
    bc[10 + 5 * k + 0] = 1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4);
    bc[10 + 5 * k + 1] = -1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
    bc[10 + 5 * k + 2] = 1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4));
    bc[10 + 5 * k + 3] = -1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4);
    bc[10 + 5 * k + 4] = 1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4);
  }
  // AUSM cell constants: the Kp / Ku altitude profiles
  // (vertical_solver_ausm.f90:1314-1352), the spherical face areas and cell
  // volume (:2029-2039) and the wind-diffusion factor (:944-946)
  double* ga = out + NGC * G + NBC;
  const double LogMaxKu = std::log(0.50), LogMinKu = std::log(0.25);
  const double LogMaxKp = std::log(1.0e-09), LogMinKp = std::log(1.0e-19);
  const double KpWidth = 15.0e+03, KpAltMidPoint = 160.0e+03;
  auto R = [&](int i) { return 1.0 / inv_r[i + 1]; };
  for (int g = 0; g < G; ++g) ga[GA_DALTC * G + g] = dalt_c[g];
  for (int i = 1; i <= nA; ++i) {
    const double LeftRadius = 0.5 * (R(i) + R(i - 1));
    const double RightRadius = 0.5 * (R(i) + R(i + 1));
    ga[GA_AP * G + i + 1] = RightRadius * RightRadius;
    ga[GA_AM * G + i + 1] = LeftRadius * LeftRadius;
    ga[GA_VOL * G + i + 1] = (1.0 / 3.0) * (std::pow(RightRadius, 3.0) - std::pow(LeftRadius, 3.0));
    const double th = std::tanh((A(i) - KpAltMidPoint) / KpWidth);
    ga[GA_KP * G + i + 1] = std::exp(LogMinKp + 0.5 * (LogMaxKp - LogMinKp) * (1.0 + th));
    ga[GA_KU * G + i + 1] = std::exp(LogMinKu + 0.5 * (LogMaxKu - LogMinKu) * (1.0 + th));
    ga[GA_DAMP * G + i + 1] = 0.35 * std::exp(-1.0 * (A(i) - A(0)) / (45.0e+03));
  }
}

// ------------------------------------------------------------------ kernels
// Launch shapes built: threads per CTA -> CTAs per SM the registers allow and
// where the RK accumulator lives.  The small CTAs keep it in a per-CTA slot
// of global scratch (L2-resident under their persistent grid) so that two or
// three CTAs share an SM and overlap each other's barrier phases.
// The 512-thread shape also keeps Orig in its scratch slot (orig_global):
// 8 columns of 50 altitudes then fit the shared memory of an SM, 16 warps at
// 128 registers.  The AUSM solver's 384-thread shape does the same (6
// columns of its larger slot instead of 4).  solver -1: any solver.
struct Shape { int threads, solver, min_blocks; bool acc_global, orig_global; };
static const Shape kShapes[] = {{128, -1, 3, true, false}, {160, -1, 2, true, false}, {192, -1, 2, true, false},
                                {256, -1, 1, false, false}, {320, -1, 1, false, false},
                                {384, GITM_SOLVER_AUSM, 1, true, true}, {384, -1, 1, false, false},
                                {512, -1, 1, true, true}};
static const int kThreadChoices[] = {128, 160, 192, 256, 320, 384, 512};

static const Shape* shape_of(int threads, int solver) {
  for (const Shape& s : kShapes)
    if (s.threads == threads && (s.solver == solver || s.solver < 0)) return &s;
  return nullptr;
}

static bool acc_global(int threads, int solver) {
  const Shape* s = shape_of(threads, solver);
  return s && s->acc_global;
}

static bool orig_global(int threads, int solver) {
  const Shape* s = shape_of(threads, solver);
  return s && s->orig_global;
}

// The step kernels, each compiled in its own translation unit
// (vert_instance.cu, one per GV_STEP_INSTANCES entry).
struct StepInstance {
  int io, threads, solver;
  bool save;
  int na;  // 0: any nAlts; > 0: members of exactly this nAlts
  const void* (*fn)();
  cudaError_t (*consts)(const Consts&);
};
static const StepInstance kInstances[] = {
#define GV_TABLE_ENTRY(id, IO, NT, MINB, ACC, SOLVER, SAVE, NA, OG) \
  {IO, NT, SOLVER, SAVE, NA, step_kernel_##id, step_consts_##id},
    GV_STEP_INSTANCES(GV_TABLE_ENTRY)
#undef GV_TABLE_ENTRY
};

// The step kernel for an array form (0 GITM arrays, 1 ModVertical), solver
// and CTA size, or nullptr when that shape is not built.  nalts > 0 (every
// member has that nAlts) prefers the instance compiled for it.
static const void* kernel_for(int io, int solver, int threads, int nalts = 0, bool save = false) {
  const StepInstance* any = nullptr;
  for (const StepInstance& k : kInstances) {
    if (k.save != save || k.io != io || k.solver != solver || k.threads != threads) continue;
    if (nalts > 0 && k.na == nalts) return k.fn();
    if (k.na == 0 && !any) any = &k;
  }
  return any ? any->fn() : nullptr;
}

// The nAlts every member of a plan shares, or 0 when they differ.
static int plan_nalts(const GitmVertPlan* P) {
  if (P->host_members.empty()) return 0;
  const int na = P->host_members[0].n_alts;
  for (const GitmColumnBatch& b : P->host_members)
    if (b.n_alts != na) return 0;
  return na;
}

// ------------------------------------------------------------------ API
extern "C" {

const char* gitm_vert_version(void) { return "gitm_b200 0.1.0 (sm_100a, FP64)"; }

void gitm_vert_default_params(GitmVertParams* p) {
  if (!p) return;
  std::memset(p, 0, sizeof *p);
  p->solver = GITM_SOLVER_RUSANOV;
  p->use_neutral_friction = 1;
  p->use_coriolis = 1;
  p->use_ion_advection = 1;
  p->use_improved_ion_advection = 1;
  p->use_nighttime_ion_bcs = 1;
  p->use_damping = 0;
  p->use_msis_bcs = 0;
  p->compute_coefficients = 1;
  p->beta_limiter = 2.0;
  p->max_vertical_velocity = 1000.0;
  p->min_tec = 2.0;
  p->omega_body = 2.0 * 3.141592653589793 / (24.0 * 3600.0);
  p->vert_tau = 1.0e9;
  p->thermal_diff_coef[5] = -0.38;
  p->compute_eddy = 0;
  p->eddy_coef = 50.0;
  p->eddy_pressure0 = 0.01;
  p->eddy_pressure1 = 0.005;
}

static int check_params(GitmVertCtx* ctx, const GitmVertParams* p) {
  if (!p) return set_err(ctx, GITM_ERR_ARG, "params is NULL");
  if (p->solver != GITM_SOLVER_RUSANOV && p->solver != GITM_SOLVER_AUSM)
    return set_err(ctx, GITM_ERR_ARG, "unknown solver %d", p->solver);
  if (!(p->beta_limiter >= 1.0 && p->beta_limiter <= 2.0))
    return set_err(ctx, GITM_ERR_ARG, "beta_limiter %g outside [1, 2]", p->beta_limiter);
  if (p->compute_eddy && !(p->eddy_pressure0 > p->eddy_pressure1))
    return set_err(ctx, GITM_ERR_ARG, "compute_eddy needs eddy_pressure0 > eddy_pressure1");
  return GITM_OK;
}

int gitm_vert_create(const GitmVertParams* params, int device, GitmVertCtx** out) {
  if (!out) return GITM_ERR_ARG;
  *out = nullptr;
  GitmVertCtx* ctx = new GitmVertCtx();
  if (params) {
    int rc = check_params(ctx, params);
    if (rc) { delete ctx; return rc; }
    ctx->params = *params;
  } else {
    gitm_vert_default_params(&ctx->params);
  }
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0 || device < 0 || device >= ndev) {
    delete ctx;
    return GITM_ERR_CUDA;
  }
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return GITM_ERR_CUDA; }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) { delete ctx; return GITM_ERR_CUDA; }
  ctx->num_sms = prop.multiProcessorCount;
  ctx->max_smem = prop.sharedMemPerBlockOptin;
  Consts k;
  fill_consts(k);
  if (cudaMemcpyToSymbol(c_k, &k, sizeof k) != cudaSuccess) { delete ctx; return GITM_ERR_CUDA; }
  if (adjoint_set_consts(k) != cudaSuccess || adjoint_set_consts_n50(k) != cudaSuccess) {
    delete ctx;
    return GITM_ERR_CUDA;
  }
  for (const StepInstance& si : kInstances)
    if (si.consts(k) != cudaSuccess) { delete ctx; return GITM_ERR_CUDA; }
  // the scratch of gitm_vert_advance_native_noalloc on this device (a host-side
  // name of a __device__ array is not its device address)
  if (noalloc_scratch_address(&ctx->noalloc_scratch) != cudaSuccess || !ctx->noalloc_scratch) {
    delete ctx;
    return GITM_ERR_CUDA;
  }
  for (const StepInstance& si : kInstances)
    cudaFuncSetAttribute(si.fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, int(ctx->max_smem));
  *out = ctx;
  return GITM_OK;
}

int gitm_vert_destroy(GitmVertCtx* ctx) {
  if (!ctx) return GITM_OK;
  cudaSetDevice(ctx->device);
  plan_free(ctx->host_plan);
  for (cudaEvent_t e : ctx->events) cudaEventDestroy(e);
  cudaFree(ctx->arena);
  cudaFree(ctx->d_scalar);
  cudaFree(ctx->hz_status);
  for (cudaStream_t& st : ctx->streams)
    if (st) cudaStreamDestroy(st);
  delete ctx;
  return GITM_OK;
}

const char* gitm_vert_last_error(const GitmVertCtx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int gitm_vert_set_params(GitmVertCtx* ctx, const GitmVertParams* params) {
  if (!ctx) return GITM_ERR_ARG;
  int rc = check_params(ctx, params);
  if (rc) return rc;
  ctx->params = *params;
  return GITM_OK;
}

}  // extern "C"

// Columns per CTA for a member of nAlts under cfg.
static int cols_per_cta(const GitmVertCtx* ctx, const GitmLaunchConfig& cfg, int nA, int solver) {
  int nc = cfg.cols_per_cta > 0 ? cfg.cols_per_cta : cfg.threads / nA;
  nc = std::min(nc, cfg.threads / 32);  // one BC warp per column
  nc = std::min(nc, cfg.threads / nA);  // every interior cell has a thread
  while (nc > 1 && smem_bytes(nA, nc, solver, orig_global(cfg.threads, solver)) > ctx->max_smem) --nc;
  return std::max(nc, 1);
}

static int build_tiles(GitmVertPlan* P) {
  GitmVertCtx* ctx = P->ctx;
  if (!kernel_for(P->io, P->solver, P->cfg.threads, plan_nalts(P)))
    return set_err(ctx, GITM_ERR_ARG, "threads per CTA %d not built for solver %d", P->cfg.threads, P->solver);
  P->tiles.clear();
  P->smem = 0;
  const bool og = orig_global(P->cfg.threads, P->solver);
  size_t orig_per_cta = 0;  // doubles of Orig a CTA's scratch slot holds (orig_global shapes)
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnBatch& b = P->host_members[m];
    const int nc = cols_per_cta(ctx, P->cfg, b.n_alts, P->solver);
    if (nc * b.n_alts > P->cfg.threads || smem_bytes(b.n_alts, nc, P->solver, og) > ctx->max_smem)
      return set_err(ctx, GITM_ERR_ARG, "nAlts %d does not fit a CTA of %d threads", b.n_alts,
                     P->cfg.threads);
    P->smem = std::max(P->smem, smem_bytes(b.n_alts, nc, P->solver, og));
    if (og) orig_per_cta = std::max(orig_per_cta, size_t(nc) * orig_doubles(b.n_alts));
    for (int64_t c0 = 0; c0 < b.n_cols; c0 += nc) {
      Tile t;
      t.member = m;
      t.nc = int(std::min<int64_t>(nc, b.n_cols - c0));
      t.c0 = c0;
      P->tiles.push_back(t);
    }
  }
  if (P->d_tiles) cudaFree(P->d_tiles);
  P->d_tiles = nullptr;
  if (!P->tiles.empty()) {
    CUDA_TRY(ctx, cudaMalloc(&P->d_tiles, P->tiles.size() * sizeof(Tile)));
    CUDA_TRY(ctx, cudaMemcpy(P->d_tiles, P->tiles.data(), P->tiles.size() * sizeof(Tile),
                             cudaMemcpyHostToDevice));
  }
  // grid: one CTA per tile, or a persistent grid of ctas_per_sm x SMs; shapes
  // that keep the accumulator in scratch always run persistent (one slot per CTA)
  const int T = P->cfg.threads;
  int grid = int(P->tiles.size());
  int per_sm = P->cfg.ctas_per_sm;
  if (acc_global(T, P->solver) && per_sm <= 0) {
    const void* fn = kernel_for(P->io, P->solver, T, plan_nalts(P));
    CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, P->smem));
    per_sm = std::max(per_sm, 1);
  }
  if (per_sm > 0) grid = std::min(grid, per_sm * ctx->num_sms);
  P->grid = std::max(grid, 1);
  P->scratch_per_cta = int64_t(NF) * T + int64_t(orig_per_cta);
  if (acc_global(T, P->solver)) {
    // at least three slots: the host-pointer path splits them over 3 streams
    const size_t need = size_t(std::max(P->grid, 3)) * size_t(P->scratch_per_cta);
    if (need > P->scratch_doubles) {
      cudaFree(P->d_scratch);
      P->d_scratch = nullptr;
      P->scratch_doubles = 0;
      if (cudaMalloc(&P->d_scratch, need * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(ctx, GITM_ERR_NOMEM, "cannot allocate %zu bytes of step scratch", need * sizeof(double));
      }
      P->scratch_doubles = need;
    }
  }
  return GITM_OK;
}

static bool is_device_ptr(const void* p) {
  if (!p) return true;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Shared by both plan kinds: grid coefficients + device member table.
static int plan_common(GitmVertPlan* P, const double* const* alt, const double* const* grav,
                       const double* const* dalt, const double* const* invr, const int* gpc) {
  GitmVertCtx* ctx = P->ctx;
  // grid coefficients: copy each member's grid to the host, compute, upload
  std::vector<size_t> goff(P->n_members);
  size_t gtotal = 0;
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnBatch& b = P->host_members[m];
    const int G = b.n_alts + 4;
    const int64_t gcols = gpc[m] ? b.n_cols : 1;
    goff[m] = gtotal;
    gtotal += grid_rows(G) * gcols;
  }
  CUDA_TRY(ctx, cudaMalloc(&P->d_grid, gtotal * sizeof(double)));
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnBatch& b = P->host_members[m];
    const int nA = b.n_alts, G = nA + 4;
    const int64_t gcols = gpc[m] ? b.n_cols : 1;
    const size_t per = size_t(G) * gcols;
    std::vector<double> ha(per), hg(per), hd(per), hi(per);
    CUDA_TRY(ctx, cudaMemcpy(ha.data(), alt[m], per * sizeof(double), cudaMemcpyDefault));
    CUDA_TRY(ctx, cudaMemcpy(hg.data(), grav[m], per * sizeof(double), cudaMemcpyDefault));
    CUDA_TRY(ctx, cudaMemcpy(hd.data(), dalt[m], per * sizeof(double), cudaMemcpyDefault));
    CUDA_TRY(ctx, cudaMemcpy(hi.data(), invr[m], per * sizeof(double), cudaMemcpyDefault));
    std::vector<double> colv(grid_rows(G)), out(grid_rows(G) * gcols);
    std::vector<double> a1(G), g1(G), d1(G), i1(G);
    for (int64_t gc = 0; gc < gcols; ++gc) {
      for (int g = 0; g < G; ++g) {
        a1[g] = ha[g * gcols + gc];
        g1[g] = hg[g * gcols + gc];
        d1[g] = hd[g * gcols + gc];
        i1[g] = hi[g * gcols + gc];
      }
      grid_coefs(nA, a1.data(), g1.data(), d1.data(), i1.data(), colv.data());
      for (size_t r = 0; r < grid_rows(G); ++r) out[r * gcols + gc] = colv[r];
    }
    CUDA_TRY(ctx, cudaMemcpy(P->d_grid + goff[m], out.data(), out.size() * sizeof(double),
                             cudaMemcpyHostToDevice));
    P->dev_members_host[m].gridc = P->d_grid + goff[m];
    P->dev_members_host[m].gcols = int32_t(gcols);
  }
  CUDA_TRY(ctx, cudaMalloc(&P->d_members, P->n_members * sizeof(DevMember)));
  CUDA_TRY(ctx, cudaMemcpy(P->d_members, P->dev_members_host.data(), P->n_members * sizeof(DevMember),
                           cudaMemcpyHostToDevice));
  CUDA_TRY(ctx, cudaMalloc(&P->d_status, std::max<int64_t>(P->n_cols_total, 1) * sizeof(uint32_t)));
  CUDA_TRY(ctx, cudaMemset(P->d_status, 0, std::max<int64_t>(P->n_cols_total, 1) * sizeof(uint32_t)));
  // default launch shape: 256 threads (no register spills), as many columns as fit
  P->cfg.threads = 256;
  P->cfg.cols_per_cta = 0;
  P->cfg.steps_per_launch = 1;
  P->cfg.ctas_per_sm = 0;
  return build_tiles(P);
}

static void plan_free(GitmVertPlan* P) {
  if (!P) return;
  cudaFree(P->d_adj_tiles);
  cudaFree(P->d_save_tiles);
  cudaFree(P->d_adj_scratch);
  cudaFree(P->d_save_scratch);
  cudaFree(P->d_bars);
  cudaFree(P->d_scratch);
  cudaFree(P->d_members);
  cudaFree(P->d_grid);
  cudaFree(P->d_status);
  cudaFree(P->d_tiles);
  delete P;
}

static int check_member(GitmVertCtx* ctx, const GitmColumnBatch& b, const GitmVertParams& prm) {
  if (b.n_alts < 8 || b.n_alts > GITM_MAX_NALTS)
    return set_err(ctx, GITM_ERR_ARG, "n_alts %d outside [8, %d]", b.n_alts, GITM_MAX_NALTS);
  if (b.n_cols < 0) return set_err(ctx, GITM_ERR_ARG, "n_cols < 0");
  if (b.n_cols == 0) return GITM_OK;
  const void* req[] = {b.ndensity_s, b.idensity_s, b.rho, b.temperature, b.velocity, b.vert_vel,
                       b.ivel_up, b.eddy, b.cos_lat, b.sza, b.mlat, b.altitude, b.gravity,
                       b.dalt_c, b.inv_r};
  for (const void* p : req)
    if (!p) return set_err(ctx, GITM_ERR_ARG, "a required GitmColumnBatch pointer is NULL");
  if (!prm.compute_coefficients && (!b.gamma || !b.mean_major_mass || !b.temp_unit || !b.cmax))
    return set_err(ctx, GITM_ERR_ARG, "compute_coefficients=0 needs gamma, mean_major_mass, temp_unit, cmax");
  if (prm.use_msis_bcs && !b.lbc)
    return set_err(ctx, GITM_ERR_ARG, "use_msis_bcs=1 needs the lbc table");
  return GITM_OK;
}

extern "C" {

int gitm_vert_plan_create(GitmVertCtx* ctx, const GitmColumnBatch* members, int n_members,
                          GitmVertPlan** out) {
  if (!ctx || !out || (n_members > 0 && !members) || n_members < 0)
    return set_err(ctx, GITM_ERR_ARG, "bad plan arguments");
  *out = nullptr;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  GitmVertPlan* P = new GitmVertPlan();
  P->ctx = ctx;
  P->io = 0;
  P->solver = ctx->params.solver;
  P->n_members = n_members;
  P->host_members.assign(members, members + n_members);
  P->dev_members_host.resize(n_members);
  std::vector<const double*> alt(n_members), grav(n_members), dalt(n_members), invr(n_members);
  std::vector<int> gpc(n_members);
  for (int m = 0; m < n_members; ++m) {
    int rc = check_member(ctx, members[m], ctx->params);
    if (rc) { plan_free(P); return rc; }
    const void* ptrs[] = {members[m].ndensity_s, members[m].idensity_s, members[m].rho,
                          members[m].temperature, members[m].velocity, members[m].vert_vel,
                          members[m].ivel_up, members[m].eddy};
    for (const void* p : ptrs)
      if (!is_device_ptr(p)) { plan_free(P); return set_err(ctx, GITM_ERR_ARG, "plan arrays must be device pointers"); }
    DevMember& d = P->dev_members_host[m];
    std::memset(&d, 0, sizeof d);
    d.b = members[m];
    d.col_offset = P->n_cols_total;
    P->n_cols_total += members[m].n_cols;
    P->max_nalts = std::max(P->max_nalts, members[m].n_alts);
    P->min_nalts = std::min(P->min_nalts, members[m].n_alts);
    alt[m] = members[m].altitude;
    grav[m] = members[m].gravity;
    dalt[m] = members[m].dalt_c;
    invr[m] = members[m].inv_r;
    gpc[m] = members[m].grid_per_column;
  }
  int rc = plan_common(P, alt.data(), grav.data(), dalt.data(), invr.data(), gpc.data());
  if (rc) { plan_free(P); return rc; }
  *out = P;
  return GITM_OK;
}

int gitm_vert_plan_destroy(GitmVertPlan* plan) {
  plan_free(plan);
  return GITM_OK;
}

int gitm_vert_plan_set_config(GitmVertPlan* P, const GitmLaunchConfig* cfg) {
  if (!P || !cfg) return GITM_ERR_ARG;
  GitmLaunchConfig old = P->cfg;
  P->cfg = *cfg;
  if (P->cfg.steps_per_launch < 1) P->cfg.steps_per_launch = 1;
  if (P->cfg.ctas_per_sm < 0) P->cfg.ctas_per_sm = 0;
  int rc = build_tiles(P);
  if (rc) {
    P->cfg = old;
    build_tiles(P);
  }
  return rc;
}

int gitm_vert_plan_get_config(const GitmVertPlan* P, GitmLaunchConfig* cfg) {
  if (!P || !cfg) return GITM_ERR_ARG;
  *cfg = P->cfg;
  return GITM_OK;
}

int gitm_vert_plan_launch_count(const GitmVertPlan* P, int n_steps) {
  if (!P || n_steps <= 0 || P->tiles.empty()) return 0;
  const int spl = std::max(1, P->cfg.steps_per_launch);
  return (n_steps + spl - 1) / spl;
}

static int launch_steps(GitmVertPlan* P, double dt, int n_steps, cudaStream_t stream) {
  GitmVertCtx* ctx = P->ctx;
  if (P->tiles.empty() || n_steps <= 0) return GITM_OK;
  const int spl = std::max(1, P->cfg.steps_per_launch);
  if (ctx->params.solver != P->solver)
    return set_err(ctx, GITM_ERR_ARG, "plan was built for solver %d, context now selects %d", P->solver,
                   ctx->params.solver);
  const void* fn = kernel_for(P->io, P->solver, P->cfg.threads, plan_nalts(P));
  if (!fn) return set_err(ctx, GITM_ERR_ARG, "no kernel for %d threads", P->cfg.threads);
  const int grid = P->grid;
  KParams kp{};
  kp.members = P->d_members;
  kp.tiles = P->d_tiles;
  kp.n_tiles = int(P->tiles.size());
  kp.dt = dt;
  kp.status = P->d_status;
  kp.scratch = P->d_scratch;
  kp.scratch_per_cta = P->scratch_per_cta;
  kp.prm = ctx->params;
  for (int done = 0; done < n_steps; done += spl) {
    kp.n_steps = std::min(spl, n_steps - done);
    void* args[] = {&kp};
    CUDA_TRY(ctx, cudaLaunchKernel(fn, dim3(grid), dim3(P->cfg.threads), args, P->smem, stream));
  }
  return GITM_OK;
}

int gitm_vert_plan_advance(GitmVertPlan* P, double dt, int n_steps, void* stream) {
  if (!P) return GITM_ERR_ARG;
  if (n_steps < 0) return set_err(P->ctx, GITM_ERR_ARG, "n_steps < 0");
  if (P->io == 1 && n_steps > 1)
    return set_err(P->ctx, GITM_ERR_ARG, "ModVertical batches advance one step per call");
  if (!(dt > 0.0)) return set_err(P->ctx, GITM_ERR_ARG, "dt must be > 0");
  CUDA_TRY(P->ctx, cudaSetDevice(P->ctx->device));
  return launch_steps(P, dt, n_steps, (cudaStream_t)stream);
}

int gitm_vert_plan_status(GitmVertPlan* P, uint32_t* status_or, int64_t* n_bad, int clear) {
  if (!P) return GITM_ERR_ARG;
  GitmVertCtx* ctx = P->ctx;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  std::vector<uint32_t> h(std::max<int64_t>(P->n_cols_total, 1));
  CUDA_TRY(ctx, cudaMemcpy(h.data(), P->d_status, h.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  uint32_t acc = 0;
  int64_t bad = 0;
  for (int64_t i = 0; i < P->n_cols_total; ++i) {
    acc |= h[i];
    bad += h[i] != 0;
  }
  if (status_or) *status_or = acc;
  if (n_bad) *n_bad = bad;
  if (clear) CUDA_TRY(ctx, cudaMemset(P->d_status, 0, h.size() * sizeof(uint32_t)));
  return GITM_OK;
}

uint32_t* gitm_vert_plan_status_words(GitmVertPlan* P) { return P ? P->d_status : nullptr; }

// Host watchdog (the reference has none; stop_gitm covers its failures): an
// event recorded on `stream` is polled until it completes or timeout_s
// passes.  Nothing on the device waits, so giving up leaves the context
// usable: the work in flight still runs to completion.
int gitm_vert_plan_wait(GitmVertPlan* P, void* stream, double timeout_s) {
  if (!P) return GITM_ERR_ARG;
  GitmVertCtx* ctx = P->ctx;
  if (!(timeout_s >= 0.0)) return set_err(ctx, GITM_ERR_ARG, "timeout_s must be >= 0");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  cudaEvent_t ev = nullptr;
  CUDA_TRY(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  cudaError_t e = cudaEventRecord(ev, static_cast<cudaStream_t>(stream));
  const auto t0 = std::chrono::steady_clock::now();
  while (e == cudaSuccess) {
    e = cudaEventQuery(ev);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) break;
    e = cudaSuccess;
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (el >= timeout_s) {
      cudaEventDestroy(ev);
      return set_err(ctx, GITM_ERR_TIMEOUT, "the stream did not finish within %.3f s", timeout_s);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  cudaEventDestroy(ev);
  if (e != cudaSuccess) return set_err(ctx, GITM_ERR_CUDA, "waiting on the stream failed: %s", cudaGetErrorString(e));
  return GITM_OK;
}

}  // extern "C"

// Saves (restore = false) or restores and frees (restore = true) device
// copies of every array a step writes, so autotune trials leave the state
// as it was.
static int snapshot(GitmVertPlan* P, std::vector<std::pair<double*, double*>>& bk, bool restore) {
  GitmVertCtx* ctx = P->ctx;
  if (!restore) {
    for (int m = 0; m < P->n_members; ++m) {
      const GitmColumnBatch& b = P->host_members[m];
      const int64_t cells = int64_t(b.n_alts + 4) * b.n_cols;
      struct F { double* p; int k; } fs[] = {{b.ndensity_s, NS}, {b.idensity_s, GITM_NIONS},
                                             {b.rho, 1}, {b.temperature, 1}, {b.velocity, 3},
                                             {b.vert_vel, NS}, {b.log_ns, NS}, {b.ndensity, 1},
                                             {b.gamma, 1}, {b.mean_major_mass, 1},
                                             {b.temp_unit, 1}, {b.cmax, 1}, {b.eddy, 1}};
      for (auto& f : fs) {
        if (!f.p) continue;
        double* cp = nullptr;
        CUDA_TRY(ctx, cudaMalloc(&cp, cells * f.k * sizeof(double)));
        CUDA_TRY(ctx, cudaMemcpy(cp, f.p, cells * f.k * sizeof(double), cudaMemcpyDeviceToDevice));
        bk.push_back({f.p, cp});
      }
    }
    return GITM_OK;
  }
  // restore: sizes are implied by the order of the saved list
  size_t idx = 0;
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnBatch& b = P->host_members[m];
    const int64_t cells = int64_t(b.n_alts + 4) * b.n_cols;
    struct F { double* p; int k; } fs[] = {{b.ndensity_s, NS}, {b.idensity_s, GITM_NIONS},
                                           {b.rho, 1}, {b.temperature, 1}, {b.velocity, 3},
                                           {b.vert_vel, NS}, {b.log_ns, NS}, {b.ndensity, 1},
                                           {b.gamma, 1}, {b.mean_major_mass, 1},
                                           {b.temp_unit, 1}, {b.cmax, 1}, {b.eddy, 1}};
    for (auto& f : fs) {
      if (!f.p) continue;
      CUDA_TRY(ctx, cudaMemcpy(f.p, bk[idx].second, cells * f.k * sizeof(double), cudaMemcpyDeviceToDevice));
      ++idx;
    }
  }
  for (auto& pr : bk) cudaFree(pr.second);
  bk.clear();
  return GITM_OK;
}

extern "C" int gitm_vert_plan_autotune(GitmVertPlan* P, double dt, int n_steps, GitmLaunchConfig* chosen) {
  if (!P) return GITM_ERR_ARG;
  GitmVertCtx* ctx = P->ctx;
  if (P->io != 0) return set_err(ctx, GITM_ERR_UNSUPPORTED, "autotune needs a GITM-array plan");
  if (n_steps < 1) n_steps = 1;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  std::vector<std::pair<double*, double*>> bk;
  int rc = snapshot(P, bk, false);
  if (rc) return rc;
  // steps per launch: one (the plain launch), n_steps and n_steps / 2
  std::vector<int> spls{1};
  if (n_steps / 2 > 1) spls.push_back(n_steps / 2);
  if (n_steps > 1) spls.push_back(n_steps);
  std::vector<GitmLaunchConfig> cands;
  for (int t : kThreadChoices)
    for (int spl : spls)
      for (int cps : {0, 1, 2, 3}) {
        GitmLaunchConfig c{t, 0, spl, cps};
        cands.push_back(c);
      }
  cudaEvent_t e0, e1;
  CUDA_TRY(ctx, cudaEventCreate(&e0));
  CUDA_TRY(ctx, cudaEventCreate(&e1));
  GitmLaunchConfig best = P->cfg;
  float best_ms = 1e30f;
  for (const GitmLaunchConfig& c : cands) {
    if (gitm_vert_plan_set_config(P, &c) != GITM_OK) continue;
    rc = launch_steps(P, dt, n_steps, 0);  // warm-up
    if (rc) break;
    CUDA_TRY(ctx, cudaEventRecord(e0));
    rc = launch_steps(P, dt, n_steps, 0);
    if (rc) break;
    CUDA_TRY(ctx, cudaEventRecord(e1));
    CUDA_TRY(ctx, cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc2 = snapshot(P, bk, true);
  CUDA_TRY(ctx, cudaMemset(P->d_status, 0, std::max<int64_t>(P->n_cols_total, 1) * sizeof(uint32_t)));
  if (rc) return rc;
  if (rc2) return rc2;
  rc = gitm_vert_plan_set_config(P, &best);
  if (chosen) *chosen = P->cfg;
  return rc;
}

extern "C" int gitm_vert_advance_native(GitmVertCtx* ctx, const GitmColumnBatch* members, int n_members,
                                        double dt, int n_steps) {
  GitmVertPlan* P = nullptr;
  int rc = gitm_vert_plan_create(ctx, members, n_members, &P);
  if (rc) return rc;
  rc = gitm_vert_plan_advance(P, dt, n_steps, nullptr);
  uint32_t st = 0;
  int64_t nbad = 0;
  if (!rc) rc = gitm_vert_plan_status(P, &st, &nbad, 0);
  plan_free(P);
  if (!rc && st) rc = set_err(ctx, GITM_ERR_COLUMN, "%lld columns reported status 0x%x", (long long)nbad, st);
  return rc;
}

// ------------------------------------------------------------------ adjoint
constexpr int kAdjThreads = ADJ_THREADS;

// Tiles, persistent grid and scratch of the adjoint kernel for the plan.
static int adjoint_prepare(GitmVertPlan* P) {
  GitmVertCtx* ctx = P->ctx;
  if (P->adj_ready) return GITM_OK;
  const int T = kAdjThreads, TS = SAVE_THREADS;
  P->adj_tiles.clear();
  P->save_tiles.clear();
  P->adj_smem = 0;
  P->adj_nc_max = 1;
  P->adj_per_max = 0;
  P->save_smem = 0;
  auto cut = [](std::vector<Tile>& out, int m, int64_t n_cols, int nc) {
    for (int64_t c0 = 0; c0 < n_cols; c0 += nc) {
      Tile t;
      t.member = m;
      t.nc = int(std::min<int64_t>(nc, n_cols - c0));
      t.c0 = c0;
      out.push_back(t);
    }
  };
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnBatch& b = P->host_members[m];
    const int nA = b.n_alts;
    int nc = std::max(1, std::min(T / nA, T / 32));
    while (nc > 1 && adj_smem_bytes(nA, nc) > ctx->max_smem) --nc;
    if (nA > T || adj_smem_bytes(nA, nc) > ctx->max_smem)
      return set_err(ctx, GITM_ERR_UNSUPPORTED, "adjoint: nAlts %d does not fit a CTA of %d threads", nA, T);
    P->adj_smem = std::max(P->adj_smem, adj_smem_bytes(nA, nc));
    P->adj_nc_max = std::max(P->adj_nc_max, nc);
    P->adj_per_max = std::max(P->adj_per_max, adj_state_doubles(nA));
    cut(P->adj_tiles, m, b.n_cols, nc);
    // the saving step kernel: columns per CTA of the forward layout
    int ns = std::max(1, std::min(TS / nA, TS / 32));
    while (ns > 1 && smem_bytes(nA, ns) > ctx->max_smem) --ns;
    if (nA > TS || smem_bytes(nA, ns) > ctx->max_smem)
      return set_err(ctx, GITM_ERR_UNSUPPORTED, "saving step: nAlts %d does not fit a CTA of %d threads", nA, TS);
    P->save_smem = std::max(P->save_smem, smem_bytes(nA, ns));
    cut(P->save_tiles, m, b.n_cols, ns);
  }
  if (P->adj_tiles.empty()) {
    P->adj_ready = true;
    return GITM_OK;
  }
  const void* fn = (plan_nalts(P) == 50) ? adjoint_kernel_fn_n50() : adjoint_kernel_fn();
  CUDA_TRY(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ctx->max_smem)));
  int per_sm = 0;
  CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, P->adj_smem));
  per_sm = std::max(per_sm, 1);
  P->adj_grid = int(std::min<size_t>(P->adj_tiles.size(), size_t(per_sm) * ctx->num_sms));
  P->adj_scratch_per_cta = size_t(ADJ_NSTATE) * P->adj_nc_max * P->adj_per_max + size_t(2) * NF * T;
  CUDA_TRY(ctx, cudaMalloc(&P->d_adj_tiles, P->adj_tiles.size() * sizeof(Tile)));
  CUDA_TRY(ctx, cudaMemcpy(P->d_adj_tiles, P->adj_tiles.data(), P->adj_tiles.size() * sizeof(Tile),
                           cudaMemcpyHostToDevice));
  if (cudaMalloc(&P->d_adj_scratch, size_t(P->adj_grid) * P->adj_scratch_per_cta * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, GITM_ERR_NOMEM, "adjoint: cannot allocate the stage-state scratch");
  }
  CUDA_TRY(ctx, cudaMalloc(&P->d_bars, std::max(1, P->n_members) * sizeof(GitmColumnAdjoint)));
  // the saving step kernel: its own tiles, the forward layout
  const void* sfn = kernel_for(0, GITM_SOLVER_RUSANOV, SAVE_THREADS, plan_nalts(P), true);
  if (!sfn) return set_err(ctx, GITM_ERR_ARG, "the saving step kernel is not built");
  CUDA_TRY(ctx, cudaFuncSetAttribute(sfn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(ctx->max_smem)));
  int sper = 0;
  CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&sper, sfn, TS, P->save_smem));
  sper = std::max(sper, 1);
  P->save_grid = int(std::min<size_t>(P->save_tiles.size(), size_t(sper) * ctx->num_sms));
  CUDA_TRY(ctx, cudaMalloc(&P->d_save_tiles, P->save_tiles.size() * sizeof(Tile)));
  CUDA_TRY(ctx, cudaMemcpy(P->d_save_tiles, P->save_tiles.data(), P->save_tiles.size() * sizeof(Tile),
                           cudaMemcpyHostToDevice));
  if (cudaMalloc(&P->d_save_scratch, size_t(P->save_grid) * NF * TS * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, GITM_ERR_NOMEM, "adjoint: cannot allocate the saving step's scratch");
  }
  P->adj_ready = true;
  return GITM_OK;
}

extern "C" int64_t gitm_vert_plan_saved_state_doubles(const GitmVertPlan* P) {
  if (!P) return 0;
  int per = 0;
  for (const GitmColumnBatch& b : P->host_members) per = std::max(per, adj_state_doubles(b.n_alts));
  return int64_t(ADJ_NSTATE) * P->n_cols_total * per;
}

static int adjoint_checks(GitmVertPlan* P) {
  GitmVertCtx* ctx = P->ctx;
  if (P->io != 0) return set_err(ctx, GITM_ERR_UNSUPPORTED, "the adjoint takes GITM-array plans");
  if (P->solver != GITM_SOLVER_RUSANOV || ctx->params.solver != GITM_SOLVER_RUSANOV)
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "the adjoint differentiates the Rusanov solver");
  if (ctx->params.compute_eddy)
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "the adjoint takes the eddy coefficient as an input: compute_eddy must be 0");
  return GITM_OK;
}

extern "C" int gitm_vert_plan_advance_saving(GitmVertPlan* P, double dt, double* states, void* stream) {
  if (!P) return GITM_ERR_ARG;
  GitmVertCtx* ctx = P->ctx;
  if (!states && P->n_cols_total > 0) return set_err(ctx, GITM_ERR_ARG, "states is NULL");
  if (!(dt > 0.0)) return set_err(ctx, GITM_ERR_ARG, "dt must be > 0");
  int rc = adjoint_checks(P);
  if (rc) return rc;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  rc = adjoint_prepare(P);
  if (rc) return rc;
  if (P->adj_tiles.empty()) return GITM_OK;
  KParams kp{};
  std::memset(&kp, 0, sizeof kp);
  kp.members = P->d_members;
  kp.tiles = P->d_save_tiles;
  kp.n_tiles = int(P->save_tiles.size());
  kp.n_steps = 1;
  kp.dt = dt;
  kp.status = P->d_status;
  kp.scratch = P->d_save_scratch;
  kp.prm = ctx->params;
  kp.save = states;
  kp.save_ncols = P->n_cols_total;
  kp.save_per = P->adj_per_max;
  void* args[] = {&kp};
  CUDA_TRY(ctx, cudaLaunchKernel(kernel_for(0, GITM_SOLVER_RUSANOV, SAVE_THREADS, plan_nalts(P), true), dim3(P->save_grid), dim3(SAVE_THREADS), args, P->save_smem,
                                 static_cast<cudaStream_t>(stream)));
  return GITM_OK;
}

extern "C" int gitm_vert_plan_adjoint(GitmVertPlan* P, const GitmColumnAdjoint* bars, double dt,
                                      const double* saved_states, void* stream) {
  if (!P) return GITM_ERR_ARG;
  GitmVertCtx* ctx = P->ctx;
  if (!bars && P->n_members > 0) return set_err(ctx, GITM_ERR_ARG, "bars is NULL");
  if (!(dt > 0.0)) return set_err(ctx, GITM_ERR_ARG, "dt must be > 0");
  int rc0 = adjoint_checks(P);
  if (rc0) return rc0;
  for (int m = 0; m < P->n_members; ++m) {
    const GitmColumnAdjoint& a = bars[m];
    if (!a.ndensity_s || !a.idensity_s || !a.rho || !a.temperature || !a.velocity || !a.vert_vel)
      return set_err(ctx, GITM_ERR_ARG, "member %d: the state adjoint arrays are required", m);
  }
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  int rc = adjoint_prepare(P);
  if (rc) return rc;
  if (P->adj_tiles.empty()) return GITM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  AParams kp;
  std::memset(&kp, 0, sizeof kp);
  if (P->n_members <= ADJ_INLINE_BARS) {
    // the descriptors travel with the launch: no copy that would wait for
    // the stream's earlier work
    for (int m = 0; m < P->n_members; ++m) kp.bars_inline[m] = bars[m];
    kp.n_inline = P->n_members;
  } else {
    CUDA_TRY(ctx, cudaMemcpyAsync(P->d_bars, bars, P->n_members * sizeof(GitmColumnAdjoint),
                                  cudaMemcpyHostToDevice, st));
  }
  kp.members = P->d_members;
  kp.bars = P->d_bars;
  kp.tiles = P->d_adj_tiles;
  kp.n_tiles = int(P->adj_tiles.size());
  kp.nc_max = P->adj_nc_max;
  kp.per_max = P->adj_per_max;
  kp.dt = dt;
  kp.status = P->d_status;
  kp.scratch = P->d_adj_scratch;
  kp.scratch_per_cta = P->adj_scratch_per_cta;
  kp.prm = ctx->params;
  kp.saved = saved_states;
  kp.saved_ncols = P->n_cols_total;
  void* args[] = {&kp};
  CUDA_TRY(ctx, cudaLaunchKernel((plan_nalts(P) == 50) ? adjoint_kernel_fn_n50() : adjoint_kernel_fn(), dim3(P->adj_grid),
                                 dim3(kAdjThreads), args, P->adj_smem, st));
  return GITM_OK;
}

// ------------------------------------------------------------------ staging
static int arena_reserve(GitmVertCtx* ctx, size_t bytes) {
  if (bytes <= ctx->arena_bytes) return GITM_OK;
  CUDA_TRY(ctx, cudaDeviceSynchronize());
  cudaFree(ctx->arena);
  ctx->arena = nullptr;
  ctx->arena_bytes = 0;
  if (cudaMalloc(&ctx->arena, bytes) != cudaSuccess) {
    cudaGetLastError();
    return set_err(ctx, GITM_ERR_NOMEM, "cannot allocate %zu bytes of device staging", bytes);
  }
  ctx->arena_bytes = bytes;
  return GITM_OK;
}

static bool is_pinned_host(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

namespace {

// One array of a member in native layout: nfield x G rows of n_cols doubles
// (or one row of n_cols for per-column scalars).
struct ArraySpec {
  double* GitmColumnBatch::* field;
  int rows_per_cell;  // fields per cell (0: a [n_cols] vector; -1: lbc [20][n_cols])
  bool in, out;
};

const ArraySpec kArrays[] = {
    {&GitmColumnBatch::ndensity_s, NS, true, true},
    {&GitmColumnBatch::idensity_s, GITM_NIONS, true, true},
    {&GitmColumnBatch::rho, 1, true, true},
    {&GitmColumnBatch::temperature, 1, true, true},
    {&GitmColumnBatch::velocity, 3, true, true},
    {&GitmColumnBatch::vert_vel, NS, true, true},
    {&GitmColumnBatch::log_ns, NS, false, true},
    {&GitmColumnBatch::ndensity, 1, false, true},
    {&GitmColumnBatch::gamma, 1, true, true},
    {&GitmColumnBatch::mean_major_mass, 1, true, true},
    {&GitmColumnBatch::temp_unit, 1, true, true},
    {&GitmColumnBatch::cmax, 1, true, true},
    {&GitmColumnBatch::eddy, 1, true, true},  // copied back when compute_eddy = 1
};
struct ConstSpec {
  const double* GitmColumnBatch::* field;
  int rows_per_cell;  // as above
};
const ConstSpec kInputs[] = {
    {&GitmColumnBatch::ivel_up, 1},   {&GitmColumnBatch::cos_lat, 0},   {&GitmColumnBatch::sza, 0},
    {&GitmColumnBatch::mlat, 0},      {&GitmColumnBatch::lbc, -1},
    {&GitmColumnBatch::altitude, 1},  {&GitmColumnBatch::gravity, 1},
    {&GitmColumnBatch::dalt_c, 1},    {&GitmColumnBatch::inv_r, 1},
    {&GitmColumnBatch::heating, 1},   {&GitmColumnBatch::heating_scale, 0},
};

inline int64_t rows_of(int rpc, int G) { return rpc > 0 ? int64_t(rpc) * G : (rpc == 0 ? 1 : 2 * GITM_LBC_NVALUES); }

}  // namespace

// Host-pointer form: each member's columns are cut into chunks; every chunk
// is copied to device staging (one 2-D copy per array), advanced and copied
// back on one of three streams, so copies of one chunk overlap the kernel of
// the previous one.
extern "C" int gitm_vert_advance_native_host(GitmVertCtx* ctx, const GitmColumnBatch* members,
                                             int n_members, double dt, int n_steps) {
  if (!ctx || (n_members > 0 && !members) || n_members < 0) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  for (cudaStream_t& st : ctx->streams)
    if (!st) CUDA_TRY(ctx, cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const GitmVertParams& prm = ctx->params;
  // chunking: about 16 chunks per member, at least 1024 columns each (the
  // copies of one chunk overlap the step of another)
  struct Chunk { int m; int64_t c0, n; size_t off; };
  std::vector<Chunk> chunks;
  size_t total = 0;
  for (int m = 0; m < n_members; ++m) {
    int rc = check_member(ctx, members[m], prm);
    if (rc) return rc;
    const GitmColumnBatch& b = members[m];
    const int G = b.n_alts + 4;
    const int64_t per = std::max<int64_t>(1024, (b.n_cols + 15) / 16);
    for (int64_t c0 = 0; c0 < b.n_cols; c0 += per) {
      Chunk ch{m, c0, std::min(per, b.n_cols - c0), total};
      size_t rows = 0;
      for (const ArraySpec& a : kArrays)
        if (b.*(a.field)) rows += rows_of(a.rows_per_cell, G);
      for (const ConstSpec& a : kInputs) {
        if (!(b.*(a.field))) continue;
        const bool grid = (a.field == &GitmColumnBatch::altitude || a.field == &GitmColumnBatch::gravity ||
                           a.field == &GitmColumnBatch::dalt_c || a.field == &GitmColumnBatch::inv_r);
        if (grid && !b.grid_per_column) continue;  // shared grid stays on the host
        rows += rows_of(a.rows_per_cell, G);
      }
      total += rows * ch.n * sizeof(double);
      total = (total + 255) & ~size_t(255);
      chunks.push_back(ch);
    }
  }
  if (chunks.empty()) return GITM_OK;
  int rc = arena_reserve(ctx, total);
  if (rc) return rc;
  // device-side member per chunk (compact layout, n_cols = chunk size)
  std::vector<GitmColumnBatch> dm(chunks.size());
  for (size_t j = 0; j < chunks.size(); ++j) {
    const Chunk& ch = chunks[j];
    const GitmColumnBatch& b = members[ch.m];
    const int G = b.n_alts + 4;
    GitmColumnBatch d = b;
    d.n_cols = ch.n;
    char* p = ctx->arena + ch.off;
    for (const ArraySpec& a : kArrays) {
      if (!(b.*(a.field))) { d.*(a.field) = nullptr; continue; }
      d.*(a.field) = reinterpret_cast<double*>(p);
      p += rows_of(a.rows_per_cell, G) * ch.n * sizeof(double);
    }
    for (const ConstSpec& a : kInputs) {
      if (!(b.*(a.field))) { d.*(a.field) = nullptr; continue; }
      const bool grid = (a.field == &GitmColumnBatch::altitude || a.field == &GitmColumnBatch::gravity ||
                         a.field == &GitmColumnBatch::dalt_c || a.field == &GitmColumnBatch::inv_r);
      if (grid && !b.grid_per_column) continue;  // host grid pointer, read at plan creation
      d.*(a.field) = reinterpret_cast<double*>(p);
      p += rows_of(a.rows_per_cell, G) * ch.n * sizeof(double);
    }
    dm[j] = d;
  }
  // per-column grids must be on the device before the plan reads them
  for (size_t j = 0; j < chunks.size(); ++j) {
    const GitmColumnBatch& b = members[chunks[j].m];
    if (!b.grid_per_column) continue;
    const int G = b.n_alts + 4;
    const size_t hp = size_t(b.n_cols) * sizeof(double), w = size_t(chunks[j].n) * sizeof(double);
    const double* src[4] = {b.altitude, b.gravity, b.dalt_c, b.inv_r};
    const double* dst[4] = {dm[j].altitude, dm[j].gravity, dm[j].dalt_c, dm[j].inv_r};
    for (int q = 0; q < 4; ++q)
      CUDA_TRY(ctx, cudaMemcpy2D(const_cast<double*>(dst[q]), w, src[q] + chunks[j].c0, hp, w, G,
                                 cudaMemcpyHostToDevice));
  }
  // the plan of the previous call serves again when nothing it was built
  // from changed: the staging arena, the solver, the chunks and the shared
  // altitude grids (compared by value); per-column grids build a new plan
  std::vector<uint64_t> key;
  bool cacheable = true;
  auto put = [&](double v) { uint64_t u; std::memcpy(&u, &v, 8); key.push_back(u); };
  key.push_back(uint64_t(reinterpret_cast<uintptr_t>(ctx->arena)));
  key.push_back(uint64_t(prm.solver));
  for (const Chunk& ch : chunks) {
    const GitmColumnBatch& b = members[ch.m];
    key.push_back(uint64_t(ch.m));
    key.push_back(uint64_t(ch.c0));
    key.push_back(uint64_t(ch.n));
    key.push_back(uint64_t(b.n_alts));
    if (b.grid_per_column) cacheable = false;
  }
  for (int m = 0; m < n_members && cacheable; ++m) {
    const GitmColumnBatch& b = members[m];
    uint64_t present = 0, bit = 1;  // which arrays the call passes (they set the arena layout)
    for (const ArraySpec& a : kArrays) { if (b.*(a.field)) present |= bit; bit <<= 1; }
    for (const ConstSpec& a : kInputs) { if (b.*(a.field)) present |= bit; bit <<= 1; }
    key.push_back(present);
    key.push_back(uint64_t(b.n_cols));
    for (const double* g : {b.altitude, b.gravity, b.dalt_c, b.inv_r})
      for (int i = 0; i < b.n_alts + 4; ++i) put(g[i]);
  }
  GitmVertPlan* P = nullptr;
  if (cacheable && ctx->host_plan && key == ctx->host_plan_key) {
    P = ctx->host_plan;
  } else {
    plan_free(ctx->host_plan);
    ctx->host_plan = nullptr;
    ctx->host_plan_key.clear();
    // plan_create checks that state arrays are device pointers: they are
    rc = gitm_vert_plan_create(ctx, dm.data(), int(dm.size()), &P);
    if (rc) return rc;
    // 128 threads with the accumulator in scratch, persistent grid
    GitmLaunchConfig cfg{128, 0, 1, 0};
    rc = gitm_vert_plan_set_config(P, &cfg);
    if (rc) { plan_free(P); return rc; }
    if (cacheable) {
      ctx->host_plan = P;
      ctx->host_plan_key = key;
    }
  }
  // tile ranges per chunk (tiles are ordered by member)
  std::vector<int> t0(chunks.size() + 1, int(P->tiles.size()));
  for (int t = int(P->tiles.size()) - 1; t >= 0; --t) t0[P->tiles[t].member] = t;
  for (int j = int(chunks.size()) - 1; j >= 0; --j)
    if (t0[j] > t0[j + 1]) t0[j] = t0[j + 1];
  const void* fn = kernel_for(0, P->solver, P->cfg.threads, plan_nalts(P));
  // one stream per role: copies in (streams[0]), steps (streams[1]), copies
  // out (streams[2]); a chunk's step waits for its copies in and its copies
  // out wait for its step, so each copy engine streams without waiting for
  // the other direction
  cudaStream_t s_in = ctx->streams[0], s_k = ctx->streams[1], s_out = ctx->streams[2];
  while (ctx->events.size() < 2 * chunks.size()) {
    cudaEvent_t e;
    CUDA_TRY(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->events.push_back(e);
  }
  for (size_t j = 0; j < chunks.size() && !rc; ++j) {
    const Chunk& ch = chunks[j];
    const GitmColumnBatch& b = members[ch.m];
    const GitmColumnBatch& d = dm[j];
    const int G = b.n_alts + 4;
    const size_t hp = size_t(b.n_cols) * sizeof(double), w = size_t(ch.n) * sizeof(double);
    cudaEvent_t e_in = ctx->events[2 * j], e_k = ctx->events[2 * j + 1];
    auto h2d = [&](double* dst, const double* src, int64_t rows) -> int {
      CUDA_TRY(ctx, cudaMemcpy2DAsync(dst, w, src + ch.c0, hp, w, rows, cudaMemcpyHostToDevice, s_in));
      return GITM_OK;
    };
    for (const ArraySpec& a : kArrays) {
      if (!a.in || !(b.*(a.field))) continue;
      if (!prm.compute_coefficients || (a.field != &GitmColumnBatch::gamma && a.field != &GitmColumnBatch::mean_major_mass &&
                                        a.field != &GitmColumnBatch::temp_unit && a.field != &GitmColumnBatch::cmax))
        if ((rc = h2d(d.*(a.field), b.*(a.field), rows_of(a.rows_per_cell, G)))) break;
    }
    for (const ConstSpec& a : kInputs) {
      if (rc || !(d.*(a.field)) || !(b.*(a.field))) continue;
      if (d.*(a.field) == b.*(a.field)) continue;  // shared grid: read from the host at plan creation
      const bool grid = (a.field == &GitmColumnBatch::altitude || a.field == &GitmColumnBatch::gravity ||
                         a.field == &GitmColumnBatch::dalt_c || a.field == &GitmColumnBatch::inv_r);
      if (grid) continue;  // per-column grid: copied before the plan was built
      if ((rc = h2d(const_cast<double*>(d.*(a.field)), b.*(a.field), rows_of(a.rows_per_cell, G)))) break;
    }
    if (rc) break;
    CUDA_TRY(ctx, cudaEventRecord(e_in, s_in));
    CUDA_TRY(ctx, cudaStreamWaitEvent(s_k, e_in, 0));
    const int spl = std::max(1, P->cfg.steps_per_launch);
    KParams kp{};
    std::memset(&kp, 0, sizeof kp);
    kp.members = P->d_members;
    kp.tiles = P->d_tiles + t0[j];
    kp.n_tiles = t0[j + 1] - t0[j];
    kp.dt = dt;
    kp.status = P->d_status;
    kp.scratch = P->d_scratch;
    kp.scratch_per_cta = P->scratch_per_cta;
    kp.prm = prm;
    const int cgrid = P->d_scratch ? std::min(kp.n_tiles, P->grid) : kp.n_tiles;
    for (int done = 0; done < n_steps && kp.n_tiles > 0; done += spl) {
      kp.n_steps = std::min(spl, n_steps - done);
      void* args[] = {&kp};
      cudaError_t e = cudaLaunchKernel(fn, dim3(cgrid), dim3(P->cfg.threads), args, P->smem, s_k);
      if (e != cudaSuccess) { rc = set_err(ctx, GITM_ERR_CUDA, "launch: %s", cudaGetErrorString(e)); break; }
    }
    if (rc) break;
    CUDA_TRY(ctx, cudaEventRecord(e_k, s_k));
    CUDA_TRY(ctx, cudaStreamWaitEvent(s_out, e_k, 0));
    for (const ArraySpec& a : kArrays) {
      if (rc || !a.out || !(b.*(a.field))) continue;
      if (!prm.compute_coefficients && (a.field == &GitmColumnBatch::gamma || a.field == &GitmColumnBatch::mean_major_mass ||
                                        a.field == &GitmColumnBatch::temp_unit || a.field == &GitmColumnBatch::cmax))
        continue;
      if (!prm.compute_eddy && a.field == &GitmColumnBatch::eddy) continue;
      cudaError_t e = cudaMemcpy2DAsync(b.*(a.field) + ch.c0, hp, d.*(a.field), w, w,
                                        rows_of(a.rows_per_cell, G), cudaMemcpyDeviceToHost, s_out);
      if (e != cudaSuccess) rc = set_err(ctx, GITM_ERR_CUDA, "copy back: %s", cudaGetErrorString(e));
    }
  }
  for (cudaStream_t st : ctx->streams) cudaStreamSynchronize(st);
  uint32_t sto = 0;
  int64_t nbad = 0;
  const int rcs = gitm_vert_plan_status(P, &sto, &nbad, 1);
  if (!rc) rc = rcs;
  if (P != ctx->host_plan) plan_free(P);
  if (!rc && sto) rc = set_err(ctx, GITM_ERR_COLUMN, "%lld columns reported status 0x%x", (long long)nbad, sto);
  (void)is_pinned_host;
  return rc;
}

// ------------------------------------------------------------------ ModVertical
extern "C" int gitm_vert_advance_1d(GitmVertCtx* ctx, const GitmModVerticalBatch* batch, double dt,
                                    uint32_t* status_words_device) {
  if (!ctx || !batch) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  const GitmModVerticalBatch& v = *batch;
  if (v.n_alts < 8 || v.n_alts > GITM_MAX_NALTS) return set_err(ctx, GITM_ERR_ARG, "n_alts out of range");
  if (v.n_cols <= 0) return GITM_OK;
  const void* req[] = {v.log_rho, v.temp, v.vel_gd, v.log_ns, v.vert_vel, v.log_ins, v.ivel, v.cmax,
                       v.mean_major_mass, v.gamma, v.eddy, v.centrifugal, v.coriolis, v.sza, v.mlat,
                       v.altitude, v.gravity, v.dalt_c, v.inv_r};
  for (const void* p : req)
    if (!p || !is_device_ptr(p)) return set_err(ctx, GITM_ERR_ARG, "ModVertical arrays must be non-NULL device pointers");
  if (ctx->params.use_msis_bcs && !v.lbc) return set_err(ctx, GITM_ERR_ARG, "use_msis_bcs=1 needs the lbc table");
  if (ctx->params.compute_eddy)
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "compute_eddy applies to the GITM-array form");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  GitmVertPlan* P = new GitmVertPlan();
  P->ctx = ctx;
  P->io = 1;
  P->solver = ctx->params.solver;
  P->n_members = 1;
  GitmColumnBatch shape;
  std::memset(&shape, 0, sizeof shape);
  shape.n_alts = v.n_alts;
  shape.n_cols = v.n_cols;
  shape.grid_per_column = v.grid_per_column;
  P->host_members.assign(1, shape);
  P->dev_members_host.resize(1);
  std::memset(&P->dev_members_host[0], 0, sizeof(DevMember));
  P->dev_members_host[0].b = shape;
  P->dev_members_host[0].mv = v;
  P->n_cols_total = v.n_cols;
  const double* alt = v.altitude;
  const double* grav = v.gravity;
  const double* dalt = v.dalt_c;
  const double* invr = v.inv_r;
  int gpc = v.grid_per_column;
  int rc = plan_common(P, &alt, &grav, &dalt, &invr, &gpc);
  if (!rc) rc = launch_steps(P, dt, 1, nullptr);
  if (!rc) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = set_err(ctx, GITM_ERR_CUDA, "step: %s", cudaGetErrorString(e));
  }
  if (!rc && status_words_device) {
    cudaError_t e = cudaMemcpy(status_words_device, P->d_status, v.n_cols * sizeof(uint32_t), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) rc = set_err(ctx, GITM_ERR_CUDA, "status copy: %s", cudaGetErrorString(e));
  }
  uint32_t sto = 0;
  int64_t nbad = 0;
  if (!rc) rc = gitm_vert_plan_status(P, &sto, &nbad, 0);
  plan_free(P);
  if (!rc && sto) rc = set_err(ctx, GITM_ERR_COLUMN, "%lld columns reported status 0x%x", (long long)nbad, sto);
  return rc;
}

// ------------------------------------------------------------------ CFL
// calc_timestep_vertical, calc_timestep.f90:109-145: cMax on cells
// 0..nAlts+1 and the per-column CFL step, reduced to one minimum.  Positive
// doubles order like their bit patterns, so the minimum is an integer atomicMin.
__global__ void cfl_kernel(GitmColumnBatch b, const double* dalt, int gpc, double cfl, int ion,
                           unsigned long long* out) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double dtl = 1.0e32;
  if (c < b.n_cols) {
    const int nA = b.n_alts, G = nA + 4;
    const int64_t n = b.n_cols;
    double mxr = 0.0, mxi = 0.0;
    for (int g = 1; g <= nA + 2; ++g) {
      double mx = fabs(b.vert_vel[(int64_t(0) * G + g) * n + c]);
      for (int s = 1; s < NS; ++s) mx = fmax(mx, fabs(b.vert_vel[(int64_t(s) * G + g) * n + c]));
      const double snd = sqrt(b.gamma[int64_t(g) * n + c] * b.temperature[int64_t(g) * n + c]);
      const double cm = mx + snd;
      if (b.cmax) b.cmax[int64_t(g) * n + c] = cm;
      if (g >= 2 && g <= nA + 1) {
        const double dz = gpc ? dalt[int64_t(g) * n + c] : dalt[g];
        mxr = fmax(mxr, cm / dz);
        if (ion) mxi = fmax(mxi, (fabs(b.ivel_up[int64_t(g) * n + c]) + snd) / dz);
      }
    }
    dtl = fmin(dtl, cfl / mxr);
    if (ion) dtl = fmin(dtl, cfl / mxi);
  }
  for (int off = 16; off > 0; off >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, off));
  if ((threadIdx.x & 31) == 0 && dtl > 0.0) atomicMin(out, __double_as_longlong(dtl));
}

extern "C" int gitm_vert_cfl_dt(GitmVertCtx* ctx, const GitmColumnBatch* members, int n_members, double cfl,
                                double dt_in, double dt_end, double* dt_out) {
  if (!ctx || !dt_out || (n_members > 0 && !members)) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (!ctx->d_scalar) CUDA_TRY(ctx, cudaMalloc(&ctx->d_scalar, sizeof(double)));
  const double init = 1.0e32;
  CUDA_TRY(ctx, cudaMemcpy(ctx->d_scalar, &init, sizeof init, cudaMemcpyHostToDevice));
  for (int m = 0; m < n_members; ++m) {
    const GitmColumnBatch& b = members[m];
    if (b.n_cols <= 0) continue;
    if (!b.vert_vel || !b.gamma || !b.temperature || !b.dalt_c || (ctx->params.use_ion_advection && !b.ivel_up))
      return set_err(ctx, GITM_ERR_ARG, "cfl needs vert_vel, gamma, temperature, dalt_c (and ivel_up)");
    const int threads = 256;
    const unsigned blocks = unsigned((b.n_cols + threads - 1) / threads);
    cfl_kernel<<<blocks, threads>>>(b, b.dalt_c, b.grid_per_column, cfl, ctx->params.use_ion_advection,
                                    reinterpret_cast<unsigned long long*>(ctx->d_scalar));
    CUDA_TRY(ctx, cudaGetLastError());
  }
  double local = 0.0;
  CUDA_TRY(ctx, cudaMemcpy(&local, ctx->d_scalar, sizeof local, cudaMemcpyDeviceToHost));
  // DtLocal = min(DtLocal, DtEnd); Dt = min(Dt, DtVertical)  (calc_timestep.f90:141-147)
  *dt_out = std::min(dt_in, std::min(local, dt_end));
  return GITM_OK;
}

// ------------------------------------------------------------------ Fortran layout
// advance_vertical for every column of a range of blocks.  The GITM arrays
// are gathered into a native-layout member (columns ordered iLon fastest,
// then iLat, then iBlock, which is also their order in Fortran memory),
// advanced with the coefficients the host computed (calc_pressure,
// calc_timestep_vertical and calc_rates ran before, as in the reference),
// and scattered back with the copies advance_vertical.f90:152-155,214-217
// makes into SpeciesDensityOld / SpeciesDensity.
namespace {

__host__ __device__ inline int64_t fa_off(const GitmFArray& a, int lon, int lat, int alt, int k, int blk) {
  return int64_t(lon - a.lower[0]) * a.stride[0] + int64_t(lat - a.lower[1]) * a.stride[1] +
         int64_t(alt - a.lower[2]) * a.stride[2] + int64_t(k - a.lower[3]) * a.stride[3] +
         int64_t(blk - a.lower[4]) * a.stride[4];
}

struct FMap {
  GitmFArray fa;  // Fortran side
  int k;          // Fortran 4th index
  int64_t nat;    // offset of this field's first row in the native buffer
  int g_lo, g_hi; // cells copied (g = iAlt + 1); g_hi < g_lo: one value per column (iAlt = alt_fixed)
  int alt_fixed;
};

// dir 0: Fortran -> native; 1: native -> Fortran
__global__ void fortran_copy_kernel(const FMap* maps, int nmaps, double* nat, int dir, int nLons, int nLats,
                                    int bf, int64_t ncols, int G) {
  const FMap mp = maps[blockIdx.y];
  const int64_t total = (mp.g_hi >= mp.g_lo) ? int64_t(mp.g_hi - mp.g_lo + 1) * ncols : ncols;
  for (int64_t w = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; w < total; w += int64_t(gridDim.x) * blockDim.x) {
    const int64_t c = w % ncols;
    const int g = (mp.g_hi >= mp.g_lo) ? int(w / ncols) + mp.g_lo : -1;
    const int lon = int(c % nLons) + 1;
    const int lat = int((c / nLons) % nLats) + 1;
    const int blk = int(c / (int64_t(nLons) * nLats)) + bf;
    const int alt = (g >= 0) ? g - 1 : mp.alt_fixed;
    double* f = mp.fa.data + fa_off(mp.fa, lon, lat, alt, mp.k, blk);
    double* v = nat + mp.nat + ((g >= 0) ? int64_t(g) * ncols + c : c);
    if (dir == 0) *v = *f;
    else *f = *v;
  }
  (void)nmaps;
  (void)G;
}

void host_copy(const FMap& mp, double* nat, int dir, int nLons, int nLats, int bf, int64_t ncols) {
  const int64_t total = (mp.g_hi >= mp.g_lo) ? int64_t(mp.g_hi - mp.g_lo + 1) * ncols : ncols;
  for (int64_t w = 0; w < total; ++w) {
    const int64_t c = w % ncols;
    const int g = (mp.g_hi >= mp.g_lo) ? int(w / ncols) + mp.g_lo : -1;
    const int lon = int(c % nLons) + 1;
    const int lat = int((c / nLons) % nLats) + 1;
    const int blk = int(c / (int64_t(nLons) * nLats)) + bf;
    const int alt = (g >= 0) ? g - 1 : mp.alt_fixed;
    double* f = mp.fa.data + fa_off(mp.fa, lon, lat, alt, mp.k, blk);
    double* v = nat + mp.nat + ((g >= 0) ? int64_t(g) * ncols + c : c);
    if (dir == 0) *v = *f;
    else *f = *v;
  }
}

}  // namespace

extern "C" int gitm_vert_advance_fortran(GitmVertCtx* ctx, const GitmFortranState* st, int block_first,
                                         int block_last, double dt, int on_device) {
  if (!ctx || !st) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  const int nLons = st->n_lons, nLats = st->n_lats, nA = st->n_alts, G = nA + 4;
  if (nLons <= 0 || nLats <= 0 || block_first < 1 || block_last < block_first || block_last > st->n_blocks)
    return set_err(ctx, GITM_ERR_ARG, "bad grid or block range");
  if (nA < 8 || nA > GITM_MAX_NALTS) return set_err(ctx, GITM_ERR_ARG, "n_alts out of range");
  const GitmFArray* req[] = {&st->ndensity_s, &st->idensity_s, &st->rho, &st->temperature, &st->velocity,
                             &st->ivelocity, &st->vertical_velocity, &st->gamma, &st->mean_major_mass,
                             &st->temp_unit, &st->cmax, &st->kappa_eddy, &st->altitude, &st->gravity,
                             &st->dalt, &st->inv_r, &st->cos_latitude, &st->sza, &st->mlatitude};
  for (const GitmFArray* a : req)
    if (!a->data) return set_err(ctx, GITM_ERR_ARG, "a required Fortran array is NULL");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t ncols = int64_t(nLons) * nLats * (block_last - block_first + 1);
  // native member layout inside one buffer
  int64_t off = 0;
  auto take = [&](int64_t rows) { int64_t o = off; off += rows * ncols; return o; };
  const int64_t o_nd = take(NS * G), o_id = take(GITM_NIONS * G), o_rho = take(G), o_t = take(G),
                o_v = take(3 * G), o_w = take(NS * G), o_lns = take(NS * G), o_n = take(G), o_gm = take(G),
                o_mm = take(G), o_tu = take(G), o_cm = take(G), o_iv = take(G), o_ed = take(G),
                o_cl = take(1), o_sz = take(1), o_ml = take(1), o_al = take(G), o_gr = take(G),
                o_dz = take(G), o_ir = take(G);
  const int64_t n_nat = off;
  std::vector<FMap> in, outm, sd_old, sd_new;
  auto add = [&](std::vector<FMap>& v, const GitmFArray& fa, int k, int64_t nat, int glo, int ghi, int altf = 0) {
    FMap m;
    m.fa = fa;
    m.k = k;
    m.nat = nat;
    m.g_lo = glo;
    m.g_hi = ghi;
    m.alt_fixed = altf;
    v.push_back(m);
  };
  const int gl = 0, gh = G - 1;
  for (int s = 0; s < NS; ++s) add(in, st->ndensity_s, s + 1, o_nd + int64_t(s) * G * ncols, gl, gh);
  for (int s = 0; s < GITM_NIONS; ++s) add(in, st->idensity_s, s + 1, o_id + int64_t(s) * G * ncols, gl, gh);
  add(in, st->rho, 1, o_rho, gl, gh);
  add(in, st->temperature, 1, o_t, gl, gh);
  for (int d = 0; d < 3; ++d) add(in, st->velocity, d + 1, o_v + int64_t(d) * G * ncols, gl, gh);
  for (int s = 0; s < NS; ++s) add(in, st->vertical_velocity, s + 1, o_w + int64_t(s) * G * ncols, gl, gh);
  add(in, st->gamma, 1, o_gm, gl, gh);
  add(in, st->mean_major_mass, 1, o_mm, gl, gh);
  add(in, st->temp_unit, 1, o_tu, gl, gh);
  add(in, st->cmax, 3, o_cm, 1, G - 2);  // cMax_GDB(:,:,0:nAlts+1,iUp_,:)
  add(in, st->ivelocity, 3, o_iv, gl, gh);
  add(in, st->kappa_eddy, 1, o_ed, 1, G - 2);  // EddyCoef_1d(0:nAlts+1)
  add(in, st->cos_latitude, 1, o_cl, 1, 0, 0);
  add(in, st->sza, 1, o_sz, 1, 0, 0);
  add(in, st->mlatitude, 1, o_ml, 1, 0, nA);  // MLatitude(iLon,iLat,nAlts,iBlock)
  add(in, st->altitude, 1, o_al, gl, gh);
  add(in, st->gravity, 1, o_gr, gl, gh);
  add(in, st->dalt, 1, o_dz, gl, gh);
  add(in, st->inv_r, 1, o_ir, gl, gh);
  for (int s = 0; s < NS; ++s) add(outm, st->ndensity_s, s + 1, o_nd + int64_t(s) * G * ncols, gl, gh);
  for (int s = 0; s < GITM_NIONS; ++s) add(outm, st->idensity_s, s + 1, o_id + int64_t(s) * G * ncols, gl, gh);
  add(outm, st->rho, 1, o_rho, gl, gh);
  add(outm, st->temperature, 1, o_t, gl, gh);
  for (int d = 0; d < 3; ++d) add(outm, st->velocity, d + 1, o_v + int64_t(d) * G * ncols, gl, gh);
  for (int s = 0; s < NS; ++s) add(outm, st->vertical_velocity, s + 1, o_w + int64_t(s) * G * ncols, gl, gh);
  if (st->log_ns.data)
    for (int s = 0; s < NS; ++s) add(outm, st->log_ns, s + 1, o_lns + int64_t(s) * G * ncols, gl, gh);
  if (st->ndensity.data) add(outm, st->ndensity, 1, o_n, gl, gh);
  // SpeciesDensity(Old)(:,:,:,1:nSpeciesTotal) = NDensityS; (nSpeciesTotal+1:) = IDensityS(1:nIons-1)
  auto species_maps = [&](std::vector<FMap>& v, const GitmFArray& sd) {
    if (!sd.data) return;
    for (int s = 0; s < NS; ++s) add(v, sd, s + 1, o_nd + int64_t(s) * G * ncols, gl, gh);
    for (int s = 0; s < GITM_NIONS - 1; ++s) add(v, sd, 11 + s + 1, o_id + int64_t(s) * G * ncols, gl, gh);
  };
  species_maps(sd_old, st->species_density_old);
  species_maps(sd_new, st->species_density);

  GitmVertParams saved = ctx->params;
  ctx->params.compute_coefficients = 0;
  ctx->params.compute_eddy = 0;  // calc_sources runs on the host
  GitmColumnBatch b;
  std::memset(&b, 0, sizeof b);
  b.n_alts = nA;
  b.grid_per_column = 1;
  b.n_cols = ncols;
  int rc = GITM_OK;
  std::vector<double> hbuf;
  double* base = nullptr;
  if (on_device) {
    rc = arena_reserve(ctx, size_t(n_nat) * sizeof(double));
    base = reinterpret_cast<double*>(ctx->arena);
  } else {
    hbuf.assign(size_t(n_nat), 0.0);
    base = hbuf.data();
  }
  if (!rc) {
    b.ndensity_s = base + o_nd; b.idensity_s = base + o_id; b.rho = base + o_rho; b.temperature = base + o_t;
    b.velocity = base + o_v; b.vert_vel = base + o_w; b.log_ns = base + o_lns; b.ndensity = base + o_n;
    b.gamma = base + o_gm; b.mean_major_mass = base + o_mm; b.temp_unit = base + o_tu; b.cmax = base + o_cm;
    b.ivel_up = base + o_iv; b.eddy = base + o_ed; b.cos_lat = base + o_cl; b.sza = base + o_sz;
    b.mlat = base + o_ml; b.altitude = base + o_al; b.gravity = base + o_gr; b.dalt_c = base + o_dz;
    b.inv_r = base + o_ir;
  }
  auto run_maps = [&](const std::vector<FMap>& v, int dir) -> int {
    if (v.empty()) return GITM_OK;
    if (!on_device) {
      for (const FMap& m : v) host_copy(m, base, dir, nLons, nLats, block_first, ncols);
      return GITM_OK;
    }
    FMap* dm = nullptr;
    CUDA_TRY(ctx, cudaMalloc(&dm, v.size() * sizeof(FMap)));
    cudaMemcpy(dm, v.data(), v.size() * sizeof(FMap), cudaMemcpyHostToDevice);
    const int64_t work = int64_t(G) * ncols;
    dim3 grid(unsigned(std::min<int64_t>((work + 255) / 256, 4096)), unsigned(v.size()));
    fortran_copy_kernel<<<grid, 256>>>(dm, int(v.size()), base, dir, nLons, nLats, block_first, ncols, G);
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(dm);
    if (e != cudaSuccess) return set_err(ctx, GITM_ERR_CUDA, "fortran copy: %s", cudaGetErrorString(e));
    return GITM_OK;
  };
  if (!rc) {
    if (on_device) CUDA_TRY(ctx, cudaMemset(base, 0, size_t(n_nat) * sizeof(double)));
    rc = run_maps(in, 0);
  }
  if (!rc) rc = run_maps(sd_old, 1);  // SpeciesDensityOld = state before the step
  if (!rc) rc = on_device ? gitm_vert_advance_native(ctx, &b, 1, dt, 1)
                          : gitm_vert_advance_native_host(ctx, &b, 1, dt, 1);
  const bool column_err = (rc == GITM_ERR_COLUMN);
  if (!rc || column_err) {
    int rc2 = run_maps(outm, 1);
    if (!rc2) rc2 = run_maps(sd_new, 1);
    if (rc2) rc = rc2;
  }
  ctx->params = saved;
  return rc;
}

// ------------------------------------------------------------------ no-allocation entry point
// gitm_vert_advance_native_noalloc: the step of one member without any device
// allocation, for callers that cannot allocate device memory while they run:
// a GITM host whose GPU memory is held by its own pool (a caching allocator
// that has reserved the device), and per-step loops that must not pay the
// device synchronisation an allocation implies.  Everything the step needs
// beyond the caller's inputs and outputs -- the member descriptor, the tile
// list, the grid coefficients and the RK accumulators of the persistent CTAs
// -- lives in the file-scope array below, which every GPU that loads this
// library holds until the process exits.
namespace {

constexpr int64_t kNoAllocMaxCols = 262144;        // columns per call
constexpr int kNoAllocThreads = 128;               // launch shape (accumulators in scratch)
constexpr int kNoAllocSlots = 448;                 // persistent CTAs (>= 3 per SM on 148 SMs)
constexpr size_t kNoAllocDescDoubles = 64;         // one DevMember
constexpr size_t kNoAllocGridDoubles = 2048;       // NGC * G + NBC for G <= GITM_MAX_NALTS + 4
constexpr size_t kNoAllocTileDoubles = size_t(kNoAllocMaxCols) * 2;  // one Tile (16 B) per column at most
constexpr size_t kNoAllocAccDoubles = size_t(kNoAllocSlots) * NF * kNoAllocThreads;
constexpr size_t kNoAllocDoubles =
    kNoAllocDescDoubles + kNoAllocGridDoubles + kNoAllocTileDoubles + kNoAllocAccDoubles;  // 12.3 MiB
static_assert(sizeof(DevMember) <= kNoAllocDescDoubles * sizeof(double), "descriptor slot too small");
static_assert(size_t(NGC) * (GITM_MAX_NALTS + 4) + NBC <= kNoAllocGridDoubles, "grid slot too small");
static_assert(sizeof(Tile) == 2 * sizeof(double), "tile size");

// The shared scratch.  Calls that overlap on the GPU (on different streams,
// or from different host threads) race on it: issue them in order.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];


// Builds the member descriptor, the grid coefficients of the member's
// shared altitude grid (the formulas of grid_coefs above) and the tile list
// in the scratch.  One CTA.
__global__ void noalloc_setup_kernel(GitmColumnBatch b, int nc, int n_tiles, double* base) {
  DevMember* dmem = reinterpret_cast<DevMember*>(base);
  double* gridc = base + kNoAllocDescDoubles;
  Tile* tiles = reinterpret_cast<Tile*>(base + kNoAllocDescDoubles + kNoAllocGridDoubles);
  const int nA = b.n_alts, G = nA + 4;
  if (threadIdx.x == 0) {
    DevMember d;
    memset(&d, 0, sizeof d);
    d.b = b;
    d.gridc = gridc;
    d.gcols = 1;
    d.col_offset = 0;
    *dmem = d;
    double dAF[GITM_MAX_NALTS + 4];
    auto A = [&](int i) { return b.altitude[i + 1]; };
    for (int i = 0; i <= nA + 2; ++i) dAF[i + 1] = A(i) - A(i - 1);
    dAF[0] = dAF[1];
    auto F = [&](int i) { return dAF[i + 1]; };
    for (int g = 0; g < NGC * G + NBC; ++g) gridc[g] = 0.0;
    for (int g = 0; g < G; ++g) {
      const double idf = 1.0 / dAF[g];
      gridc[GC_DALTF * G + g] = dAF[g];
      gridc[GC_H2 * G + g] = idf * 2.0;
      gridc[GC_IDF * G + g] = idf;
      gridc[GC_IDC * G + g] = 1.0 / b.dalt_c[g];
      gridc[GC_GRAV * G + g] = b.gravity[g];
      gridc[GC_INVR * G + g] = b.inv_r[g];
      gridc[GC_R * G + g] = 1.0 / b.inv_r[g];
      gridc[GC_ALT * G + g] = b.altitude[g];
    }
    for (int i = 1; i <= nA; ++i) {
      const double h1 = F(i - 1), h2 = F(i), h3 = F(i + 1), h4 = F(i + 2);
      const double H2 = h2 + h1, H3 = h3 + h2 + h1, H4 = h4 + h3 + h2 + h1;
      gridc[(GC_M0 + 0) * G + i + 1] = (h2 * h3 * (h3 + h4)) / (h1 * H2 * H3 * H4);
      gridc[(GC_M0 + 1) * G + i + 1] = -1.0 * (H2 * h3 * (h3 + h4)) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
      gridc[(GC_M0 + 2) * G + i + 1] =
          (h2 * h3 * (h3 + h4) + H2 * h3 * (h3 + h4) - H2 * h2 * (h3 + h4) - H2 * h2 * h3) /
          (H2 * h2 * h3 * (h3 + h4));
      gridc[(GC_M0 + 3) * G + i + 1] = H2 * h2 * (h4 + h3) / (H3 * (h2 + h3) * h3 * h4);
      gridc[(GC_M0 + 4) * G + i + 1] = -1.0 * H2 * h2 * h3 / (H4 * (h2 + h3 + h4) * (h3 + h4) * h4);
    }
    double* bc = gridc + NGC * G;
    for (int k = 0; k < 2; ++k) {
      const int iAlt = -k;
      const double h1 = F(iAlt + 2), h2 = F(iAlt + 3), h3 = F(iAlt + 4), h4 = F(iAlt + 5);
      const double M1 = h1, M2 = h1 + h2, M3 = h1 + h2 + h3, M4 = h1 + h2 + h3 + h4;
      bc[5 * k + 0] = -1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4);
      bc[5 * k + 1] = 1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
      bc[5 * k + 2] = -1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4));
      bc[5 * k + 3] = 1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4);
      bc[5 * k + 4] = -1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4);
    }
    for (int k = 0; k < 2; ++k) {
      const int iAlt = nA + 1 + k;
      const double h1 = F(iAlt - 1), h2 = F(iAlt - 2), h3 = F(iAlt - 3), h4 = F(iAlt - 4);
      const double M1 = h1, M2 = h1 + h2, M3 = h1 + h2 + h3, M4 = h1 + h2 + h3 + h4;
      bc[10 + 5 * k + 0] = 1.0 * (M2 * M3 * M4 + M1 * M3 * M4 + M1 * M2 * M4 + M1 * M2 * M3) / (M1 * M2 * M3 * M4);
      bc[10 + 5 * k + 1] = -1.0 * (M2 * M3 * M4) / (h1 * h2 * (h2 + h3) * (h2 + h3 + h4));
      bc[10 + 5 * k + 2] = 1.0 * (M1 * M3 * M4) / (M2 * h2 * h3 * (h3 + h4));
      bc[10 + 5 * k + 3] = -1.0 * (M1 * M2 * M4) / (M3 * (h3 + h2) * h3 * h4);
      bc[10 + 5 * k + 4] = 1.0 * (M1 * M2 * M3) / (M4 * (h2 + h3 + h4) * (h3 + h4) * h4);
    }
  }
  for (int t = threadIdx.x; t < n_tiles; t += blockDim.x) {
    Tile tl;
    tl.member = 0;
    tl.c0 = int64_t(t) * nc;
    tl.nc = int(min(int64_t(nc), b.n_cols - tl.c0));
    tiles[t] = tl;
  }
}

}  // namespace

// The device address of g_noalloc_scratch on the current device; called by
// gitm_vert_create with the context's device current.
static cudaError_t noalloc_scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  *out = (e == cudaSuccess) ? static_cast<double*>(p) : nullptr;
  return e;
}

extern "C" int gitm_vert_advance_native_noalloc(GitmVertCtx* ctx, const GitmColumnBatch* member,
                                                double dt, int n_steps, uint32_t* status_words,
                                                void* stream) {
  if (!ctx || !member || !status_words) return set_err(ctx, GITM_ERR_ARG, "ctx, member and status_words are required");
  const GitmColumnBatch& b = *member;
  int rc = check_member(ctx, b, ctx->params);
  if (rc) return rc;
  if (b.grid_per_column)
    return set_err(ctx, GITM_ERR_ARG, "the no-allocation step takes one altitude grid per member (grid_per_column = 0)");
  if (ctx->params.solver != GITM_SOLVER_RUSANOV)
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "the no-allocation step runs the Rusanov solver only");
  if (b.n_cols > kNoAllocMaxCols)
    return set_err(ctx, GITM_ERR_ARG, "n_cols %lld exceeds the no-allocation limit of %lld columns per call",
                   (long long)b.n_cols, (long long)kNoAllocMaxCols);
  if (!(dt > 0.0)) return set_err(ctx, GITM_ERR_ARG, "dt must be > 0");
  if (n_steps < 0) return set_err(ctx, GITM_ERR_ARG, "n_steps < 0");
  if (b.n_cols == 0 || n_steps == 0) return GITM_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  // the kernels read every pointer of the member on the device: host arrays
  // are refused here (pointer queries enqueue no work and allocate nothing)
  const void* ptrs[] = {b.ndensity_s, b.idensity_s, b.rho, b.temperature, b.velocity, b.vert_vel,
                        b.log_ns, b.ndensity, b.gamma, b.mean_major_mass, b.temp_unit, b.cmax,
                        b.ivel_up, b.eddy, b.cos_lat, b.sza, b.mlat, b.lbc, b.altitude, b.gravity,
                        b.dalt_c, b.inv_r, b.heating, b.heating_scale, status_words};
  for (const void* p : ptrs)
    if (!is_device_ptr(p))
      return set_err(ctx, GITM_ERR_ARG, "the no-allocation step takes device pointers only");
  double* base = ctx->noalloc_scratch;
  const int nA = b.n_alts;
  int nc = std::min(kNoAllocThreads / nA, kNoAllocThreads / 32);
  while (nc > 1 && smem_bytes(nA, nc) > ctx->max_smem) --nc;
  nc = std::max(nc, 1);
  const size_t smem = smem_bytes(nA, nc);
  if (smem > ctx->max_smem) return set_err(ctx, GITM_ERR_ARG, "nAlts %d does not fit the no-allocation shape", nA);
  const int n_tiles = int((b.n_cols + nc - 1) / nc);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(ctx, cudaMemsetAsync(status_words, 0, size_t(b.n_cols) * sizeof(uint32_t), st));
  noalloc_setup_kernel<<<1, 128, 0, st>>>(b, nc, n_tiles, base);
  CUDA_TRY(ctx, cudaGetLastError());
  KParams kp{};
  kp.members = reinterpret_cast<const DevMember*>(base);
  kp.tiles = reinterpret_cast<const Tile*>(base + kNoAllocDescDoubles + kNoAllocGridDoubles);
  kp.n_tiles = n_tiles;
  kp.n_steps = n_steps;
  kp.dt = dt;
  kp.status = status_words;
  kp.scratch = base + kNoAllocDescDoubles + kNoAllocGridDoubles + kNoAllocTileDoubles;
  kp.prm = ctx->params;
  void* args[] = {&kp};
  // CTA x keeps its RK accumulators at scratch + x * NF * kNoAllocThreads:
  // the grid never exceeds the kNoAllocSlots slots kNoAllocAccDoubles holds
  const int grid = std::min(n_tiles, kNoAllocSlots);
  CUDA_TRY(ctx, cudaLaunchKernel(kernel_for(0, GITM_SOLVER_RUSANOV, kNoAllocThreads), dim3(grid),
                                 dim3(kNoAllocThreads), args, smem, st));
  return GITM_OK;
}

// ------------------------------------------------------------------ horizontal advance
// gitm_hz_advance / gitm_hz_status (include/gitm_hz.h): advance_horizontal
// (advance_horizontal.f90:58-924) for every block of GITM's own device
// arrays; the kernel is in hz_kernel.cu.
extern "C" int gitm_hz_advance(GitmVertCtx* ctx, const GitmHzParams* params, const GitmHzBlocks* blocks, double dt,
                               void* stream) {
  if (!ctx || !params || !blocks) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  const GitmHzBlocks& b = *blocks;
  if (b.n_lons < 1 || b.n_lats < 1 || b.n_alts < 1 || b.n_blocks < 0)
    return set_err(ctx, GITM_ERR_ARG, "bad block shape %d x %d x %d, %d blocks", b.n_lons, b.n_lats, b.n_alts,
                   b.n_blocks);
  if (hz_threads(b.n_lons, b.n_lats) == 0)
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "blocks of %d x %d cells: at most 256 cells per block are built",
                   b.n_lons, b.n_lats);
  if (int64_t(b.n_blocks) * b.n_alts > int64_t(0x7fffffff))
    return set_err(ctx, GITM_ERR_ARG, "too many (block, altitude) planes");
  if (!(dt > 0.0)) return set_err(ctx, GITM_ERR_ARG, "dt must be > 0");
  if (!(params->beta_limiter >= 1.0 && params->beta_limiter <= 2.0))
    return set_err(ctx, GITM_ERR_ARG, "beta_limiter %g outside [1, 2]", params->beta_limiter);
  const bool div = params->use_ion_advection && params->use_improved_ion_advection;
  const void* req[] = {b.rho, b.temperature, b.velocity, b.vert_vel, b.ndensity_s, b.idensity_s, b.gamma, b.cmax,
                       b.ivelocity, b.latitude, b.tan_latitude, b.cos_latitude, b.radial_distance,
                       b.inv_radial_distance, b.inv_dlon_dist_gb, b.inv_dlon_dist_fb, b.dlon_dist_fb,
                       b.inv_dlat_dist_gb, b.inv_dlat_dist_fb, b.dlat_dist_fb};
  for (const void* p : req)
    if (!p || !is_device_ptr(p)) return set_err(ctx, GITM_ERR_ARG, "the block arrays must be non-NULL device pointers");
  if (div) {
    const void* dreq[] = {params->non_magnetic ? (const void*)b.ivelocity : (const void*)b.ivelocity_par,
                          b.grad_lon_m, b.grad_lon_0, b.grad_lon_p, b.grad_lat_m, b.grad_lat_0, b.grad_lat_p};
    for (const void* p : dreq)
      if (!p || !is_device_ptr(p))
        return set_err(ctx, GITM_ERR_ARG, "the ion-divergence term needs IVelocityPar and the GradLon/GradLat arrays");
  }
  if (!is_device_ptr(b.temp_source)) return set_err(ctx, GITM_ERR_ARG, "temp_source must be a device pointer");
  if (b.n_blocks == 0) return GITM_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (ctx->hz_status_n < b.n_blocks) {
    cudaFree(ctx->hz_status);
    ctx->hz_status = nullptr;
    ctx->hz_status_n = 0;
    if (cudaMalloc(&ctx->hz_status, size_t(b.n_blocks) * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, GITM_ERR_NOMEM, "cannot allocate the block status words");
    }
    ctx->hz_status_n = b.n_blocks;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->hz_status, 0, size_t(b.n_blocks) * sizeof(uint32_t), st));
  const size_t smem = hz_smem_bytes(b.n_lons, b.n_lats);
  if (smem > ctx->max_smem) return set_err(ctx, GITM_ERR_UNSUPPORTED, "block plane needs %zu bytes of shared memory", smem);
  cudaError_t e = hz_launch(*params, b, dt, ctx->hz_status, st);
  if (e != cudaSuccess) return set_err(ctx, GITM_ERR_CUDA, "hz launch: %s", cudaGetErrorString(e));
  ctx->hz_blocks = b.n_blocks;
  ctx->hz_stream = st;
  return GITM_OK;
}

extern "C" int gitm_hz_exchange(GitmVertCtx* ctx, const GitmHzExchange* x, void* stream) {
  if (!ctx || !x) return set_err(ctx, GITM_ERR_ARG, "bad arguments");
  if (x->n_lons < 2 || x->n_lats < 2 || x->n_alts < 1 || x->n_blocks_lon < 1 || x->n_blocks_lat < 1)
    return set_err(ctx, GITM_ERR_ARG, "bad block grid (the two-cell ghost ring needs blocks of 2 x 2 cells or more)");
  if ((x->north_pole || x->south_pole) && (x->n_blocks_lon % 2 != 0))
    return set_err(ctx, GITM_ERR_UNSUPPORTED, "a pole connection needs an even number of blocks in longitude");
  const int64_t nb = int64_t(x->n_blocks_lon) * x->n_blocks_lat;
  if (nb * x->n_alts > int64_t(0x7fffffff)) return set_err(ctx, GITM_ERR_ARG, "too many (block, altitude) planes");
  const void* req[] = {x->rho, x->temperature, x->velocity, x->vert_vel, x->ndensity_s, x->latitude,
                       x->non_magnetic ? x->ivelocity : x->ivelocity_par};
  for (const void* p : req)
    if (!p || !is_device_ptr(p)) return set_err(ctx, GITM_ERR_ARG, "the exchanged arrays must be non-NULL device pointers");
  if (x->use_ion_advection && (!x->idensity_s || !is_device_ptr(x->idensity_s)))
    return set_err(ctx, GITM_ERR_ARG, "use_ion_advection needs IDensityS");
  if (!is_device_ptr(x->itemperature) || !is_device_ptr(x->etemperature))
    return set_err(ctx, GITM_ERR_ARG, "itemperature / etemperature must be device pointers or NULL");
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (ctx->hz_status_n < nb) {
    cudaFree(ctx->hz_status);
    ctx->hz_status = nullptr;
    ctx->hz_status_n = 0;
    if (cudaMalloc(&ctx->hz_status, size_t(nb) * sizeof(uint32_t)) != cudaSuccess) {
      cudaGetLastError();
      return set_err(ctx, GITM_ERR_NOMEM, "cannot allocate the block status words");
    }
    ctx->hz_status_n = nb;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CUDA_TRY(ctx, cudaMemsetAsync(ctx->hz_status, 0, size_t(nb) * sizeof(uint32_t), st));
  cudaError_t e = hz_exchange_launch(*x, ctx->hz_status, st);
  if (e != cudaSuccess) return set_err(ctx, GITM_ERR_CUDA, "hz exchange launch: %s", cudaGetErrorString(e));
  ctx->hz_blocks = nb;
  ctx->hz_stream = st;
  return GITM_OK;
}

extern "C" int gitm_hz_status(GitmVertCtx* ctx, uint32_t* or_out, int64_t* n_bad, int clear) {
  if (!ctx) return GITM_ERR_ARG;
  if (or_out) *or_out = 0;
  if (n_bad) *n_bad = 0;
  if (ctx->hz_blocks == 0) return GITM_OK;
  CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  CUDA_TRY(ctx, cudaStreamSynchronize(ctx->hz_stream));
  std::vector<uint32_t> w(size_t(ctx->hz_blocks));
  CUDA_TRY(ctx, cudaMemcpy(w.data(), ctx->hz_status, w.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  uint32_t acc = 0;
  int64_t nb = 0;
  for (uint32_t x : w) {
    acc |= x;
    nb += (x != 0);
  }
  if (or_out) *or_out = acc;
  if (n_bad) *n_bad = nb;
  if (clear) CUDA_TRY(ctx, cudaMemset(ctx->hz_status, 0, w.size() * sizeof(uint32_t)));
  return GITM_OK;
}
