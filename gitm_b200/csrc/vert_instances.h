// vert_instances.h -- the step-kernel instantiations the library is built with.
//
// X(id, IO, NT, MINB, ACC_GLOBAL, SOLVER, SAVE, NA, OG): vert_step_kernel<IO,
// NT, MINB, ACC_GLOBAL, SOLVER, SAVE, NA, OG> (vert_kernel.cuh).  Each entry is compiled
// in a translation unit of its own (vert_instance.cu, built once per entry
// with -DGV_ID=id -DGV_IO=... by gitm_b200/build.py, which reads this list):
// instantiated side by side in one unit, the compiler kept arrays of the
// shared device functions (the friction matrix, ColCtx copies) in a 400- to
// 700-byte local-memory frame in most of them; alone, each compiles with
// little or none.  Every unit has its own copy of the constant table c_k,
// set through step_consts_<id> when a context is created.
//
// SOLVER: 0 Rusanov, 1 AUSM.  IO: 0 GITM arrays, 1 ModVertical arrays.
// NA: 0 = nAlts read from the member at run time; NA > 0 = an instance for
// members of exactly that nAlts (GITM's default 50), whose shared-memory
// offsets and loop bounds are compile-time constants; the host launches it
// when every member of a plan has that nAlts.  OG: Orig in global scratch
// (the 512-thread shape: 8 columns of 50 altitudes, 16 warps per SM at 128
// registers).
#pragma once

#include "vert_common.cuh"

#define GV_STEP_INSTANCES(X)                                  \
  X(rus0_t128, 0, 128, 3, true, 0, false, 0, false)           \
  X(rus0_t160, 0, 160, 2, true, 0, false, 0, false)           \
  X(rus0_t192, 0, 192, 2, true, 0, false, 0, false)           \
  X(rus0_t256, 0, 256, 1, false, 0, false, 0, false)          \
  X(rus0_t320, 0, 320, 1, false, 0, false, 0, false)          \
  X(rus0_t384, 0, 384, 1, false, 0, false, 0, false)          \
  X(rus1_t128, 1, 128, 3, true, 0, false, 0, false)           \
  X(rus1_t160, 1, 160, 2, true, 0, false, 0, false)           \
  X(rus1_t192, 1, 192, 2, true, 0, false, 0, false)           \
  X(rus1_t256, 1, 256, 1, false, 0, false, 0, false)          \
  X(rus1_t320, 1, 320, 1, false, 0, false, 0, false)          \
  X(rus1_t384, 1, 384, 1, false, 0, false, 0, false)          \
  X(ausm0_t128, 0, 128, 2, true, 1, false, 0, false)          \
  X(ausm0_t256, 0, 256, 1, false, 1, false, 0, false)         \
  X(ausm1_t128, 1, 128, 2, true, 1, false, 0, false)          \
  X(ausm1_t256, 1, 256, 1, false, 1, false, 0, false)         \
  X(rus0_t128_save, 0, 128, 3, true, 0, true, 0, false)       \
  X(rus0_t128_n50, 0, 128, 3, true, 0, false, 50, false)      \
  X(rus0_t192_n50, 0, 192, 2, true, 0, false, 50, false)      \
  X(rus0_t256_n50, 0, 256, 1, false, 0, false, 50, false)     \
  X(rus0_t384_n50, 0, 384, 1, false, 0, false, 50, false)     \
  X(ausm0_t128_n50, 0, 128, 2, true, 1, false, 50, false)     \
  X(ausm0_t256_n50, 0, 256, 1, false, 1, false, 50, false)    \
  X(rus0_t128_save_n50, 0, 128, 3, true, 0, true, 50, false)  \
  X(rus0_t512_og, 0, 512, 1, true, 0, false, 0, true)         \
  X(rus0_t512_og_n50, 0, 512, 1, true, 0, false, 50, true)    \
  X(ausm0_t384_og_n50, 0, 384, 1, true, 1, false, 50, true)

namespace gv {
#define GV_DECLARE_INSTANCE(id, IO, NT, MINB, ACC, SOLVER, SAVE, NA, OG) \
  const void* step_kernel_##id();                                \
  cudaError_t step_consts_##id(const Consts& k);
GV_STEP_INSTANCES(GV_DECLARE_INSTANCE)
#undef GV_DECLARE_INSTANCE
}  // namespace gv
