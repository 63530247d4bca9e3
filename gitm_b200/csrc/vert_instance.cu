// vert_instance.cu -- one step-kernel instantiation per translation unit.
//
// Built once for every entry of GV_STEP_INSTANCES (vert_instances.h) with
// -DGV_ID=<id> -DGV_IO=... -DGV_NT=... -DGV_MINB=... -DGV_ACC=...
// -DGV_SOLVER=... -DGV_SAVE=... -DGV_NA=... -DGV_OG=...; exports the kernel's address and the setter
// of this unit's copy of the constant table.
#include "vert_common.cuh"
#include "vert_kernel.cuh"
#include "vert_instances.h"

#if !defined(GV_ID) || !defined(GV_IO) || !defined(GV_NT) || !defined(GV_MINB) || !defined(GV_ACC) || \
    !defined(GV_SOLVER) || !defined(GV_SAVE) || !defined(GV_NA) || !defined(GV_OG)
#error "vert_instance.cu is built once per GV_STEP_INSTANCES entry with its -DGV_* values"
#endif

#define GV_CAT2(a, b) a##b
#define GV_CAT(a, b) GV_CAT2(a, b)

namespace gv {

const void* GV_CAT(step_kernel_, GV_ID)() {
  return (const void*)vert_step_kernel<GV_IO, GV_NT, GV_MINB, GV_ACC, GV_SOLVER, GV_SAVE, GV_NA, GV_OG>;
}

cudaError_t GV_CAT(step_consts_, GV_ID)(const Consts& k) { return cudaMemcpyToSymbol(c_k, &k, sizeof k); }

}  // namespace gv
