// vert_adjoint.cu -- translation unit of the adjoint kernel.
//
// The adjoint kernel shares device functions with the forward step kernel
// (rusanov_cell, bc_column, friction_solve, ...).  Compiled in the same
// translation unit, its instantiation changes how those functions are
// compiled into the forward kernel (a 400-byte local-memory frame and a
// slower step), so it is built here, apart, as every step kernel is.
// Without relocatable device code this unit has its own copy of the
// constant table c_k, which the host sets through adjoint_set_consts when a
// context is created.  Built twice: as is (any nAlts) and with
// -DGV_ADJ_NA=50 (the instance for members of 50 altitudes, in a unit of
// its own for the same reason).
#include "vert_common.cuh"
#include "vert_kernel.cuh"
#include "vert_adjoint.cuh"
#include "vert_instances.h"

namespace gv {

#if !defined(GV_ADJ_NA) || GV_ADJ_NA == 0
const void* adjoint_kernel_fn() { return (const void*)vert_adjoint_kernel<ADJ_THREADS>; }

cudaError_t adjoint_set_consts(const Consts& k) { return cudaMemcpyToSymbol(c_k, &k, sizeof k); }
#elif GV_ADJ_NA == 50
const void* adjoint_kernel_fn_n50() { return (const void*)vert_adjoint_kernel<ADJ_THREADS, 50>; }

cudaError_t adjoint_set_consts_n50(const Consts& k) { return cudaMemcpyToSymbol(c_k, &k, sizeof k); }
#else
#error "vert_adjoint.cu: GV_ADJ_NA is 0 or 50"
#endif

}  // namespace gv
