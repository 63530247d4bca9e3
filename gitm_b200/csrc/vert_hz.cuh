// vert_hz.cuh -- host-side entry of the horizontal-advance kernel
// (hz_kernel.cu, its own translation unit).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/gitm_hz.h"

namespace gv {

// Dynamic shared memory of one (block, altitude) plane.
size_t hz_smem_bytes(int n_lons, int n_lats);
// Threads per CTA for blocks of n_lons x n_lats cells; 0 when none is built.
int hz_threads(int n_lons, int n_lats);
// One advance_horizontal for every block; status: one word per block.
cudaError_t hz_launch(const GitmHzParams& prm, const GitmHzBlocks& b, double dt, uint32_t* status,
                      cudaStream_t stream);
// exchange_messages_sphere over every (block, altitude) plane.
cudaError_t hz_exchange_launch(const GitmHzExchange& x, uint32_t* status, cudaStream_t stream);

}  // namespace gv
