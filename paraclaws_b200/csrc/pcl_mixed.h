// pcl_mixed.h -- the mixed-precision precision form (kernels_mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {
int mixed_create(const GridDev& g, cudaStream_t st, void** ws);
void mixed_free(void* ws);
void mixed_set_tile_rows(void* ws, int ty);   // rows per work item of the fused kernel
void launch_sweeps_mixed(const GridDev& g, void* ws, cudaStream_t st);
}  // namespace pcl
