// pcl_mixed.h -- the mixed-precision precision form (kernels_mixed.cu).
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {
int mixed_create(const GridDev& g, cudaStream_t st, void** ws);
void mixed_free(void* ws);
void mixed_set_tile_rows(void* ws, int ty);   // rows per work item of the fused kernel
// test of the timeout path: the bulk copy of `row` is not issued and waits give up after
// `probes` probes (row < 0: off)
void mixed_set_injection(void* ws, int row, unsigned probes);
void launch_sweeps_mixed(const GridDev& g, void* ws, cudaStream_t st);
// one whole attempt of the device loop in one launch: the fused sweeps, then the time control
// and the ghost fill by the CTAs (no host hook may run in between)
void launch_step_mixed(const GridDev& g, void* ws, cudaStream_t st);
bool mixed_injection_on(const void* ws);   // a copy stall is injected (the test build runs)
}  // namespace pcl
