// pcl_batch.h -- device-side view of a batch of independent grids (instances) advanced by one
// persistent kernel launch per attempted step.
//
// Work items (int4 {slot, kind, a, b}), read from device memory so the batch can change between
// launches without re-capturing the CUDA graph:
//   kind kItemX     FP64 xi sweep of rows a .. a+rows-1 of the segment starting at column b
//   kind kItemY     FP64 eta sweep of the columns from a, strip of rows from b
//   kind kItemMixed mixed-precision fused item: strip a, row segment b
// Per instance, counters[2*slot] counts finished xi items (eta items of that instance wait for
// all of them) and counters[2*slot+1] all finished items; the CTA that finishes the last item
// runs the instance's time control and ghost fill and clears both counters.
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {

enum : int { kItemX = 0, kItemY = 1, kItemMixed = 2 };

struct BatchView {
  const GridDev* inst;   // [max_slots]
  const int4* items;     // [n_items]
  const int* n_items;    // device scalar
  unsigned* head;        // device scalar: the work queue head (zeroed before each launch)
  int* counters;         // [2*max_slots]
  const int* totals;     // [2*max_slots]: xi items, all items of each slot this step
  int x_rows;            // rows per FP64 xi item
  int y_rows;            // rows per FP64 eta strip
  int tile_rows;         // rows per mixed item
  unsigned spin_limit;   // bounded waits of eta items for their xi items
};

void launch_batch_fp64(const BatchView& v, int grid, cudaStream_t st);
void launch_batch_mixed(const BatchView& v, int grid, cudaStream_t st);
int batch_fp64_threads();   // also the columns of an FP64 eta item
int batch_fp64_segment();   // cells of an FP64 xi item's row segment
int batch_mixed_threads();
// largest number of resident CTAs per SM of each persistent kernel
int batch_fp64_occupancy();
int batch_mixed_occupancy();

}  // namespace pcl
