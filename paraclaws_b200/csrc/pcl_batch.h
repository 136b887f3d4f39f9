// pcl_batch.h -- device-side view of a batch of independent grids (instances) advanced by one
// persistent kernel launch per attempted step.
//
// Work items (int4 {slot, kind, a, b}), read from device memory so the batch can change between
// launches without re-capturing the CUDA graph:
//   kind kItemX     FP64 xi sweep of rows a .. a+rows-1 of the segment starting at column b
//   kind kItemY     FP64 eta sweep of the 4-column band from column a (-1 + 4k), rows b ..
//                   b+rows-1
//   kind kItemMixed mixed-precision fused item: strip a, row segment b
// Per instance, counters[2*slot] counts finished xi items (eta items of that instance wait for
// all of them) and counters[2*slot+1] all finished items; the CTA that finishes the last item
// runs the instance's time control and ghost fill and clears both counters.
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {

enum : int { kItemX = 0, kItemY = 1, kItemMixed = 2 };

// The fields of GridDev one mixed item reads.  A batch that owns a range of the constant-memory
// pool keeps its instances' descriptors there: loads from the constant bank can be repeated
// instead of held in registers, so the persistent kernel fits five CTAs per SM.
struct ItemDesc {
  double* state;
  long long bufstride, plane;
  Ctl* ctl;
  double grav;
  int mx, my, pitch;
  int mode;  // 0: first order; else 1 + limiter (0: unlimited correction, 1..4 by code)
};
constexpr int kDescPool = 1024;  // descriptors in the pool (56 KB of constant memory)

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
  int desc_base;         // first pool descriptor of this batch (mixed, pool build only)
  int item_ghosts;       // 1: the builds whose edge items fill ghost cells, 0: the builds
                         // whose finishing CTA fills them all
  unsigned spin_limit;   // bounded waits of eta items for their xi items
  int* flags;            // device scalar: bit 0 set when any bounded wait of the launch gave up
  int stall_slot;        // test of the timeout path (-1: off): the eta items of this slot wait
                         // for one xi item more than the step has, so their wait runs out
  int fast_div;          // FP64: every instance's g is inside the shared-reciprocal range
};

void launch_batch_fp64(const BatchView& v, int grid, cudaStream_t st);
// pool = true: item descriptors from the constant pool at v.desc_base (the builds for five CTAs
// per SM); false: from v.inst in global memory.  mode 0..5 (ItemDesc::mode): every instance has
// that mode and the pool build specialised for it runs; -1: any mix.
void launch_batch_mixed(const BatchView& v, int grid, bool pool, int mode, cudaStream_t st);
// copy one descriptor into the pool (stream-ordered with the launches)
cudaError_t batch_mixed_set_desc(int index, const ItemDesc& d, cudaStream_t st);
// reserve n consecutive pool descriptors on the current device: the first index, or -1 if
// there is no room; release them again
int batch_desc_reserve(int n);
void batch_desc_release(int base, int n);
int batch_fp64_threads();
int batch_fp64_segment();   // cells of an FP64 xi item's row segment
int batch_fp64_band();      // columns of an FP64 eta item's band
int batch_mixed_threads();
// largest number of resident CTAs per SM of each persistent kernel
int batch_fp64_occupancy();
int batch_mixed_occupancy(bool pool, int mode);

}  // namespace pcl
