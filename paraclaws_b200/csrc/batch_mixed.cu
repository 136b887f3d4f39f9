// batch_mixed.cu -- the precision form for a batch of grids in one persistent launch.
//
// CTAs (128 threads) pull fused work items (instance, strip, row segment) from a queue and run
// them with the single-grid item body (pcl_stream_mixed.cuh); the shared-memory row ring and its
// mbarriers are set up once per CTA and carried across items.  The CTA that finishes an
// instance's last item runs that instance's time control and ghost fill.  A batched instance is
// bit-identical to the same grid run alone: no cell's arithmetic depends on the schedule.
#include <cuda_runtime.h>

#include "pcl_batch.h"
#include "pcl_ghost.cuh"
#include "pcl_stream_mixed.cuh"
#include "pcl_timectl.cuh"

namespace pcl {
namespace {

using mixed::NT;
using mixed::Smem;

__device__ __forceinline__ void dispatch_item(const GridDev& g, int strip, int seg, int ty, Smem& S, unsigned& rows) {
  if (!g.second_order) {
    mixed::mixed_item<0, false>(g, strip, seg, ty, S, rows);
    return;
  }
  switch (g.limiter) {
    case 1: mixed::mixed_item<1, true>(g, strip, seg, ty, S, rows); break;
    case 2: mixed::mixed_item<2, true>(g, strip, seg, ty, S, rows); break;
    case 3: mixed::mixed_item<3, true>(g, strip, seg, ty, S, rows); break;
    case 4: mixed::mixed_item<4, true>(g, strip, seg, ty, S, rows); break;
    default: mixed::mixed_item<0, true>(g, strip, seg, ty, S, rows); break;
  }
}

__global__ void __launch_bounds__(NT) batch_mixed_kernel(BatchView v) {
  __shared__ Smem S;
  __shared__ int s_item;
  __shared__ int s_last;
  mixed::init_ring(S);
  unsigned rows = 0;
  const int n = *v.n_items;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(v.head, 1u);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= n) break;
    const int4 w = v.items[it];
    const GridDev g = v.inst[w.x];
    Ctl* ctl = g.ctl;
    int* alldone = v.counters + 2 * w.x + 1;
    if (!ctl->done) dispatch_item(g, w.z, w.w, v.tile_rows, S, rows);
    __threadfence();  // every thread's writes of this item precede its completion count
    __syncthreads();
    if (threadIdx.x == 0) {
      s_last = atomicAdd(alldone, 1) + 1 == v.totals[2 * w.x + 1];
      if (s_last) {
        __threadfence();
        full_step(ctl, g);  // CFL, accept/reject, updateTime, snapshot, reset_CFL, log
        *alldone = 0;
        __threadfence();
      }
    }
    __syncthreads();
    if (s_last && ctl->ierr == 1) {  // update_rank_boundaries of the accepted instance
      double* b = buffer(g, ctl->cur);
      const int ng = ghost_items(g);
      for (int k = threadIdx.x; k < ng; k += blockDim.x) ghost_item(g, b, k);
    }
    __syncthreads();
  }
}

}  // namespace

void launch_batch_mixed(const BatchView& v, int grid, cudaStream_t st) {
  batch_mixed_kernel<<<grid, NT, 0, st>>>(v);
}
int batch_mixed_threads() { return NT; }
int batch_mixed_occupancy() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_mixed_kernel, NT, 0);
  return n > 0 ? n : 1;
}

}  // namespace pcl
