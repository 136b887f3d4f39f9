// batch_mixed.cu -- the precision form for a batch of grids in one persistent launch.
//
// CTAs (128 threads) pull fused work items (instance, strip, row segment) from a queue and run
// them with the single-grid item body (pcl_stream_mixed.cuh); the shared-memory row ring and its
// mbarriers are set up once per CTA and carried across items.  The CTA that finishes an
// instance's last item runs that instance's time control and ghost fill.  A batched instance is
// bit-identical to the same grid run alone: no cell's arithmetic depends on the schedule.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <vector>

#include "pcl_batch.h"
#include "pcl_ghost.cuh"
#include "pcl_stream_mixed.cuh"
#include "pcl_timectl.cuh"

namespace pcl {

__constant__ ItemDesc c_desc[kDescPool];

namespace {

using mixed::NT;
using mixed::Smem;

template <class G>
__device__ __forceinline__ void dispatch_item(const G& g, int mode, int strip, int seg, int ty, Smem& S,
                                              unsigned& rows) {
  switch (mode) {
    case 0: mixed::mixed_item<0, false>(g, strip, seg, ty, S, rows); break;
    case 2: mixed::mixed_item<1, true>(g, strip, seg, ty, S, rows); break;
    case 3: mixed::mixed_item<2, true>(g, strip, seg, ty, S, rows); break;
    case 4: mixed::mixed_item<3, true>(g, strip, seg, ty, S, rows); break;
    case 5: mixed::mixed_item<4, true>(g, strip, seg, ty, S, rows); break;
    default: mixed::mixed_item<0, true>(g, strip, seg, ty, S, rows); break;
  }
}

// One mode only: the row loop unrolled by two, as in the single-grid kernel (it still fits five
// CTAs per SM when the kernel holds one item body instead of six).
template <int MODE, class G>
__device__ __forceinline__ void mode_item(const G& g, int strip, int seg, int ty, Smem& S, unsigned& rows) {
  if (MODE == 0) mixed::mixed_item<0, false, 2>(g, strip, seg, ty, S, rows);
  else if (MODE == 1) mixed::mixed_item<0, true, 2>(g, strip, seg, ty, S, rows);
  else mixed::mixed_item<(MODE >= 2 ? MODE - 1 : 0), true, 2>(g, strip, seg, ty, S, rows);
}

__device__ __forceinline__ int item_mode(const GridDev& g) { return g.second_order ? 1 + g.limiter : 0; }

// POOL: the item's descriptor is read from the constant pool (c_desc[v.desc_base + slot]);
// otherwise from v.inst.  MODE >= 0: every instance of the batch has that mode (built for it
// alone); -1: any mix of modes.  The finishing CTA reads the instance's full GridDev from v.inst.
template <bool POOL, int MODE>
__global__ void __launch_bounds__(NT, POOL ? 5 : 4) batch_mixed_kernel(BatchView v) {
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
    Ctl* ctl;
    if (POOL) {
      const ItemDesc& d = c_desc[v.desc_base + w.x];
      ctl = d.ctl;
      if (!ctl->done) {
        if (MODE >= 0)
          mode_item<MODE>(d, w.z, w.w, v.tile_rows, S, rows);
        else
          dispatch_item(d, d.mode, w.z, w.w, v.tile_rows, S, rows);
      }
    } else {
      const GridDev g = v.inst[w.x];
      ctl = g.ctl;
      if (!ctl->done) dispatch_item(g, item_mode(g), w.z, w.w, v.tile_rows, S, rows);
    }
    int* alldone = v.counters + 2 * w.x + 1;
    __threadfence();  // every thread's writes of this item precede its completion count
    __syncthreads();
    if (threadIdx.x == 0) {
      s_last = atomicAdd(alldone, 1) + 1 == v.totals[2 * w.x + 1];
      if (s_last) {
        __threadfence();
        full_step(ctl, v.inst[w.x]);  // CFL, accept/reject, updateTime, snapshot, reset_CFL, log
        *alldone = 0;
        __threadfence();
      }
    }
    __syncthreads();
    if (s_last && ctl->ierr == 1) {  // update_rank_boundaries of the accepted instance
      const GridDev& g = v.inst[w.x];
      double* b = buffer(g, ctl->cur);
      const int ng = ghost_items(g);
      for (int k = threadIdx.x; k < ng; k += blockDim.x) ghost_item(g, b, k);
    }
    __syncthreads();
  }
}

using KernelFn = void (*)(BatchView);

// the build for (pool, mode); mode -1 or out of range: any mix of modes
KernelFn kernel_for(bool pool, int mode) {
  if (!pool) return batch_mixed_kernel<false, -1>;
  switch (mode) {
    case 0: return batch_mixed_kernel<true, 0>;
    case 1: return batch_mixed_kernel<true, 1>;
    case 2: return batch_mixed_kernel<true, 2>;
    case 3: return batch_mixed_kernel<true, 3>;
    case 4: return batch_mixed_kernel<true, 4>;
    case 5: return batch_mixed_kernel<true, 5>;
    default: return batch_mixed_kernel<true, -1>;
  }
}

// pool reservations per device: used[d][k] for descriptor k
std::mutex g_pool_mu;
std::map<int, std::vector<char>> g_pool_used;

}  // namespace

void launch_batch_mixed(const BatchView& v, int grid, bool pool, int mode, cudaStream_t st) {
  kernel_for(pool, mode)<<<grid, NT, 0, st>>>(v);
}
int batch_mixed_threads() { return NT; }
int batch_mixed_occupancy(bool pool, int mode) {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_for(pool, mode), NT, 0);
  return n > 0 ? n : 1;
}

cudaError_t batch_mixed_set_desc(int index, const ItemDesc& d, cudaStream_t st) {
  if (index < 0 || index >= kDescPool) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbolAsync(c_desc, &d, sizeof(ItemDesc), sizeof(ItemDesc) * (size_t)index,
                                 cudaMemcpyHostToDevice, st);
}

int batch_desc_reserve(int n) {
  int dev = 0;
  if (n < 1 || n > kDescPool || cudaGetDevice(&dev) != cudaSuccess) return -1;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto& used = g_pool_used[dev];
  if (used.empty()) used.assign(kDescPool, 0);
  for (int base = 0; base + n <= kDescPool; ++base) {
    int k = 0;
    while (k < n && !used[base + k]) ++k;
    if (k == n) {
      for (k = 0; k < n; ++k) used[base + k] = 1;
      return base;
    }
    base += k;  // skip past the used entry
  }
  return -1;
}

void batch_desc_release(int base, int n) {
  int dev = 0;
  if (base < 0 || cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  auto& used = g_pool_used[dev];
  for (int k = base; k < base + n && k < (int)used.size(); ++k) used[k] = 0;
}

}  // namespace pcl
