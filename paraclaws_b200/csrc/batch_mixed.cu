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

// Each returns false when a bounded wait of the item gave up (mixed_item).
template <class G>
__device__ __forceinline__ bool dispatch_item(const G& g, int mode, int strip, int seg, int ty, Smem& S,
                                              unsigned& rows) {
  switch (mode) {
    case 0: return mixed::mixed_item<0, false>(g, strip, seg, ty, S, rows);
    case 2: return mixed::mixed_item<1, true>(g, strip, seg, ty, S, rows);
    case 3: return mixed::mixed_item<2, true>(g, strip, seg, ty, S, rows);
    case 4: return mixed::mixed_item<3, true>(g, strip, seg, ty, S, rows);
    case 5: return mixed::mixed_item<4, true>(g, strip, seg, ty, S, rows);
    default: return mixed::mixed_item<0, true>(g, strip, seg, ty, S, rows);
  }
}

// One mode only: the row loop unrolled by two, as in the single-grid kernel (it still fits five
// CTAs per SM when the kernel holds one item body instead of six).
template <int MODE, class G>
__device__ __forceinline__ bool mode_item(const G& g, int strip, int seg, int ty, Smem& S, unsigned& rows) {
  if (MODE == 0) return mixed::mixed_item<0, false, 2>(g, strip, seg, ty, S, rows);
  if (MODE == 1) return mixed::mixed_item<0, true, 2>(g, strip, seg, ty, S, rows);
  return mixed::mixed_item<(MODE >= 2 ? MODE - 1 : 0), true, 2>(g, strip, seg, ty, S, rows);
}

__device__ __forceinline__ int item_mode(const GridDev& g) { return g.second_order ? 1 + g.limiter : 0; }

// Ghost cells (update_rank_boundaries) filled by the items themselves, when the batch is small
// enough that its step time is a few items' latency (the IG builds; with many items the
// finishing CTA's fill overlaps other CTAs' items and costs less).  Same values either way:
// an edge item fills the ghosts next to the cells it wrote (ghost_fill_block), into the step's
// output buffer, before its completion count.
__device__ __forceinline__ void item_ghosts(const GridDev& g, int strip, int seg, int ty) {
  const int cur = g.ctl->cur;
  const int i0 = 1 + strip * mixed::TXI, j0 = 1 + seg * ty;
  ghost_fill_block(g, buffer(g, cur == 0 ? 2 : cur - 1), i0, min(i0 + mixed::TXI - 1, g.mx), j0,
                   min(j0 + ty - 1, g.my));
}

// The sides item_ghosts leaves open, after an accepted step (b: the new current buffer).
__device__ __forceinline__ void finisher_ghosts(const GridDev& g, int ty, double* b) {
  ghost_fill_open_sides(g, b, (g.mx - 1) % mixed::TXI == 0, (g.my - 1) % ty == 0);
}

// True for an item on the edge of its grid (first or last strip or segment): only those write
// ghost cells, and the rest skip item_ghosts without reading the grid's descriptor.
__device__ __forceinline__ bool edge_item(int mx, int my, int strip, int seg, int ty) {
  return strip == 0 || seg == 0 || (strip + 1) * mixed::TXI >= mx || (seg + 1) * ty >= my;
}

// POOL: the item's descriptor is read from the constant pool (c_desc[v.desc_base + slot]);
// otherwise from v.inst.  MODE >= 0: every instance of the batch has that mode (built for it
// alone); -1: any mix of modes.  IG: edge items fill the ghost cells (item_ghosts), else the
// finishing CTA fills them all; separate builds, so the item loop of the IG = false builds is
// compiled without the ghost code.  The finishing CTA reads the instance's GridDev from v.inst.
template <bool POOL, int MODE, bool IG>
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
    bool ok = true;
    if (POOL) {
      const ItemDesc& d = c_desc[v.desc_base + w.x];
      ctl = d.ctl;
      if (!ctl->done) {
        if (MODE >= 0)
          ok = mode_item<MODE>(d, w.z, w.w, v.tile_rows, S, rows);
        else
          ok = dispatch_item(d, d.mode, w.z, w.w, v.tile_rows, S, rows);
        if (ok && IG && edge_item(d.mx, d.my, w.z, w.w, v.tile_rows))
          item_ghosts(v.inst[w.x], w.z, w.w, v.tile_rows);
      }
    } else {
      const GridDev g = v.inst[w.x];
      ctl = g.ctl;
      if (!ctl->done) {
        ok = dispatch_item(g, item_mode(g), w.z, w.w, v.tile_rows, S, rows);
        if (ok && IG && edge_item(g.mx, g.my, w.z, w.w, v.tile_rows)) item_ghosts(g, w.z, w.w, v.tile_rows);
      }
    }
    if (!ok && threadIdx.x == 0) atomicOr(v.flags, 1);
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
    if (s_last && ctl->ierr == 1) {  // update_rank_boundaries (the rest of it after item_ghosts)
      const GridDev& g = v.inst[w.x];
      double* b = buffer(g, ctl->cur);
      if (IG) {
        finisher_ghosts(g, v.tile_rows, b);
      } else {
        const int ng = ghost_items(g);
        for (int k = threadIdx.x; k < ng; k += blockDim.x) ghost_item(g, b, k);
      }
    }
    __syncthreads();
    // After a wait gave up, this CTA's row ring is out of phase: it takes no further items (the
    // queue hands them to the other CTAs; the item was counted, so its instance still finishes
    // the step, as a void attempt).
    if (!ok) break;
  }
}

using KernelFn = void (*)(BatchView);

template <bool IG>
KernelFn kernel_for_ig(bool pool, int mode) {
  if (!pool) return batch_mixed_kernel<false, -1, IG>;
  switch (mode) {
    case 0: return batch_mixed_kernel<true, 0, IG>;
    case 1: return batch_mixed_kernel<true, 1, IG>;
    case 2: return batch_mixed_kernel<true, 2, IG>;
    case 3: return batch_mixed_kernel<true, 3, IG>;
    case 4: return batch_mixed_kernel<true, 4, IG>;
    case 5: return batch_mixed_kernel<true, 5, IG>;
    default: return batch_mixed_kernel<true, -1, IG>;
  }
}

// the build for (pool, mode, item ghosts); mode -1 or out of range: any mix of modes
KernelFn kernel_for(bool pool, int mode, bool ig) {
  return ig ? kernel_for_ig<true>(pool, mode) : kernel_for_ig<false>(pool, mode);
}

// pool reservations per device: used[d][k] for descriptor k
std::mutex g_pool_mu;
std::map<int, std::vector<char>> g_pool_used;

}  // namespace

void launch_batch_mixed(const BatchView& v, int grid, bool pool, int mode, cudaStream_t st) {
  kernel_for(pool, mode, v.item_ghosts != 0)<<<grid, NT, 0, st>>>(v);
}
int batch_mixed_threads() { return NT; }
int batch_mixed_occupancy(bool pool, int mode) {
  int n = 0;  // the same for both ghost builds (same launch bounds)
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel_for(pool, mode, false), NT, 0);
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
