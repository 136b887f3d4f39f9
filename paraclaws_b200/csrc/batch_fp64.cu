// batch_fp64.cu -- the FP64 parity step for a batch of grids in one persistent launch.
//
// CTAs (128 threads) pull work items from a queue: first every instance's xi-sweep items, then
// every instance's eta-sweep items.  An eta item waits (bounded) until all xi items of its
// instance are done.  Those xi items were dequeued before it by CTAs that are running and never
// wait, so the wait always ends.  The CTA that finishes an instance's last item runs that
// instance's time control (pcl_timectl.cuh) and, if the attempt was accepted, its ghost fill.
// Per-cell arithmetic is the single-grid kernels' (pcl_sweeps_fp64.cuh): a batched instance is
// bit-identical to the same grid run alone.  Built with --fmad=false.
#include <cuda_runtime.h>

#include "pcl_batch.h"
#include "pcl_ghost.cuh"
#include "pcl_sweeps_fp64.cuh"
#include "pcl_timectl.cuh"

namespace pcl {
namespace {

// 128-thread CTAs, 6 per SM (80 registers): measured on B200 with 512 uneven dam breaks, 1.55x
// the 256-thread, 2-per-SM shape, because both sweeps are latency bound on FP64 division chains.
constexpr int kThreads = 128;
constexpr int kMinBlocks = 6;

template <int LIM, bool SO, int MK>
__device__ __forceinline__ void run_item(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                         XSmem<kThreads>& S) {
  if (kind == kItemX) {
    const int jend = min(a + v.x_rows - 1, g.my);
    double smax = 0.0;
    int bad = 0;
    for (int j = a; j <= jend; ++j) {
      xsweep_segment<kThreads, LIM, SO, MK>(g, j, b, S, smax, bad);
      __syncthreads();  // the segment's shared arrays are reused by the next row
    }
    xsweep_finish<kThreads>(g, smax, bad, S);
  } else {
    ysweep_strip<LIM, SO, MK>(g, a, b, v.y_rows);
  }
}

template <int MK>
__device__ __forceinline__ void dispatch_lim(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                             XSmem<kThreads>& S) {
  if (!g.second_order) return run_item<0, false, MK>(g, kind, a, b, v, S);
  switch (g.limiter) {
    case 1: return run_item<1, true, MK>(g, kind, a, b, v, S);
    case 2: return run_item<2, true, MK>(g, kind, a, b, v, S);
    case 3: return run_item<3, true, MK>(g, kind, a, b, v, S);
    case 4: return run_item<4, true, MK>(g, kind, a, b, v, S);
    default: return run_item<0, true, MK>(g, kind, a, b, v, S);
  }
}

__device__ __forceinline__ void dispatch_item(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                              XSmem<kThreads>& S) {
  // batched instances are uniform grids (pcl_batch_add builds the row/column tables)
  if (g.metric == kMetricUnit) return dispatch_lim<kMetricUnit>(g, kind, a, b, v, S);
  return dispatch_lim<kMetricTable>(g, kind, a, b, v, S);
}

// IG: eta items on the edge of their grid fill the ghost cells next to the cells they wrote
// (ghost_fill_block) and the finishing CTA only the sides left open; else the finishing CTA
// fills them all.  Separate builds, so the item loop of the IG = false build carries no ghost
// code.  Same values either way.
template <bool IG>
__global__ void __launch_bounds__(kThreads, kMinBlocks) batch_fp64_kernel(BatchView v) {
  __shared__ XSmem<kThreads> S;
  __shared__ int s_item;
  __shared__ int s_flag;
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
    int* xdone = v.counters + 2 * w.x;
    int* alldone = xdone + 1;
    if (!ctl->done) {
      if (w.y == kItemY) {
        // wait for every xi item of this instance (bounded; they are all in flight or done)
        if (threadIdx.x == 0) {
          const int need = v.totals[2 * w.x] + (w.x == v.stall_slot ? 1 : 0);
          unsigned k = 0;
          while (atomicAdd(xdone, 0) < need && k < v.spin_limit) {
            __nanosleep(64);
            ++k;
          }
          s_flag = atomicAdd(xdone, 0) >= need;
          if (!s_flag) {
            atomicOr(&ctl->status, kStatusTimeout);
            atomicOr(v.flags, 1);
          }
          __threadfence();
        }
        __syncthreads();
        if (s_flag) {
          dispatch_item(g, w.y, w.z, w.w, v, S);
          if (IG) {
            const int i1 = min(w.z + kThreads - 1, g.mx), j1 = min(w.w + v.y_rows - 1, g.my);
            if (w.z == 1 || w.w == 1 || i1 == g.mx || j1 == g.my) {
              __syncthreads();  // the strip's cells, written by every thread, before any is read
              const int cur = ctl->cur;
              ghost_fill_block(g, buffer(g, cur == 0 ? 2 : cur - 1), w.z, i1, w.w, j1);
            }
          }
        }
      } else {
        dispatch_item(g, w.y, w.z, w.w, v, S);
      }
    }
    __threadfence();  // every thread's writes of this item precede its completion count
    __syncthreads();
    if (threadIdx.x == 0) {
      if (w.y == kItemX) atomicAdd(xdone, 1);
      s_flag = atomicAdd(alldone, 1) + 1 == v.totals[2 * w.x + 1];
      if (s_flag) {
        __threadfence();
        full_step(ctl, g);  // CFL, accept/reject, updateTime, snapshot, reset_CFL, log
        *xdone = 0;
        *alldone = 0;
        __threadfence();
      }
    }
    __syncthreads();
    if (s_flag && ctl->ierr == 1) {  // update_rank_boundaries of the accepted instance
      double* b = buffer(g, ctl->cur);
      if (IG) {
        ghost_fill_open_sides(g, b, (g.mx - 1) % kThreads == 0, (g.my - 1) % v.y_rows == 0);
      } else {
        const int ng = ghost_items(g);
        for (int k = threadIdx.x; k < ng; k += blockDim.x) ghost_item(g, b, k);
      }
    }
    __syncthreads();
  }
}

}  // namespace

void launch_batch_fp64(const BatchView& v, int grid, cudaStream_t st) {
  if (v.item_ghosts)
    batch_fp64_kernel<true><<<grid, kThreads, 0, st>>>(v);
  else
    batch_fp64_kernel<false><<<grid, kThreads, 0, st>>>(v);
}
int batch_fp64_threads() { return kThreads; }
int batch_fp64_segment() { return kThreads - 4; }
int batch_fp64_occupancy() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_fp64_kernel<false>, kThreads, 0);
  return n > 0 ? n : 1;
}

}  // namespace pcl
