// batch_fp64.cu -- the FP64 parity step for a batch of grids in one persistent launch.
//
// CTAs (128 threads) pull work items from a queue: first every instance's xi-sweep items (rows
// of a row segment), then every instance's eta-sweep items (a chunk of rows of a 4-column band).
// An eta item waits (bounded) until all xi items of its instance are done.  Those xi items were
// dequeued before it by CTAs that are running and never wait, so the wait always ends.  The CTA that finishes an instance's last item runs that
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

// 128-thread CTAs, 8 per SM: both item kinds run the sweeps' shared-memory phases (xi items:
// rows of a 124-cell segment; eta items: a chunk of rows of a 4-column band, ysweep_band), which
// fit 64 registers.  The item's grid descriptor is staged in shared memory, so the sweeps read
// its fields there instead of from a stack copy.  Batched grids are uniform, so the bands carry
// no mapped-grid metrics.  Measured on C4's 512 grids: 12.5 G cell-updates/s with these bands,
// 10.6 G with the single-grid kernel's 8-column bands and cp.async staging (fewer, longer items
// for the many small grids).
constexpr int kThreads = 128;
constexpr int kMinBlocks = 8;
constexpr int kBandCols = 4;

union BatchSmem {
  XSmem<kThreads> x;
  YBSmem<kThreads, kBandCols, false, false> y;
};

template <int LIM, bool SO, int MK, int OPT>
__device__ __forceinline__ void run_item(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                         BatchSmem& S) {
  double smax = 0.0;
  int bad = 0;
  if (kind == kItemX) {
    const int jend = min(a + v.x_rows - 1, g.my);
    for (int j = a, par = 0; j <= jend; ++j, par ^= 1)
      xsweep_segment<kThreads, LIM, SO, MK, OPT>(g, j, b, S.x, smax, bad, par);
    xsweep_finish<kThreads>(g, smax, bad, S.x);
  } else {
    if (!eta_valid(g)) return;  // the same answer for every thread: all xi items are done
    ysweep_band<kThreads, kBandCols, LIM, SO, MK, OPT, false, false>(g, a, b, b + v.y_rows - 1, S.y, smax, bad);
    block_max_to<kThreads>(&g.ctl->smax_y, smax, S.y.red);
    if (bad) atomicOr(&g.ctl->status, bad);
  }
}

template <int MK, int OPT>
__device__ __forceinline__ void dispatch_lim(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                             BatchSmem& S) {
  if (!g.second_order) return run_item<0, false, MK, OPT>(g, kind, a, b, v, S);
  switch (g.limiter) {
    case 1: return run_item<1, true, MK, OPT>(g, kind, a, b, v, S);
    case 2: return run_item<2, true, MK, OPT>(g, kind, a, b, v, S);
    case 3: return run_item<3, true, MK, OPT>(g, kind, a, b, v, S);
    case 4: return run_item<4, true, MK, OPT>(g, kind, a, b, v, S);
    default: return run_item<0, true, MK, OPT>(g, kind, a, b, v, S);
  }
}

// FD: every instance's g lies in the range of the shared-reciprocal quotients (kOptFastDiv,
// bit-identical to division), chosen by the host per launch.
template <int FD>
__device__ __forceinline__ void dispatch_item(const GridDev& g, int kind, int a, int b, const BatchView& v,
                                              BatchSmem& S) {
  // batched instances are uniform grids (pcl_batch_add builds the row/column tables)
  if (g.metric == kMetricUnit) return dispatch_lim<kMetricUnit, FD ? kOptFastDiv : 0>(g, kind, a, b, v, S);
  return dispatch_lim<kMetricTable, FD ? kOptFastDiv : 0>(g, kind, a, b, v, S);
}

// IG: eta items on the edge of their grid fill the ghost cells next to the cells they wrote
// (ghost_fill_block) and the finishing CTA only the sides left open; else the finishing CTA
// fills them all.  Separate builds, so the item loop of the IG = false build carries no ghost
// code.  Same values either way.
template <bool IG, int FD>
__global__ void __launch_bounds__(kThreads, kMinBlocks) batch_fp64_kernel(BatchView v) {
  __shared__ BatchSmem S;
  __shared__ GridDev sg;
  __shared__ int s_item;
  __shared__ int s_flag;
  const int n = *v.n_items;
  for (;;) {
    if (threadIdx.x == 0) s_item = (int)atomicAdd(v.head, 1u);
    __syncthreads();
    const int it = s_item;
    if (it >= n) break;
    const int4 w = v.items[it];
    {  // the item's grid descriptor into shared memory
      static_assert(sizeof(GridDev) % sizeof(int) == 0, "descriptor copy");
      const int* src = reinterpret_cast<const int*>(v.inst + w.x);
      int* dst = reinterpret_cast<int*>(&sg);
      for (int k = threadIdx.x; k < (int)(sizeof(GridDev) / sizeof(int)); k += kThreads) dst[k] = src[k];
    }
    __syncthreads();
    const GridDev& g = sg;
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
          dispatch_item<FD>(g, w.y, w.z, w.w, v, S);
          if (IG) {
            const int i0 = max(w.z, 1), i1 = min(w.z + kBandCols - 1, g.mx), j1 = min(w.w + v.y_rows - 1, g.my);
            if (i0 == 1 || w.w == 1 || i1 == g.mx || j1 == g.my) {
              __syncthreads();  // the chunk's cells, written by every thread, before any is read
              const int cur = ctl->cur;
              ghost_fill_block(g, buffer(g, cur == 0 ? 2 : cur - 1), i0, i1, w.w, j1);
            }
          }
        }
      } else {
        dispatch_item<FD>(g, w.y, w.z, w.w, v, S);
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
        // the last band or chunk one cell wide leaves its high side to the finisher
        const int lb = max(-1 + kBandCols * ((g.mx + 1) / kBandCols), 1);
        ghost_fill_open_sides(g, b, g.mx - lb + 1 < 2, (g.my - 1) % v.y_rows == 0);
      } else {
        const int ng = ghost_items(g);
        for (int k = threadIdx.x; k < ng; k += blockDim.x) ghost_item(g, b, k);
      }
    }
    __syncthreads();
  }
}

template <bool IG, int FD>
void launch(const BatchView& v, int grid, cudaStream_t st) {
  batch_fp64_kernel<IG, FD><<<grid, kThreads, 0, st>>>(v);
}

}  // namespace

void launch_batch_fp64(const BatchView& v, int grid, cudaStream_t st) {
  if (v.item_ghosts)
    v.fast_div ? launch<true, 1>(v, grid, st) : launch<true, 0>(v, grid, st);
  else
    v.fast_div ? launch<false, 1>(v, grid, st) : launch<false, 0>(v, grid, st);
}
int batch_fp64_threads() { return kThreads; }
int batch_fp64_segment() { return kThreads - 4; }
int batch_fp64_band() { return kBandCols; }
int batch_fp64_occupancy() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_fp64_kernel<false, 1>, kThreads, 0);
  return n > 0 ? n : 1;
}

}  // namespace pcl
