// kernels_mixed.cu -- the precision form for one grid: one CTA per work item of the fused
// row-streaming kernel in pcl_stream_mixed.cuh.  Built with --fmad=false (explicit multiply-adds).
#include <cuda_runtime.h>

#include "../../include/paraclaws_b200.h"
#include "pcl_ghost.cuh"
#include "pcl_mixed.h"
#include "pcl_stream_mixed.cuh"
#include "pcl_timectl.cuh"

namespace pcl {
namespace mixed {

// INJ: the build for the test of the timeout path (mixed_item), launched only while a copy
// stall is injected from the host (mixed_set_injection).
template <int LIM, bool SO, bool INJ = false>
__global__ void __launch_bounds__(NT) fused_mixed_kernel(GridDev g, int TY, int nstrips, int inj_row,
                                                         unsigned probes) {
  __shared__ Smem S;
  if (g.ctl->done) return;
  init_ring(S);
  unsigned rows = 0;
  mixed_item<LIM, SO, 2, INJ>(g, blockIdx.x % nstrips, blockIdx.x / nstrips, TY, S, rows, inj_row, probes);
}

// The whole attempt in one launch (the device loop when no host hook runs between the time
// control and the ghost fill): a CTA whose item lies on the edge of the grid fills the ghost
// cells next to the cells it wrote, into the step's output buffer (unused if the step is
// rejected); the CTA that finishes the last item runs the time control (full_step: CFL,
// accept/reject, updateTime, snapshot index, reset_CFL, log) and, after an accepted step, the
// ghost sides no item could fill (a last strip or segment one cell wide).  The same values as
// the separate time-control and ghost kernels: only where they are computed changes.
template <int LIM, bool SO>
__global__ void __launch_bounds__(NT, 5) fused_mixed_step_kernel(GridDev g, int TY, int nstrips) {
  __shared__ Smem S;
  __shared__ int s_last;
  Ctl* ctl = g.ctl;
  if (ctl->done) return;
  init_ring(S);
  unsigned rows = 0;
  const int strip = blockIdx.x % nstrips, seg = blockIdx.x / nstrips;
  const bool ok = mixed_item<LIM, SO, 2>(g, strip, seg, TY, S, rows);
  if (ok && (strip == 0 || seg == 0 || (strip + 1) * TXI >= g.mx || (seg + 1) * TY >= g.my)) {
    const int cur = ctl->cur;
    const int i0 = 1 + strip * TXI, j0 = 1 + seg * TY;
    ghost_fill_block(g, buffer(g, cur == 0 ? 2 : cur - 1), i0, min(i0 + TXI - 1, g.mx), j0, min(j0 + TY - 1, g.my));
  }
  __threadfence();  // every thread's writes of this item precede its completion count
  __syncthreads();
  if (threadIdx.x == 0) {
    s_last = atomicAdd(&ctl->items_done, 1) + 1 == (int)gridDim.x;
    if (s_last) {
      __threadfence();
      full_step(ctl, g);
      ctl->items_done = 0;
      __threadfence();
    }
  }
  __syncthreads();
  if (s_last && ctl->ierr == 1)
    ghost_fill_open_sides(g, buffer(g, ctl->cur), (g.mx - 1) % TXI == 0, (g.my - 1) % TY == 0);
}

struct Workspace {
  int ty;
  int inj_row = -1;        // row whose bulk copy is not issued (-1: none)
  unsigned probes = 0;     // probe limit of the waits in that build
};

}  // namespace mixed

// Default rows per CTA: 128 where that still makes at least four waves of CTAs (fewer halo
// rows per row computed), else 64.  Measured on B200: 8192^2 runs best at 128, 4096^2 at 64,
// where 128 leaves 1.5 waves and the last one half empty.
int mixed_create(const GridDev& g, cudaStream_t, void** ws) {
  auto* w = new mixed::Workspace();
  w->ty = 64;
  int dev = 0, sms = 0, per = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) ==
                                                 cudaSuccess &&
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, mixed::fused_mixed_kernel<1, true>, mixed::NT, 0) ==
          cudaSuccess &&
      sms > 0 && per > 0) {
    const long long ctas = (long long)((g.mx + mixed::TXI - 1) / mixed::TXI) * ((g.my + 127) / 128);
    if (ctas >= 4LL * sms * per) w->ty = 128;
  }
  *ws = w;
  return PCL_OK;
}

void mixed_free(void* ws) { delete static_cast<mixed::Workspace*>(ws); }

void mixed_set_tile_rows(void* ws, int ty) {
  if (ws && ty >= 4) static_cast<mixed::Workspace*>(ws)->ty = ty;
}

void mixed_set_injection(void* ws, int row, unsigned probes) {
  if (!ws) return;
  auto* w = static_cast<mixed::Workspace*>(ws);
  w->inj_row = row;
  w->probes = probes > 0 ? probes : 1u;
}

namespace {
template <int LIM, bool SO>
void launch_t(const GridDev& g, const mixed::Workspace* w, cudaStream_t st) {
  const int ty = w ? w->ty : 64;
  const int nstrips = (g.mx + mixed::TXI - 1) / mixed::TXI;
  const int nseg = (g.my + ty - 1) / ty;
  if (w && w->inj_row >= 0)
    mixed::fused_mixed_kernel<LIM, SO, true><<<nstrips * nseg, mixed::NT, 0, st>>>(g, ty, nstrips, w->inj_row,
                                                                                  w->probes);
  else
    mixed::fused_mixed_kernel<LIM, SO><<<nstrips * nseg, mixed::NT, 0, st>>>(g, ty, nstrips, -1, 0u);
}
}  // namespace

namespace {
template <int LIM, bool SO>
void launch_step_t(const GridDev& g, const mixed::Workspace* w, cudaStream_t st) {
  const int ty = w ? w->ty : 64;
  const int nstrips = (g.mx + mixed::TXI - 1) / mixed::TXI;
  const int nseg = (g.my + ty - 1) / ty;
  mixed::fused_mixed_step_kernel<LIM, SO><<<nstrips * nseg, mixed::NT, 0, st>>>(g, ty, nstrips);
}
}  // namespace

void launch_step_mixed(const GridDev& g, void* ws, cudaStream_t st) {
  const auto* w = static_cast<const mixed::Workspace*>(ws);
  if (!g.second_order) return launch_step_t<0, false>(g, w, st);
  switch (g.limiter) {
    case 1: return launch_step_t<1, true>(g, w, st);
    case 2: return launch_step_t<2, true>(g, w, st);
    case 3: return launch_step_t<3, true>(g, w, st);
    case 4: return launch_step_t<4, true>(g, w, st);
    default: return launch_step_t<0, true>(g, w, st);
  }
}

bool mixed_injection_on(const void* ws) {
  return ws && static_cast<const mixed::Workspace*>(ws)->inj_row >= 0;
}

void launch_sweeps_mixed(const GridDev& g, void* ws, cudaStream_t st) {
  const auto* w = static_cast<const mixed::Workspace*>(ws);
  if (!g.second_order) return launch_t<0, false>(g, w, st);
  switch (g.limiter) {
    case 1: return launch_t<1, true>(g, w, st);
    case 2: return launch_t<2, true>(g, w, st);
    case 3: return launch_t<3, true>(g, w, st);
    case 4: return launch_t<4, true>(g, w, st);
    default: return launch_t<0, true>(g, w, st);
  }
}

}  // namespace pcl
