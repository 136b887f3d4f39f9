// kernels_mixed.cu -- the precision form for one grid: one CTA per work item of the fused
// row-streaming kernel in pcl_stream_mixed.cuh.  Built with --fmad=false (explicit multiply-adds).
#include <cuda_runtime.h>

#include "../../include/paraclaws_b200.h"
#include "pcl_mixed.h"
#include "pcl_stream_mixed.cuh"

namespace pcl {
namespace mixed {

template <int LIM, bool SO>
__global__ void __launch_bounds__(NT) fused_mixed_kernel(GridDev g, int TY, int nstrips) {
  __shared__ Smem S;
  if (g.ctl->done) return;
  init_ring(S);
  unsigned rows = 0;
  mixed_item<LIM, SO, 2>(g, blockIdx.x % nstrips, blockIdx.x / nstrips, TY, S, rows);
}

struct Workspace {
  int ty;
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

namespace {
template <int LIM, bool SO>
void launch_t(const GridDev& g, int ty, cudaStream_t st) {
  const int nstrips = (g.mx + mixed::TXI - 1) / mixed::TXI;
  const int nseg = (g.my + ty - 1) / ty;
  mixed::fused_mixed_kernel<LIM, SO><<<nstrips * nseg, mixed::NT, 0, st>>>(g, ty, nstrips);
}
}  // namespace

void launch_sweeps_mixed(const GridDev& g, void* ws, cudaStream_t st) {
  const int ty = ws ? static_cast<mixed::Workspace*>(ws)->ty : 64;
  if (!g.second_order) return launch_t<0, false>(g, ty, st);
  switch (g.limiter) {
    case 1: return launch_t<1, true>(g, ty, st);
    case 2: return launch_t<2, true>(g, ty, st);
    case 3: return launch_t<3, true>(g, ty, st);
    case 4: return launch_t<4, true>(g, ty, st);
    default: return launch_t<0, true>(g, ty, st);
  }
}

}  // namespace pcl
