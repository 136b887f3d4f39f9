// kernels_gen.cu -- the FP64 step for the equation modules other than the specialised shallow
// water (pcl_equations.h), for contexts of N = 1, 3 or 4 equations: one kernel per sweep
// direction over the bodies in pcl_sweeps_gen.cuh.  Built with --fmad=false.
#include <cuda_runtime.h>

#include "pcl_launch.h"
#include "pcl_sweeps_gen.cuh"

namespace pcl {
namespace {

constexpr int kGXT = 128;  // threads (slots) of an xi-sweep CTA
constexpr int kGXRows = 4; // rows of one segment per xi-sweep CTA
constexpr int kGYT = 128;  // columns of an eta-sweep window CTA
constexpr int kGYS = 32;   // rows of an eta-sweep strip
// Eta sweep in bands (the default; gen::ysweep_band): 128-thread CTAs on 8-column bands, 16 rows
// per step, chunks of 252 rows, 124 or 60 while the grid makes fewer than 3 waves, 6 CTAs per SM.
// At 4096^2 the dam-break module runs at 11.0 G cell-updates/s (10.7 G with 256-row chunks, whose
// last step ran half used) against 9.1 G with the column windows (5 CTAs per SM without the
// register cap: 10.4 G); acoustics 13.1 G (12.8 G with 256-row chunks and with the windows).
constexpr int kGBT = 128;
constexpr int kGBX = 8;

template <int N, int LIM, bool SO>
__global__ void __launch_bounds__(kGXT) xsweep_gen_kernel(GridDev g) {
  __shared__ gen::XSmem<kGXT, N> S;
  if (g.ctl->done) return;
  double smax = 0.0;
  int bad = 0;
  for (int jb = 1 + blockIdx.y * kGXRows; jb <= g.my; jb += gridDim.y * kGXRows) {
    const int je = min(jb + kGXRows - 1, g.my);
    for (int j = jb; j <= je; ++j) {
      gen::xsweep_segment<kGXT, N, LIM, SO>(g, j, 1 + blockIdx.x * (kGXT - 4), S, smax, bad);
      __syncthreads();
    }
  }
  gen::xsweep_finish<kGXT, N>(g, smax, bad, S);
}

template <int N, int LIM, bool SO>
__global__ void __launch_bounds__(kGYT) ysweep_gen_kernel(GridDev g) {
  if (g.ctl->done) return;
  gen::ysweep_strip<N, LIM, SO>(g, 1 + blockIdx.x * kGYT, 1 + blockIdx.y * kGYS, kGYS);
}

template <int N, int LIM, bool SO>
__global__ void __launch_bounds__(kGBT, 6) yband_gen_kernel(GridDev g, int chunk) {
  __shared__ gen::YBSmem<kGBT, kGBX, N> S;
  if (g.ctl->done || !eta_valid(g)) return;
  double smax = 0.0;
  int bad = 0;
  const int j0 = 1 + blockIdx.y * chunk;
  gen::ysweep_band<kGBT, kGBX, N, LIM, SO>(g, (int)blockIdx.x * kGBX - 1, j0, j0 + chunk - 1, S, smax, bad);
  block_max_to<kGBT>(&g.ctl->smax_y, smax, S.red);
  if (bad) atomicOr(&g.ctl->status, bad);
}

int sm_count_gen() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

template <int N, int LIM, bool SO>
struct GenLaunch {
  static void x(const GridDev& g, cudaStream_t st) {
    const int rb = (g.my + kGXRows - 1) / kGXRows;
    dim3 gx((g.mx + (kGXT - 4) - 1) / (kGXT - 4), rb < 65535 ? rb : 65535);
    xsweep_gen_kernel<N, LIM, SO><<<gx, kGXT, 0, st>>>(g);
  }
  static void y(const GridDev& g, cudaStream_t st) {
    if (g.eta_shape == kEtaWindow) {
      dim3 gy((g.mx + kGYT - 1) / kGYT, (g.my + kGYS - 1) / kGYS);
      ysweep_gen_kernel<N, LIM, SO><<<gy, kGYT, 0, st>>>(g);
      return;
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, yband_gen_kernel<N, LIM, SO>, kGBT, 0);
    const long long bands = (g.mx + 2 + kGBX - 1) / kGBX, want = 3LL * (occ > 0 ? occ : 1) * sm_count_gen();
    // a chunk of c rows takes (c + 4) / 16 steps (the first fills the 4-row halo): chunks 4 rows
    // short of 256, 128 or 64 leave no step half used
    int c = 256;
    while (c > 64 && bands * ((g.my + c - 5) / (c - 4)) < want) c /= 2;
    const int chunk = c - 4;
    dim3 gb((unsigned)bands, (g.my + chunk - 1) / chunk);
    yband_gen_kernel<N, LIM, SO><<<gb, kGBT, 0, st>>>(g, chunk);
  }
};

template <int N>
void dispatch_n(const GridDev& g, bool xi, cudaStream_t st) {
#define PCL_GEN_CASE(LIM, SO) return xi ? GenLaunch<N, LIM, SO>::x(g, st) : GenLaunch<N, LIM, SO>::y(g, st)
  if (!g.second_order) PCL_GEN_CASE(0, false);
  switch (g.limiter) {
    case 1: PCL_GEN_CASE(1, true);
    case 2: PCL_GEN_CASE(2, true);
    case 3: PCL_GEN_CASE(3, true);
    case 4: PCL_GEN_CASE(4, true);
    default: PCL_GEN_CASE(0, true);
  }
#undef PCL_GEN_CASE
}

void dispatch(const GridDev& g, bool xi, cudaStream_t st) {
  switch (g.neq) {
    case 1: return dispatch_n<1>(g, xi, st);
    case 4: return dispatch_n<4>(g, xi, st);
    default: return dispatch_n<3>(g, xi, st);
  }
}

}  // namespace

void launch_xsweep_gen(const GridDev& g, cudaStream_t st) { dispatch(g, true, st); }
void launch_ysweep_gen(const GridDev& g, cudaStream_t st) { dispatch(g, false, st); }

}  // namespace pcl
