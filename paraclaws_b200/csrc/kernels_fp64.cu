// kernels_fp64.cu -- the FP64 parity path for one grid: one fused kernel per sweep direction
// doing the HLL Riemann solve, fluctuation splitting, first-order update, wave limiter,
// second-order correction flux and correction update of solver/MOD_solve.f90:23-293, plus the
// sweep's max-wave-speed reduction (MOD_solve.f90:72-86 / 126-139).  The bodies live in
// pcl_sweeps_fp64.cuh.  Built with --fmad=false.
#include <cuda_runtime.h>

#include "pcl_launch.h"
#include "pcl_sweeps_fp64.cuh"

namespace pcl {

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
namespace {
// Launch shapes (measured on B200, 4096^2 minmod): the xi sweep at 5 CTAs of 256 threads per SM
// (48 registers) and the eta sweep at 6 CTAs of 128 threads per SM (80 registers, a few spilled
// window values) with 16-row strips beat the unconstrained register counts (4 CTAs each) by
// 20 %: both kernels are latency bound on chains of FP64 divisions and need the warps.
constexpr int kXT = 256;   // threads (and slots) of an xi-sweep CTA
constexpr int kXMinBlocks = 5;
constexpr int kYT = 128;   // columns of an eta-sweep CTA
constexpr int kYMinBlocks = 6;
constexpr int kYS = 16;    // rows of an eta-sweep strip

// A CTA sweeps R consecutive rows of one segment (blockIdx.y*R ..), strided by gridDim.y*R
// when the grid has more rows than one launch's blocks cover.
template <int NT, int LIM, bool SO, int MK, int R = 1, int OPT = 0>
__global__ void __launch_bounds__(NT, kXMinBlocks) xsweep_fp64_kernel(GridDev g) {
  __shared__ XSmem<NT> S;
  if (g.ctl->done) return;
  double smax = 0.0;
  int bad = 0;
  for (int jb = 1 + blockIdx.y * R; jb <= g.my; jb += gridDim.y * R) {
    const int je = min(jb + R - 1, g.my);
    for (int j = jb; j <= je; ++j) {
      xsweep_segment<NT, LIM, SO, MK, OPT>(g, j, 1 + blockIdx.x * (NT - 4), S, smax, bad);
      __syncthreads();  // the shared arrays are reused by the next row
    }
  }
  xsweep_finish<NT>(g, smax, bad, S);
}

template <int NTX, int STRIP, int LIM, bool SO, int MK>
__global__ void __launch_bounds__(NTX, kYMinBlocks) ysweep_fp64_kernel(GridDev g) {
  if (g.ctl->done) return;
  ysweep_strip<LIM, SO, MK>(g, 1 + blockIdx.x * NTX, 1 + blockIdx.y * STRIP, STRIP);
}

template <int LIM, bool SO, int MK>
void launch_x_t(const GridDev& g, cudaStream_t st) {
  dim3 gx((g.mx + (kXT - 4) - 1) / (kXT - 4), g.my < 65535 ? g.my : 65535);
  xsweep_fp64_kernel<kXT, LIM, SO, MK><<<gx, kXT, 0, st>>>(g);
}
template <int LIM, bool SO, int MK>
void launch_y_t(const GridDev& g, cudaStream_t st) {
  dim3 gy((g.mx + kYT - 1) / kYT, (g.my + kYS - 1) / kYS);
  ysweep_fp64_kernel<kYT, kYS, LIM, SO, MK><<<gy, kYT, 0, st>>>(g);
}
template <template <int, bool, int> class F, int MK>
void dispatch_lim(const GridDev& g, cudaStream_t st) {
  if (!g.second_order) return F<0, false, MK>::run(g, st);
  switch (g.limiter) {
    case 1: return F<1, true, MK>::run(g, st);
    case 2: return F<2, true, MK>::run(g, st);
    case 3: return F<3, true, MK>::run(g, st);
    case 4: return F<4, true, MK>::run(g, st);
    default: return F<0, true, MK>::run(g, st);
  }
}
template <template <int, bool, int> class F>
void dispatch(const GridDev& g, cudaStream_t st) {
  if (g.metric == kMetricUnit) return dispatch_lim<F, kMetricUnit>(g, st);
  if (g.metric == kMetricMapped) return dispatch_lim<F, kMetricMapped>(g, st);
  return dispatch_lim<F, kMetricTable>(g, st);
}
template <int LIM, bool SO, int MK>
struct XL {
  static void run(const GridDev& g, cudaStream_t st) { launch_x_t<LIM, SO, MK>(g, st); }
};
template <int LIM, bool SO, int MK>
struct YL {
  static void run(const GridDev& g, cudaStream_t st) { launch_y_t<LIM, SO, MK>(g, st); }
};
}  // namespace

// Modules other than the specialised shallow water run the generic sweeps (kernels_gen.cu).
void launch_xsweep_fp64(const GridDev& g, cudaStream_t st) {
  if (g.eq != PCL_EQ_SHALLOW_WATER) return launch_xsweep_gen(g, st);
  dispatch<XL>(g, st);
}
void launch_ysweep_fp64(const GridDev& g, cudaStream_t st) {
  if (g.eq != PCL_EQ_SHALLOW_WATER) return launch_ysweep_gen(g, st);
  dispatch<YL>(g, st);
}
void launch_sweeps_fp64(const GridDev& g, cudaStream_t st) {
  launch_xsweep_fp64(g, st);
  launch_ysweep_fp64(g, st);
}

}  // namespace pcl
