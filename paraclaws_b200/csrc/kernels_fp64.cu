// kernels_fp64.cu -- the FP64 parity path for one grid: one fused kernel per sweep direction
// doing the HLL Riemann solve, fluctuation splitting, first-order update, wave limiter,
// second-order correction flux and correction update of solver/MOD_solve.f90:23-293, plus the
// sweep's max-wave-speed reduction (MOD_solve.f90:72-86 / 126-139).  The bodies live in
// pcl_sweeps_fp64.cuh.  Built with --fmad=false.
#include <cuda_runtime.h>

#include <atomic>

#include "pcl_launch.h"
#include "pcl_sweeps_fp64.cuh"

namespace pcl {

// ------------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------------
namespace {
// Launch shapes (measured on B200, bumps after 100-300 steps, minmod; every variant
// bit-identical): the xi sweep at 8 CTAs of 128 threads per SM, each CTA sweeping 8 rows of its
// segment with one block reduction at the end, with the shared-reciprocal quotients
// (kOptFastDiv) and the row parity buffers: 0.387 ms at 4096^2 against 0.508 ms for one row per
// 256-thread CTA at 5 CTAs per SM (4 rows: 0.397; the limiter shortcut on top: 0.399; 8 rows in
// 256-thread CTAs with 252-cell segments, 4 per SM: 0.415).
// The eta sweep has two shapes.  Column windows (ysweep_strip) at 6 CTAs of 128 threads per SM
// (80 registers, a few spilled window values) with 24-row strips (16 rows: +1%, 32: +1%).  Bands
// (ysweep_band), 64 registers (4 bytes spilled), each thread staging its cell of the next step by
// cp.async while the phases of this one run, cell states by step parity (three barriers per
// step): 16 columns x 8 rows per step in 128-thread CTAs, 8 per SM (28 KB of shared memory
// each).  Same box, back to back, eta sweep in ms: 2048^2 0.134 (64-row chunks) against 0.142
// for 16 columns x 16 rows in 256-thread CTAs at 4 per SM (128-row chunks); 4096^2 0.433
// (128-row chunks) against 0.453 (256); 8192^2 1.544 against 1.623 (256 both); 8 columns x 16
// rows in 128-thread CTAs: 0.141, 0.458, 1.645.  The 256-thread CTAs had gained from the
// parity copies themselves: 0.452 against 0.459 ms at 4096^2 with a fourth barrier closing each
// step and the staging in a separate buffer.  Before them: 8 columns x 32 rows in 256 threads
// 0.503 ms, 16 columns x 32 rows in 512 threads (2 CTAs per SM) 0.521 ms.  Lab, eta sweep in
// ms on bumps after 8 / 200 steps, windows against 8-column bands: 4096^2 0.482 / 0.499
// against 0.465 / 0.468; 2048^2 0.155 / 0.156 against 0.141 / 0.144.  Without the staging the
// bands took 0.473 / 0.480 at 4096^2; 4-column bands 0.548 / 0.556 (their rows are single
// 32-byte sectors).  Bands run wherever the shared-reciprocal quotients do; the chunk is the
// tallest of 256, 128 and 64 rows that still makes kYWaves waves of CTAs, less the 4-row halo.
// Six waves of 8 CTAs per SM picked the fastest chunk, measured, at 1024^2 and 2048^2 (64),
// 4096^2 (128: 256 leaves 3.5 waves, the last one half empty) and 8192^2 (256); the halo
// rows off (252, 124, 60: no step half used) took the eta sweep from 0.046 / 0.134 / 0.431 /
// 1.543 ms to 0.045 / 0.127 / 0.420 / 1.513 ms at those sizes.  Measured and dropped: the two
// shortcuts and an unrolled row loop in the windows (more registers, more spills); tiles that
// recompute their 4 halo rows instead of carrying them (0.489 ms at 4096^2 at best); an xi sweep
// that stores its result transposed so the eta sweep can read contiguous lines (0.645 + 0.653
// ms: the strided stores cost more than the phases save); and the same cp.async staging in the
// xi sweep (0.3864 against 0.3875 ms: its row loads are fully coalesced already).
constexpr int kXT = 128;   // threads (and slots) of an xi-sweep CTA
constexpr int kXMinBlocks = 8;
constexpr int kXRows = 8;  // rows of one segment per xi-sweep CTA
constexpr int kYT = 128;   // columns of an eta-sweep window CTA
constexpr int kYMinBlocks = 6;
constexpr int kYS = 24;    // rows of an eta-sweep strip
constexpr int kBT = 128;   // threads of an eta-sweep band CTA
constexpr int kBX = 16;    // columns of a band
constexpr int kBMinBlocks = 8;
constexpr int kYWaves = 6;

// A CTA sweeps R consecutive rows of one segment (blockIdx.y*R ..), strided by gridDim.y*R
// when the grid has more rows than one launch's blocks cover.
template <int NT, int LIM, bool SO, int MK, int R = 1, int OPT = 0>
__global__ void __launch_bounds__(NT, kXMinBlocks) xsweep_fp64_kernel(GridDev g) {
  __shared__ XSmem<NT> S;
  if (g.ctl->done) return;
  double smax = 0.0;
  int bad = 0;
  int par = 0;
  for (int jb = 1 + blockIdx.y * R; jb <= g.my; jb += gridDim.y * R) {
    const int je = min(jb + R - 1, g.my);
    for (int j = jb; j <= je; ++j, par ^= 1)
      xsweep_segment<NT, LIM, SO, MK, OPT>(g, j, 1 + blockIdx.x * (NT - 4), S, smax, bad, par);
  }
  xsweep_finish<NT>(g, smax, bad, S);
}

template <int NTX, int STRIP, int LIM, bool SO, int MK>
__global__ void __launch_bounds__(NTX, kYMinBlocks) ysweep_fp64_kernel(GridDev g) {
  if (g.ctl->done) return;
  ysweep_strip<LIM, SO, MK>(g, 1 + blockIdx.x * NTX, 1 + blockIdx.y * STRIP, STRIP);
}

template <int LIM, bool SO, int MK>
__global__ void __launch_bounds__(kBT, kBMinBlocks) yband_fp64_kernel(GridDev g, int chunk) {
  extern __shared__ __align__(16) unsigned char band_smem[];
  auto& S = *reinterpret_cast<YBSmem<kBT, kBX, MK == kMetricMapped>*>(band_smem);
  if (g.ctl->done || !eta_valid(g)) return;
  double smax = 0.0;
  int bad = 0;
  const int j0 = 1 + blockIdx.y * chunk;
  ysweep_band<kBT, kBX, LIM, SO, MK, kOptFastDiv, true>(g, (int)blockIdx.x * kBX - 1, j0, j0 + chunk - 1, S, smax,
                                                        bad);
  block_max_to<kBT>(&g.ctl->smax_y, smax, S.red);
  if (bad) atomicOr(&g.ctl->status, bad);
}

// The shortcuts' range argument assumes g in [2^-20, 2^20] (pcl_fp64.cuh: kOptFastDiv).
inline bool fast_div_ok(const GridDev& g) { return g.grav >= 0x1p-20 && g.grav <= 0x1p20; }

template <int LIM, bool SO, int MK>
void launch_x_t(const GridDev& g, cudaStream_t st) {
  const int rb = (g.my + kXRows - 1) / kXRows;
  dim3 gx((g.mx + (kXT - 4) - 1) / (kXT - 4), rb < 65535 ? rb : 65535);
  if (fast_div_ok(g))
    xsweep_fp64_kernel<kXT, LIM, SO, MK, kXRows, kOptFastDiv><<<gx, kXT, 0, st>>>(g);
  else
    xsweep_fp64_kernel<kXT, LIM, SO, MK, kXRows><<<gx, kXT, 0, st>>>(g);
}
int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}
}  // namespace

// The eta shape the launcher runs for g (kEtaWindow or kEtaBand).
int eta_shape_of(const GridDev& g) {
  // the generic modules' bands need no shared reciprocals (kernels_gen.cu)
  if (g.eq == PCL_EQ_SHALLOW_WATER && !fast_div_ok(g)) return kEtaWindow;
  return g.eta_shape == kEtaWindow ? kEtaWindow : kEtaBand;
}

namespace {
template <int LIM, bool SO, int MK>
void launch_y_t(const GridDev& g, cudaStream_t st) {
  dim3 gy((g.mx + kYT - 1) / kYT, (g.my + kYS - 1) / kYS);
  if (eta_shape_of(g) == kEtaBand) {
    const long long bands = (g.mx + 2 + kBX - 1) / kBX, want = (long long)kYWaves * kBMinBlocks * sm_count();
    // A chunk of c rows takes (c + 4) / L steps of L = kBT / kBX rows (its first step fills the
    // 4-row halo), so chunks 4 rows short of 256, 128 or 64 leave no step half used.
    int c = 256;
    while (c > 64 && bands * ((g.my + c - 5) / (c - 4)) < want) c /= 2;
    const int chunk = c - 4;
    static_assert((64 % (kBT / kBX)) == 0, "chunk heights: multiples of the step height, less the halo");
    dim3 gb((unsigned)bands, (g.my + chunk - 1) / chunk);
    // 28 KB (mapped grids: 30 KB) of dynamic shared memory: allowed once per device for each build
    constexpr int smem = (int)sizeof(YBSmem<kBT, kBX, MK == kMetricMapped>);
    static std::atomic<unsigned long long> allowed{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const unsigned long long bit = 1ull << (dev & 63);
    if (!(allowed.load() & bit)) {
      cudaFuncSetAttribute(yband_fp64_kernel<LIM, SO, MK>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      allowed.fetch_or(bit);
    }
    yband_fp64_kernel<LIM, SO, MK><<<gb, kBT, smem, st>>>(g, chunk);
  } else {
    ysweep_fp64_kernel<kYT, kYS, LIM, SO, MK><<<gy, kYT, 0, st>>>(g);
  }
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
