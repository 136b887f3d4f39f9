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
// Launch shapes (measured on B200, 4096^2 bumps after 300 steps, minmod; every variant
// bit-identical): the xi sweep at 8 CTAs of 128 threads per SM, each CTA sweeping 8 rows of its
// segment with one block reduction at the end, with the shared-reciprocal quotients
// (kOptFastDiv): 0.391 ms against 0.508 ms for one row per 256-thread CTA at 5 CTAs per SM (4
// rows: 0.397; the limiter shortcut on top: 0.399).  The eta sweep at 6 CTAs of 128 threads per
// SM (80 registers, a few spilled window values) with 24-row strips: 0.487 ms (16 rows: 0.492,
// 32: 0.492).  Neither shortcut nor unrolling its row loop helps it (more registers, more
// spills), and the xi sweep's phases run along columns of transposed tiles (ysweep_tile) are
// slower (0.516 ms at best, with 4-column tiles and four tiles per CTA).
constexpr int kXT = 128;   // threads (and slots) of an xi-sweep CTA
constexpr int kXMinBlocks = 8;
constexpr int kXRows = 8;  // rows of one segment per xi-sweep CTA
constexpr int kYT = 128;   // columns of an eta-sweep CTA
constexpr int kYMinBlocks = 6;
constexpr int kYS = 24;    // rows of an eta-sweep strip

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

// ---- the sweeps through a transposed intermediate (pcl_sweeps_fp64.cuh: line_sweep) ----
// xi sweep: a CTA takes R consecutive rows (R even, so pairs of rows start at an odd row) of one
// segment of NT-4 cells and writes each cell's new value into the transposed xi-swept buffer,
// two rows at a time: cells (i, j-1) and (i, j) are adjacent there.
template <int NT, int R, int LIM, bool SO, int MK, int OPT>
__global__ void __launch_bounds__(NT, kXMinBlocks) xsweep_t_kernel(GridDev g) {
  static_assert(R % 2 == 0, "rows come in pairs");
  __shared__ XSmem<NT> S;
  const Ctl* ctl = g.ctl;
  if (ctl->done) return;
  const int cur = ctl->cur;
  double* T = buffer(g, cur == 2 ? 0 : cur + 1);
  const int i0 = 1 + blockIdx.x * (NT - 4);
  const int i = i0 + threadIdx.x;
  double smax = 0.0;
  int bad = 0;
  for (int jb = 1 + blockIdx.y * R; jb <= g.my; jb += gridDim.y * R) {
    const int je = min(jb + R - 1, g.my);
    double prev[3];
    for (int j = jb; j <= je; ++j) {
      double v[3];
      const bool mine = line_sweep<NT, 0, LIM, SO, MK, OPT>(g, j, i0, S, smax, bad, v);
      __syncthreads();  // the shared arrays are reused by the next row
      if (!mine) continue;
      double* dst = T + (long long)(i + 1) * g.tpitch + (j + 1);
      if ((j - jb) & 1) {
        store_pair(dst - 1, g.tplane, prev, v);
      } else if (j == je) {
        store_cell(dst, g.tplane, v);
      } else {
#pragma unroll
        for (int me = 0; me < 3; ++me) prev[me] = v[me];
      }
    }
  }
  xsweep_finish<NT>(g, smax, bad, S);
}

// eta sweep: a CTA takes R consecutive columns (from an odd column) of one segment of NT-4 rows,
// reads them from the transposed buffer and writes the new values in the normal layout, two
// columns at a time; it also carries the pre-step ghost cells next to its cells into the new
// buffer (main.f90:210 vs :246).
template <int NT, int R, int LIM, bool SO, int MK, int OPT>
__global__ void __launch_bounds__(NT, kXMinBlocks) ysweep_t_kernel(GridDev g) {
  static_assert(R % 2 == 0, "columns come in pairs");
  __shared__ XSmem<NT> S;
  Ctl* ctl = g.ctl;
  if (ctl->done) return;
  if (!eta_valid(g)) return;
  const int cur = ctl->cur;
  const double* pre = buffer(g, cur);
  double* Y = buffer(g, cur == 0 ? 2 : cur - 1);
  const int mx = g.mx, my = g.my;
  const long long P = g.pitch;
  const int j0 = 1 + blockIdx.x * (NT - 4);
  const int j1 = min(j0 + NT - 5, my);
  const int t = threadIdx.x;
  const int j = j0 + t;
  double smax = 0.0;
  int bad = 0;
  for (int ib = 1 + blockIdx.y * R; ib <= mx; ib += gridDim.y * R) {
    const int ie = min(ib + R - 1, mx);
    double prev[3];
    for (int i = ib; i <= ie; ++i) {
      double v[3];
      const bool mine = line_sweep<NT, 1, LIM, SO, MK, OPT>(g, i, j0, S, smax, bad, v);
      __syncthreads();  // the shared arrays are reused by the next column
      if (mine) {
        double* dst = Y + (long long)(j + 1) * P + (i + 1);
        if ((i - ib) & 1) {
          store_pair(dst - 1, g.plane, prev, v);
        } else if (i == ie) {
          store_cell(dst, g.plane, v);
        } else {
#pragma unroll
          for (int me = 0; me < 3; ++me) prev[me] = v[me];
        }
        if (i == 1 || i == mx) {  // the ghost columns beside this row
          const long long o = (long long)(j + 1) * P + (i == 1 ? 0 : mx + 2);
#pragma unroll
          for (int me = 0; me < 3; ++me) {
            Y[o + me * g.plane] = pre[o + me * g.plane];
            Y[o + 1 + me * g.plane] = pre[o + 1 + me * g.plane];
          }
        }
      }
      // the ghost rows below and above this column
      const int gr = t < 2 && j0 == 1 ? t - 1 : (t >= 2 && t < 4 && j1 == my ? my + t - 1 : -9);
      if (gr != -9) {
        const long long o = (long long)(gr + 1) * P + (i + 1);
#pragma unroll
        for (int me = 0; me < 3; ++me) Y[o + me * g.plane] = pre[o + me * g.plane];
      }
    }
  }
  block_max_to<NT>(&ctl->smax_y, smax, S.red);
  if (bad) atomicOr(&ctl->status, bad);
}

// The shortcuts' range argument assumes g in [2^-20, 2^20] (pcl_fp64.cuh: kOptFastDiv).
inline bool fast_div_ok(const GridDev& g) { return g.grav >= 0x1p-20 && g.grav <= 0x1p20; }

// Uniform grids run both sweeps through the transposed intermediate; mapped grids (per-cell
// metric arrays in the normal layout) the row kernel and the eta register window.
inline bool transposed(const GridDev& g) { return g.tpitch > 0 && g.metric != kMetricMapped; }

template <int LIM, bool SO, int MK>
void launch_x_t(const GridDev& g, cudaStream_t st) {
  const int rb = (g.my + kXRows - 1) / kXRows;
  dim3 gx((g.mx + (kXT - 4) - 1) / (kXT - 4), rb < 65535 ? rb : 65535);
  if constexpr (MK != kMetricMapped) {
    if (transposed(g)) {
      if (fast_div_ok(g))
        xsweep_t_kernel<kXT, kXRows, LIM, SO, MK, kOptFastDiv><<<gx, kXT, 0, st>>>(g);
      else
        xsweep_t_kernel<kXT, kXRows, LIM, SO, MK, 0><<<gx, kXT, 0, st>>>(g);
      return;
    }
  }
  if (fast_div_ok(g))
    xsweep_fp64_kernel<kXT, LIM, SO, MK, kXRows, kOptFastDiv><<<gx, kXT, 0, st>>>(g);
  else
    xsweep_fp64_kernel<kXT, LIM, SO, MK, kXRows><<<gx, kXT, 0, st>>>(g);
}
template <int LIM, bool SO, int MK>
void launch_y_t(const GridDev& g, cudaStream_t st) {
  if constexpr (MK != kMetricMapped) {
    if (transposed(g)) {
      const int cb = (g.mx + kXRows - 1) / kXRows;
      dim3 gy((g.my + (kXT - 4) - 1) / (kXT - 4), cb < 65535 ? cb : 65535);
      if (fast_div_ok(g))
        ysweep_t_kernel<kXT, kXRows, LIM, SO, MK, kOptFastDiv><<<gy, kXT, 0, st>>>(g);
      else
        ysweep_t_kernel<kXT, kXRows, LIM, SO, MK, 0><<<gy, kXT, 0, st>>>(g);
      return;
    }
  }
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
