// kernels_aux.cu -- device time control, ghost-cell fill and the AoS <-> SoA transposes at the
// C-ABI boundary.  Built with --fmad=false: the time-control arithmetic must round exactly as
// time_control/MOD_time_control.f90 does.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>

#include "pcl_fp64.cuh"
#include "pcl_ghost.cuh"
#include "pcl_launch.h"
#include "pcl_timectl.cuh"
#include "pcl_types.h"

namespace pcl {

// ------------------------------------------------------------------------------------------
// time control (one thread; the logic lives in pcl_timectl.cuh)
// ------------------------------------------------------------------------------------------
__global__ void timectl_kernel(GridDev g, int op, int arg, double value) {
  Ctl* c = g.ctl;
  switch (op) {
    case kOpInit:
      c->smax_x = c->smax_y = 0ull;
      derive_dtod(c, g);
      refresh_done(c);
      break;
    case kOpFinalizeSolve:
      finalize_solve(c, g);
      break;
    case kOpUpdateTime:
      if (!update_time(c, arg != 0)) c->status |= kStatusFatalDt;
      if (arg != 0) c->accepted += 1;
      derive_dtod(c, g);
      refresh_done(c);
      break;
    case kOpResetCFL:
      reset_cfl(c);
      break;
    case kOpAdvanceSnapshot:
      c->snapshot_index += 1;
      break;
    case kOpSetDt:
      c->dt = value;
      derive_dtod(c, g);
      break;
    case kOpFullStep:
      full_step(c, g);
      break;
    case kOpSetPause:
      c->pause_on_snapshot = arg;
      c->paused = 0;
      refresh_done(c);
      break;
    default:
      break;
  }
}

void launch_timectl(const GridDev& g, int op, int arg, double value, cudaStream_t st) {
  timectl_kernel<<<1, 1, 0, st>>>(g, op, arg, value);
}

// ------------------------------------------------------------------------------------------
// metric check: on grids whose corner coordinates are exact (e.g. 2^k cells on [-1, 1]) every
// capacity evaluates to exactly 1 and every length ratio is exactly 1; the sweeps then drop
// the divisions by kappa and the multiplications by gamma, which are exact identities there.
// ------------------------------------------------------------------------------------------
__global__ void metric_check_kernel(GridDev g) {
  const int ni = g.mx + 4, nj = g.my + 4;
  const long long n = (long long)ni * nj;
  int bad = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(k % ni) - 1, j = (int)(k / ni) - 1;
    if (capacity(g.rowm, g.colm, i, j, g.area_scale) != 1.0) bad = 1;
    if (i == 1 && j >= 1 && j <= g.my && g.rowm[(j + 1) * kRowMetrics + 2] != 1.0) bad = 1;
    if (j == 1 && i >= 1 && i <= g.mx && g.colm[(i + 1) * kColMetrics + 2] != 1.0) bad = 1;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(&g.ctl->nonunit_metric, 1);
}

void launch_metric_check(const GridDev& g, cudaStream_t st) {
  const long long n = (long long)(g.mx + 4) * (g.my + 4);
  const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
  metric_check_kernel<<<blocks, 256, 0, st>>>(g);
}

// ------------------------------------------------------------------------------------------
// ghost fill (the logic lives in pcl_ghost.cuh)
// ------------------------------------------------------------------------------------------
template <int N>
__global__ void ghost_kernel(GridDev g, int force) {
  const Ctl* c = g.ctl;
  if (!force && c->ierr != 1) return;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid < ghost_items(g)) ghost_item<N>(g, buffer(g, c->cur), tid);
}

void launch_ghost(const GridDev& g, int force, cudaStream_t st) {
  const int n = g.mx > g.my ? g.mx : g.my;
  const int total = 4 * 2 * n;
  const int blocks = (total + 255) / 256;
  if (g.neq == 1)
    ghost_kernel<1><<<blocks, 256, 0, st>>>(g, force);
  else if (g.neq == 4)
    ghost_kernel<4><<<blocks, 256, 0, st>>>(g, force);
  else
    ghost_kernel<3><<<blocks, 256, 0, st>>>(g, force);
}

// ------------------------------------------------------------------------------------------
// AoS (reference layout vars(neq, -1:m+2, -1:m+2)) <-> SoA planes.  Upload writes all three
// rotation buffers so every buffer carries the initial corner ghosts, which the reference
// never overwrites.
// ------------------------------------------------------------------------------------------
__global__ void upload_kernel(GridDev g, const double* __restrict__ aos) {
  const int ni = g.mx + 4, nj = g.my + 4, ne = g.neq;
  const long long n = (long long)ni * nj;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(c / ni), ii = (int)(c - (long long)jj * ni);
    const long long o = (long long)jj * g.pitch + ii;
    for (int p = 0; p < ne; ++p) {
      const double v = aos[c * ne + p];
      for (int b = 0; b < 3; ++b) buffer(g, b)[o + p * g.plane] = v;
    }
  }
}

__global__ void download_kernel(GridDev g, double* __restrict__ aos) {
  const int ni = g.mx + 4, nj = g.my + 4, ne = g.neq;
  const long long n = (long long)ni * nj;
  const double* b = buffer(g, g.ctl->cur);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(c / ni), ii = (int)(c - (long long)jj * ni);
    const long long o = (long long)jj * g.pitch + ii;
    for (int p = 0; p < ne; ++p) aos[c * ne + p] = b[o + p * g.plane];
  }
}

// ------------------------------------------------------------------------------------------
// set_initial_conditions of the dam-break example on the device
// (examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:34-46): h = h_in where
// sqrt(x^2 + y^2) < radius at the cell centre (shifted by x0, y0 when they are non-zero), else
// h_out; hu = hv = 0; the padded block including ghosts, into every rotation buffer.  The cell
// centres come from the mesh tables, so the bits equal the host generator's.
// ------------------------------------------------------------------------------------------
__global__ void dam_ic_kernel(GridDev g, double radius, double h_in, double h_out, double x0, double y0) {
  const int ni = g.mx + 4, nj = g.my + 4;
  const long long n = (long long)ni * nj;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(c / ni), ii = (int)(c - (long long)jj * ni);
    double x = __ldg(g.colm + ii * kColMetrics + 3);
    double y = __ldg(g.rowm + jj * kRowMetrics + 3);
    if (x0 != 0.0) x = x - x0;
    if (y0 != 0.0) y = y - y0;
    const double h = sqrt(x * x + y * y) < radius ? h_in : h_out;
    const long long o = (long long)jj * g.pitch + ii;
    for (int b = 0; b < 3; ++b) {
      buffer(g, b)[o] = h;
      buffer(g, b)[o + g.plane] = 0.0;
      buffer(g, b)[o + 2 * g.plane] = 0.0;
    }
  }
}

void launch_dam_ic(const GridDev& g, double radius, double h_in, double h_out, double x0, double y0, cudaStream_t st) {
  dam_ic_kernel<<<148 * 8, 256, 0, st>>>(g, radius, h_in, h_out, x0, y0);
}

// ------------------------------------------------------------------------------------------
// FP64 conservation sums over the interior: each block sums whole rows in a fixed order and
// writes one partial per row; the host adds the partials in row order, so the result does not
// depend on scheduling.
// ------------------------------------------------------------------------------------------
__global__ void row_sums_kernel(GridDev g, double* __restrict__ partial) {
  __shared__ double red[3][256];
  const int j = 1 + blockIdx.x;
  const double* b = buffer(g, g.ctl->cur) + (long long)(j + 1) * g.pitch;
  double s[3] = {0.0, 0.0, 0.0};
  for (int i = 1 + threadIdx.x; i <= g.mx; i += blockDim.x)
    for (int p = 0; p < 3; ++p) s[p] += b[p * g.plane + i + 1];
  for (int p = 0; p < 3; ++p) red[p][threadIdx.x] = s[p];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int p = 0; p < 3; ++p) red[p][threadIdx.x] += red[p][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int p = 0; p < 3; ++p) partial[(long long)blockIdx.x * 3 + p] = red[p][0];
}

void launch_row_sums(const GridDev& g, double* partial, cudaStream_t st) {
  row_sums_kernel<<<g.my, 256, 0, st>>>(g, partial);
}

void launch_upload(const GridDev& g, const double* staging_aos, cudaStream_t st) {
  upload_kernel<<<148 * 8, 256, 0, st>>>(g, staging_aos);
}
void launch_download(const GridDev& g, double* staging_aos, cudaStream_t st) {
  download_kernel<<<148 * 8, 256, 0, st>>>(g, staging_aos);
}

}  // namespace pcl
