// kernels_aux.cu -- device time control, ghost-cell fill and the AoS <-> SoA transposes at the
// C-ABI boundary.  Built with --fmad=false: the time-control arithmetic must round exactly as
// time_control/MOD_time_control.f90 does.
#include <cuda_runtime.h>
#include <math.h>

#include "pcl_launch.h"
#include "pcl_types.h"

namespace pcl {

// ------------------------------------------------------------------------------------------
// time control (one thread)
// ------------------------------------------------------------------------------------------
__device__ double next_snapshot(const Ctl* c) {
  int k = c->snapshot_index;
  if (k > c->n_snapshots) k = c->n_snapshots;  // the reference's loop ends at time_final first
  return c->snap_times[k - 1];
}

__device__ void derive_dtod(Ctl* c, const GridDev& g) {
  c->dtod_x = c->dt / g.dxi;  // dt_over_delta (MOD_solve.f90:202-204)
  c->dtod_y = c->dt / g.deta;
}

// updateTime (MOD_time_control.f90:153-243); returns false on end_program
__device__ bool update_time(Ctl* c, bool step_valid) {
  double change_factor, dt_step;
  c->dt_previous = c->dt;
  dt_step = c->dt;
  if (step_valid) {
    if (c->adaptive) {
      if (c->CFL > 0.0)
        change_factor = c->CFL_target / c->CFL;
      else
        change_factor = 1.0;
      if (change_factor >= c->growth)
        change_factor = c->growth;
      else if (fabs(change_factor - 1.0) <= c->time_precision)
        change_factor = 1.0;
      dt_step = c->dt_previous * change_factor;
    }
    const double ts = next_snapshot(c);
    if (c->time + dt_step > ts) {
      dt_step = ts - c->time;
      c->snapshot_exception = 1;
    } else {
      c->snapshot_exception = 0;
    }
  } else {
    if (!c->adaptive) return false;
    dt_step = c->emergency * c->dt;
  }
  if (dt_step > c->dt_max) dt_step = c->dt_max;
  if (dt_step < c->dt_min) {
    if (!c->adaptive && !c->snapshot_exception) return false;
    dt_step = c->dt_min;
  }
  if (step_valid) c->time = c->time + dt_step;
  c->dt = dt_step;
  return true;
}

// CFL reduction result and accept/reject (MOD_solve.f90:101-174): CFL_local is the running
// max over both sweeps and t_ctrl%CFL = max(CFL, CFL_local) after each sweep.
__device__ void finalize_solve(Ctl* c, const GridDev& g) {
  const double sx = __longlong_as_double((long long)c->smax_x);
  const double sy = __longlong_as_double((long long)c->smax_y);
  double cfl_local = sx * c->dt / g.dxi;
  c->cfl_x = cfl_local;
  c->CFL = fmax(c->CFL, cfl_local);
  const bool vx = c->CFL_target / c->CFL >= c->shrink;
  c->valid_x = vx;
  bool ok = vx;
  if (vx) {
    cfl_local = fmax(cfl_local, sy * c->dt / g.deta);
    c->CFL = fmax(c->CFL, cfl_local);
    ok = c->CFL_target / c->CFL >= c->shrink;
  }
  c->cfl_y = cfl_local;
  c->ierr = ok ? 1 : -1;
  if (ok) c->cur = c->cur == 0 ? 2 : c->cur - 1;  // the eta-swept buffer becomes current
  c->smax_x = 0ull;
  c->smax_y = 0ull;
  c->attempts += 1;
}

__device__ void reset_cfl(Ctl* c) {
  c->CFL_previous_timestep = c->CFL;
  c->CFL = 0.0;
}

__device__ void refresh_done(Ctl* c) {
  c->done = (c->time >= c->time_final) || (c->max_accepted > 0 && c->accepted >= c->max_accepted) ||
            (c->status != 0);
}

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
    case kOpFullStep: {
      if (c->done) {
        c->ierr = 0;  // no attempt: the ghost fill that follows is skipped
        break;
      }
      const double dt_used = c->dt;
      finalize_solve(c, g);
      const double cfl = c->CFL;
      bool ok = true;
      if (c->ierr < 0) {
        ok = update_time(c, false);  // dt *= 0.25; buffer cur was never touched
        reset_cfl(c);
      } else {
        // integrate_source_term: phi = 0 leaves finite q unchanged (MOD_solve.f90:295-336)
        ok = update_time(c, true);
        if (ok && c->time >= next_snapshot(c) && c->snapshot_index <= c->n_snapshots) c->snapshot_index += 1;
        reset_cfl(c);
        c->accepted += 1;
      }
      if (!ok) c->status |= kStatusFatalDt;
      derive_dtod(c, g);
      if (c->log && c->log_len < c->log_cap) {
        StepLogEntry& e = c->log[c->log_len];
        e.dt = dt_used;
        e.cfl = cfl;
        e.time = c->time;
        e.dt_next = c->dt;
        e.ierr = c->ierr;
        e.snapshot_index = c->snapshot_index;
        c->log_len += 1;
      }
      refresh_done(c);
      break;
    }
    default:
      break;
  }
}

void launch_timectl(const GridDev& g, int op, int arg, double value, cudaStream_t st) {
  timectl_kernel<<<1, 1, 0, st>>>(g, op, arg, value);
}

// ------------------------------------------------------------------------------------------
// ghost fill: update_rank_boundaries -> apply_physical_boundaries
// (user_subroutines/SMOD_boundary_conditions.f90:58-213).  Corners are never written.
// Code 1 (BC_USER, which aborts in the reference) is a reflective wall here: the two ghost
// layers mirror the two nearest interior cells with the normal momentum negated.
// ------------------------------------------------------------------------------------------
__global__ void ghost_kernel(GridDev g, int force) {
  const Ctl* c = g.ctl;
  if (!force && c->ierr != 1) return;
  const int mx = g.mx, my = g.my;
  const int n = max(mx, my);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int side = tid / (2 * n);
  const int rem = tid - side * 2 * n;
  const int layer = rem / n;
  const int idx = 1 + rem - layer * n;  // 1-based position along the side
  if (side >= 4) return;
  const long long P = g.pitch;
  double* b = buffer(g, c->cur);
  const int bc = g.bc[side];
  if (side < 2) {  // xi boundaries, rows j = 1 .. m_eta
    const int j = idx;
    if (j > my) return;
    const int i = side == 0 ? -1 + layer : mx + 1 + layer;
    const int i1 = side == 0 ? 1 : mx;          // nearest interior cell
    const int i2 = side == 0 ? 2 : mx - 1;      // second interior cell
    const int im = side == 0 ? 1 - i : 2 * mx + 1 - i;
    const double xg = __ldg(g.colm + (i + 1) * kColMetrics + 3);
    const double x1 = __ldg(g.colm + (i1 + 1) * kColMetrics + 3);
    const double x2 = __ldg(g.colm + (i2 + 1) * kColMetrics + 3);
    for (int me = 0; me < 3; ++me) {
      double* p = b + me * g.plane + (long long)(j + 1) * P;
      double v;
      if (bc == 2) {
        v = p[i1 + 1];
      } else if (bc == 3) {
        // deriv_2p(x_a, x_b, y_a, y_b) = (y_b - y_a)/(x_b - x_a) with (a, b) = (ilow, ilow+1)
        // on the left and (ihigh-1, ihigh) on the right (SMOD_boundary_conditions.f90:101-104)
        const double ya = side == 0 ? p[i1 + 1] : p[i2 + 1];
        const double yb = side == 0 ? p[i2 + 1] : p[i1 + 1];
        const double xa = side == 0 ? x1 : x2;
        const double xb = side == 0 ? x2 : x1;
        v = p[i1 + 1] + (yb - ya) / (xb - xa) * (xg - x1);
      } else {
        v = me == 1 ? -p[im + 1] : p[im + 1];
      }
      p[i + 1] = v;
    }
  } else {  // eta boundaries, columns i = 1 .. m_xi
    const int i = idx;
    if (i > mx) return;
    const int j = side == 2 ? -1 + layer : my + 1 + layer;
    const int j1 = side == 2 ? 1 : my;
    const int j2 = side == 2 ? 2 : my - 1;
    const int jm = side == 2 ? 1 - j : 2 * my + 1 - j;
    const double yg = __ldg(g.rowm + (j + 1) * kRowMetrics + 3);
    const double y1 = __ldg(g.rowm + (j1 + 1) * kRowMetrics + 3);
    const double y2 = __ldg(g.rowm + (j2 + 1) * kRowMetrics + 3);
    for (int me = 0; me < 3; ++me) {
      double* p = b + me * g.plane + (i + 1);
      double v;
      if (bc == 2) {
        v = p[(long long)(j1 + 1) * P];
      } else if (bc == 3) {
        const double va = side == 2 ? p[(long long)(j1 + 1) * P] : p[(long long)(j2 + 1) * P];
        const double vb = side == 2 ? p[(long long)(j2 + 1) * P] : p[(long long)(j1 + 1) * P];
        const double ya = side == 2 ? y1 : y2;
        const double yb = side == 2 ? y2 : y1;
        v = p[(long long)(j1 + 1) * P] + (vb - va) / (yb - ya) * (yg - y1);
      } else {
        v = me == 2 ? -p[(long long)(jm + 1) * P] : p[(long long)(jm + 1) * P];
      }
      p[(long long)(j + 1) * P] = v;
    }
  }
}

void launch_ghost(const GridDev& g, int force, cudaStream_t st) {
  const int n = g.mx > g.my ? g.mx : g.my;
  const int total = 4 * 2 * n;
  ghost_kernel<<<(total + 255) / 256, 256, 0, st>>>(g, force);
}

// ------------------------------------------------------------------------------------------
// AoS (reference layout vars(3, -1:m+2, -1:m+2)) <-> SoA planes.  Upload writes all three
// rotation buffers so every buffer carries the initial corner ghosts, which the reference
// never overwrites.
// ------------------------------------------------------------------------------------------
__global__ void upload_kernel(GridDev g, const double* __restrict__ aos) {
  const int ni = g.mx + 4, nj = g.my + 4;
  const long long n = (long long)ni * nj;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(c / ni), ii = (int)(c - (long long)jj * ni);
    const long long o = (long long)jj * g.pitch + ii;
    const double h = aos[c * 3], hu = aos[c * 3 + 1], hv = aos[c * 3 + 2];
    for (int b = 0; b < 3; ++b) {
      buffer(g, b)[o] = h;
      buffer(g, b)[o + g.plane] = hu;
      buffer(g, b)[o + 2 * g.plane] = hv;
    }
  }
}

__global__ void download_kernel(GridDev g, double* __restrict__ aos) {
  const int ni = g.mx + 4, nj = g.my + 4;
  const long long n = (long long)ni * nj;
  const double* b = buffer(g, g.ctl->cur);
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
    const int jj = (int)(c / ni), ii = (int)(c - (long long)jj * ni);
    const long long o = (long long)jj * g.pitch + ii;
    aos[c * 3] = b[o];
    aos[c * 3 + 1] = b[o + g.plane];
    aos[c * 3 + 2] = b[o + 2 * g.plane];
  }
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
