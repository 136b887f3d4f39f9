// pcl_timectl.cuh -- the reference's time control on the device, shared by the single-grid
// time-control kernel (kernels_aux.cu) and the per-instance finalisation of the batched kernels.
// Restates time_control/MOD_time_control.f90 in FP64; no expression here has a multiply feeding
// an add, so it rounds the same whether or not its translation unit contracts.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "pcl_types.h"

namespace pcl {

__device__ __forceinline__ double next_snapshot(const Ctl* c) {
  int k = c->snapshot_index;
  if (k > c->n_snapshots) k = c->n_snapshots;  // the reference's loop ends at time_final first
  return c->snap_times[k - 1];
}

__device__ __forceinline__ void derive_dtod(Ctl* c, const GridDev& g) {
  c->dtod_x = c->dt / g.dxi;  // dt_over_delta (MOD_solve.f90:202-204)
  c->dtod_y = c->dt / g.deta;
}

// updateTime (MOD_time_control.f90:153-243); returns false on end_program
__device__ __forceinline__ bool update_time(Ctl* c, bool step_valid) {
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
__device__ __forceinline__ void finalize_solve(Ctl* c, const GridDev& g) {
  c->dt_step = c->dt;
  // the reduction words are written by atomics from other CTAs of the same (batched) launch:
  // read them at L2, past this SM's L1
  const double sx = __longlong_as_double((long long)__ldcg(&c->smax_x));
  const double sy = __longlong_as_double((long long)__ldcg(&c->smax_y));
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
  // A bounded wait that gave up (kStatusTimeout) voids the attempt: some of its cells were never
  // written, so the eta-swept buffer must not become current.  The host sees the status.
  if (__ldcg(&c->status) & kStatusTimeout) ok = false;
  c->ierr = ok ? 1 : -1;
  if (ok) c->cur = c->cur == 0 ? 2 : c->cur - 1;  // the eta-swept buffer becomes current
  c->smax_x = 0ull;
  c->smax_y = 0ull;
  c->attempts += 1;
}

__device__ __forceinline__ void reset_cfl(Ctl* c) {
  c->CFL_previous_timestep = c->CFL;
  c->CFL = 0.0;
}

__device__ __forceinline__ void refresh_done(Ctl* c) {
  c->done = (c->time >= c->time_final) || (c->max_accepted > 0 && c->accepted >= c->max_accepted) ||
            (__ldcg(&c->status) != 0) || c->paused;
}

// Everything main.f90:210-275 does after the sweeps of one attempt: accept/reject, updateTime,
// the snapshot index, reset_CFL, and one step-log record.  Leaves ierr = 0 when nothing ran
// (the ghost fill that follows then skips).
__device__ __forceinline__ void full_step(Ctl* c, const GridDev& g) {
  if (c->done) {
    c->ierr = 0;
    return;
  }
  const double dt_used = c->dt;
  finalize_solve(c, g);
  if (__ldcg(&c->status) & kStatusTimeout) {  // void attempt: no time update, no ghost fill, no log
    c->ierr = 0;
    reset_cfl(c);
    refresh_done(c);
    return;
  }
  const double cfl = c->CFL;
  bool ok = true;
  if (c->ierr < 0) {
    ok = update_time(c, false);  // dt *= 0.25; buffer cur was never touched
    reset_cfl(c);
  } else {
    // integrate_source_term: phi = 0 leaves finite q unchanged (MOD_solve.f90:295-336)
    ok = update_time(c, true);
    if (ok && c->time >= next_snapshot(c) && c->snapshot_index <= c->n_snapshots) {
      c->snapshot_index += 1;
      if (c->pause_on_snapshot) c->paused = 1;  // main.f90:256-268 writes the snapshot here
    }
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
}

}  // namespace pcl
