// pcl_launch.h -- host-side launchers of the device kernels (one translation unit each).
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {

// time-control operations run by a single device thread (kernels_aux.cu)
enum TimeOp : int {
  kOpInit = 0,            // derive dt/d_xi, dt/d_eta; clear the per-attempt words
  kOpFinalizeSolve = 1,   // CFL and accept/reject of the attempt (MOD_solve.f90:101-174)
  kOpUpdateTime = 2,      // updateTime(arg != 0) (MOD_time_control.f90:153-243)
  kOpResetCFL = 3,        // reset_CFL (MOD_time_control.f90:270-279)
  kOpAdvanceSnapshot = 4, // advance_snapshot_index
  kOpFullStep = 5,        // finalize + the main-loop branch of main.f90:210-275
  kOpSetDt = 6,           // dt = value (host override, e.g. to force a rejection)
  kOpSetPause = 7,        // pause_on_snapshot = arg, paused = 0
};

void launch_sweeps_fp64(const GridDev& g, cudaStream_t st);
// the FP64 sweeps of the equation modules other than the specialised shallow water
void launch_xsweep_gen(const GridDev& g, cudaStream_t st);
void launch_ysweep_gen(const GridDev& g, cudaStream_t st);
void launch_xsweep_fp64(const GridDev& g, cudaStream_t st);
void launch_ysweep_fp64(const GridDev& g, cudaStream_t st);
// the eta-sweep shape the specialised FP64 launcher runs for g (kEtaWindow or kEtaBand)
int eta_shape_of(const GridDev& g);
void launch_timectl(const GridDev& g, int op, int arg, double value, cudaStream_t st);
void launch_ghost(const GridDev& g, int force, cudaStream_t st);
void launch_upload(const GridDev& g, const double* staging_aos, cudaStream_t st);
void launch_dam_ic(const GridDev& g, double radius, double h_in, double h_out, double x0, double y0,
                   cudaStream_t st);
void launch_row_sums(const GridDev& g, double* partial /* 3 per interior row */, cudaStream_t st);
void launch_download(const GridDev& g, double* staging_aos, cudaStream_t st);
// Sets g.ctl->nonunit_metric (cleared beforehand) when a capacity of cells -1 .. m+2 or an
// interior length ratio differs from 1.0 as the sweeps compute them.
void launch_metric_check(const GridDev& g, cudaStream_t st);

}  // namespace pcl
