// pcl_types.h -- host/device shared types of the paraclaws_b200 CUDA path.
//
// Device state of one grid ("instance"):
//   * three state buffers (rotation: current / x-swept / y-swept), each num_equations SoA
//     planes (shallow water: h, hu, hv) of (m_eta+4) rows x pitch doubles; cell (i, j) of the
//     reference's 1-based padded block (i, j = -1 .. m+2) sits at plane[(j+1)*pitch + (i+1)].
//     pitch is a multiple of 32 doubles so every row starts on a 256-byte boundary.
//   * per-row and per-column mesh tables (uniform mapping: the capacity kappa(i,j) is rebuilt
//     in-kernel from them in the reference's operation order);
//   * a control block: the reference's time_control (time_control/MOD_time_control.f90:16-66)
//     plus the per-attempt reduction words, the buffer index and the status word.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define PCL_HD __host__ __device__
#else
#define PCL_HD
#endif

namespace pcl {

constexpr double kUdPrecision = 1e-10;  // constant/MOD_constants.f90:18
constexpr int kMaxSnapshots = 4096;
constexpr int kRowMetrics = 4;  // per row j:   p1 = 0.5*(e1+e1), p3 = 0.5*(e3+e3), gamma_xi, eta centre
constexpr int kColMetrics = 4;  // per column i: d = c1-c2, d' = c2-c1, gamma_eta, xi centre

// status bits (device); the C ABI maps them to negative codes
enum : int {
  kStatusNaN = 1,
  kStatusNegDepth = 2,
  kStatusFatalDt = 4,
  kStatusTimeout = 8,
};

// precision forms
enum : int { kPrecFP64 = 0, kPrecMixed = 1 };

// How the FP64 sweeps obtain the mesh metrics (capacity kappa, length ratios gamma):
//   kMetricTable  uniform grid: kappa rebuilt per cell from the row/column tables
//   kMetricUnit   uniform grid whose kappa and gamma are all exactly 1.0 (identities dropped)
//   kMetricMapped mapped grid: per-cell arrays kap, lrx, lry (the reference's capacity,
//                 length_ratio_xi(1,:,:), length_ratio_eta(1,:,:))
enum : int { kMetricTable = 0, kMetricUnit = 1, kMetricMapped = 2 };

// Shape of the FP64 eta sweep (same results for every shape): chosen by grid size, or forced
// (pcl_set_sweep_shape).  Column windows: one thread per column over a strip of rows; bands:
// shared-memory phases along the columns of 4-column bands.
enum : int { kEtaAuto = 0, kEtaWindow = 1, kEtaBand = 2 };

struct StepLogEntry {   // one attempted step, as main.f90 prints it
  double dt;            // dt used by the attempt
  double cfl;           // CFL of the attempt (t_ctrl%CFL before reset_CFL)
  double time;          // time after updateTime
  double dt_next;       // dt after updateTime
  int ierr;             // 1 accepted, -1 rejected
  int snapshot_index;   // after the snapshot check
};

struct Ctl {
  // ---- time_control ----
  double time, time_initial, time_final;
  double dt, dt_previous, dt_max, dt_min;
  double time_precision, CFL, CFL_target, CFL_previous_timestep;
  double shrink, growth, emergency;
  int snapshot_index;        // 1-based, as current_snapshot_index
  int n_snapshots;
  int adaptive, snapshot_exception;
  // ---- per attempt ----
  double dtod_x, dtod_y;     // dt/d_xi, dt/d_eta for the current dt
  double dt_step;            // dt of the attempt being finalised (integrate_source_term's get_dt())
  unsigned long long smax_x, smax_y;  // IEEE bits of max wave speed s2 per sweep (>= 0)
  double cfl_x, cfl_y;       // CFL_local after the xi sweep / after both sweeps
  int valid_x;               // xi-sweep validity (early reject, MOD_solve.f90:107-120)
  int items_done;            // work items of the attempt finished so far (kernels whose last CTA
                             // runs the time control); the last one resets it
  int ierr;                  // last attempt: 1 accepted, -1 rejected, 0 none yet
  int cur;                   // index of the current state buffer (0..2)
  int done;                  // time >= time_final, accepted-step cap reached, or error
  int status;                // kStatus* bits
  int nonunit_metric;        // set by the metric check when some kappa or gamma is not exactly 1
  int pause_on_snapshot;     // pcl_advance_to_snapshot: stop after the attempt that reaches a snapshot
  int paused;                // set then; counts as done until the host clears it
  long long attempts, accepted, max_accepted;
  long long log_cap, log_len;
  StepLogEntry* log;         // optional device log (may be null)
  double snap_times[kMaxSnapshots];
};

// Everything a sweep kernel needs about one grid.
struct GridDev {
  double* state;             // 3 state buffers; plane p of buffer b at state + b*bufstride + p*plane
  long long bufstride;       // doubles per buffer (neq planes)
  const double* rowm;        // (m_eta+4) x kRowMetrics
  const double* colm;        // (m_xi+4) x kColMetrics
  Ctl* ctl;
  long long plane;           // doubles per plane
  int mx, my, pitch;
  int bc[4];                 // xi_low, xi_high, eta_low, eta_high (1 wall, 2 zero grad., 3 const. grad.)
  int second_order, limiter; // limiter 0: unlimited correction; 1..4 by code
  int metric;                // kMetric*
  int user_bc;               // 1: sides coded 1 are filled by the host's user hook, not the wall
  int eq;                    // equation module (pcl_equations.h); 0: the specialised shallow water,
                             // -1: none chosen yet (contexts of num_equations != 3)
  int neq;                   // planes per buffer: num_equations (3 for every path but the generic one)
  double eqp[2];             // its parameters (shallow water: g)
  int eta_shape;             // kEta*: the FP64 eta sweep's shape
  double dxi, deta, area_scale /* d_xi*d_eta */, grav;
  // kMetricMapped only: per-cell metrics, cell (i, j) at [(j+1)*pitch + (i+1)]
  const double* kap;         // capacity(i, j)
  const double* lrx;         // length ratio of the xi face between cells i-1 and i
  const double* lry;         // length ratio of the eta face between cells j-1 and j
};

PCL_HD inline long long cell_index(int pitch, int i, int j) {
  return (long long)(j + 1) * pitch + (i + 1);
}

PCL_HD inline double* buffer(const GridDev& g, int b) { return g.state + (long long)b * g.bufstride; }

}  // namespace pcl
