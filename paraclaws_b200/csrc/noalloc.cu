// noalloc.cu -- one attempted FP64 step for callers that cannot allocate device memory.
//
// The regular entry points keep their scratch (the xi-swept intermediate state, the mesh tables
// and the time-control block with its reduction words) in memory that pcl_create allocates.
// Some hosts cannot do that: a solver embedded in a larger application whose device memory is
// owned by someone else's pool, a step called from a time-critical loop that must not pay the
// device-wide synchronisation cudaFree implies, or a batch system that accounts for every byte
// of device memory before the job starts.  pcl_solve_dimensional_split_noalloc serves them: the
// caller passes the input and output states in its own device memory, and all scratch lives in
// one file-scope __device__ array, sized for grids of at most kNoAllocMaxSide^2 interior cells.
//
// The array is part of the library image: every GPU that loads the library holds it
// (about 1.6 MB) until the process exits.  Calls share it and it keeps the last call's contents,
// so every call rewrites what the step reads before reading it (control block, tables, input
// copy); two calls whose work overlaps on the GPU (different streams or devices of one process
// that run at the same time on the same device) race on the array.
//
// The array's device address is looked up once per device and kept: it belongs to that device's
// primary context and stays valid while the context lives.  A cudaDeviceReset on the device ends
// the context, and the kept address with it: a process that resets a device must not call this
// entry point on it afterwards.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/paraclaws_b200.h"
#include "pcl_launch.h"
#include "pcl_types.h"

// mesh tables in the reference's operation order (capi.cu)
extern "C" void build_tables(const pcl_solver_control* c, double dxi, double deta, std::vector<double>& rowm,
                             std::vector<double>& colm);

namespace {

constexpr int kNoAllocMaxSide = 128;                        // largest m_xi and m_eta
constexpr int kMaxPitch = (kNoAllocMaxSide + 4 + 31) / 32 * 32;
constexpr int kMaxRows = kNoAllocMaxSide + 4;
constexpr long long kMaxPlane = (long long)kMaxPitch * kMaxRows;
constexpr long long kStateDoubles = 9 * kMaxPlane;           // 3 rotation buffers x 3 planes
constexpr long long kTableOffset = kStateDoubles;
constexpr long long kTableDoubles = 2LL * kMaxRows * 4;      // row and column mesh tables
constexpr long long kCtlOffset = (kTableOffset + kTableDoubles + 31) / 32 * 32;
constexpr long long kCtlDoubles = (sizeof(pcl::Ctl) + sizeof(double) - 1) / sizeof(double);
constexpr long long kScratchDoubles = kCtlOffset + kCtlDoubles;
constexpr int kMaxDevices = 64;

// bytes of the control block the kernels of one attempt read and write (not the snapshot table)
constexpr size_t kCtlHot = offsetof(pcl::Ctl, snap_times);

std::mutex g_setup_mu;
double* g_scratch_addr[kMaxDevices] = {};

}  // namespace

// The scratch array.  Host code must not use the name as an address: it only stands in for
// the device symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Once per device, with that device current: look up the device address of the array.
static int scratch_address(int device, double** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "pcl_solve_dimensional_split_noalloc: cudaGetSymbolAddress failed on device %d: %s\n",
                   device, cudaGetErrorString(e));
      return PCL_ERR_CUDA;
    }
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return PCL_OK;
}

// True when every capacity of cells -1 .. m+2 and every interior face length ratio of the
// uniform grid is exactly 1.0, computed from the tables with the sweeps' own expression
// (pcl_fp64.cuh: capacity) without contraction, as the regular contexts' metric check does on
// the device.  The sweeps then drop those identity operations (same bits, fewer instructions).
static bool unit_metric(const std::vector<double>& rowm, const std::vector<double>& colm, int mx, int my,
                        double area_scale) {
  for (int j = -1; j <= my + 2; ++j)
    for (int i = -1; i <= mx + 2; ++i) {
      const double* r = &rowm[(size_t)(j + 1) * pcl::kRowMetrics];
      const double* c = &colm[(size_t)(i + 1) * pcl::kColMetrics];
      if ((r[0] * c[0] + r[1] * c[1]) / area_scale != 1.0) return false;
    }
  for (int j = 1; j <= my; ++j)
    if (rowm[(size_t)(j + 1) * pcl::kRowMetrics + 2] != 1.0) return false;
  for (int i = 1; i <= mx; ++i)
    if (colm[(size_t)(i + 1) * pcl::kColMetrics + 2] != 1.0) return false;
  return true;
}

static int status_code(int st) {
  if (st & pcl::kStatusNaN) return PCL_ERR_NAN;
  if (st & pcl::kStatusNegDepth) return PCL_ERR_NEG_DEPTH;
  return PCL_OK;
}

#define NA_CK(call)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess) {                                                                            \
      std::fprintf(stderr, "pcl_solve_dimensional_split_noalloc: %s: %s\n", #call, cudaGetErrorString(e_)); \
      rc = PCL_ERR_CUDA;                                                                                \
      goto done;                                                                                        \
    }                                                                                                   \
  } while (0)

extern "C" int pcl_solve_dimensional_split_noalloc(const pcl_solver_control* c, int device, void* stream,
                                                   const double* d_in, double* d_out, long long ld, double dt,
                                                   double* cfl, int* ierr) {
  if (!c || !d_in || !d_out || !ierr) return PCL_ERR_BADARG;
  if (c->m_xi < 2 || c->m_eta < 2 || c->m_xi > kNoAllocMaxSide || c->m_eta > kNoAllocMaxSide) {
    std::fprintf(stderr,
                 "pcl_solve_dimensional_split_noalloc: grid %d x %d is outside 2..%d per direction, the size "
                 "of its static scratch; use pcl_create/pcl_solve_dimensional_split for larger grids\n",
                 c->m_xi, c->m_eta, kNoAllocMaxSide);
    return PCL_ERR_BADARG;
  }
  if (c->num_equations != 3 || c->num_waves != 2 || c->num_ghost != 2 || c->precision_mode != PCL_PREC_FP64 ||
      ld < c->m_xi + 4 || !(dt > 0.0) || device < 0 || device >= kMaxDevices)
    return PCL_ERR_BADARG;
  for (int b : {c->bc_xi_lower, c->bc_xi_upper, c->bc_eta_lower, c->bc_eta_upper})
    if (b < 1 || b > 3) return PCL_ERR_BADARG;
  if (c->higher_order_flux_correction && c->use_limiter && (c->limiter_method < 1 || c->limiter_method > 4))
    return PCL_ERR_BADARG;

  int rc = PCL_OK;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* base = nullptr;
  pcl::GridDev g{};
  pcl::Ctl h{};
  std::vector<double> rowm, colm;
  const int mx = c->m_xi, my = c->m_eta;
  const int pitch = (mx + 4 + 31) / 32 * 32;
  const long long plane = (long long)pitch * (my + 4);
  const double dxi = (c->xi_max - c->xi_min) / mx;
  const double deta = (c->eta_max - c->eta_min) / my;

  NA_CK(cudaSetDevice(device));
  rc = scratch_address(device, &base);
  if (rc != PCL_OK) goto done;

  // mesh tables and a fresh control block for this attempt (the array keeps the last call's)
  build_tables(c, dxi, deta, rowm, colm);
  std::memset(&h, 0, sizeof(h));
  h.time = 0.0;
  h.time_final = 1.0;
  h.dt = dt;
  h.dt_previous = dt;
  h.CFL = 0.0;
  h.CFL_target = c->cfl_limit;
  h.shrink = c->dt_min_shrink_ratio;
  h.growth = c->dt_max_growth_ratio;
  h.emergency = 0.25;
  h.time_precision = 0.01;
  h.adaptive = 1;
  h.n_snapshots = 1;
  h.snapshot_index = 1;
  h.cur = 0;
  h.log = nullptr;

  g.state = base;
  g.bufstride = 3 * plane;
  g.neq = 3;
  g.rowm = base + kTableOffset;
  g.colm = base + kTableOffset + (long long)(my + 4) * pcl::kRowMetrics;
  g.ctl = reinterpret_cast<pcl::Ctl*>(base + kCtlOffset);
  g.plane = plane;
  g.mx = mx;
  g.my = my;
  g.pitch = pitch;
  g.bc[0] = c->bc_xi_lower; g.bc[1] = c->bc_xi_upper; g.bc[2] = c->bc_eta_lower; g.bc[3] = c->bc_eta_upper;
  g.second_order = c->higher_order_flux_correction ? 1 : 0;
  g.limiter = c->use_limiter ? c->limiter_method : 0;
  g.dxi = dxi;
  g.deta = deta;
  g.area_scale = dxi * deta;
  g.grav = c->grav;
  g.metric = unit_metric(rowm, colm, mx, my, g.area_scale) ? pcl::kMetricUnit : pcl::kMetricTable;

  NA_CK(cudaMemcpyAsync(const_cast<double*>(g.rowm), rowm.data(), sizeof(double) * rowm.size(),
                        cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(const_cast<double*>(g.colm), colm.data(), sizeof(double) * colm.size(),
                        cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(g.ctl, &h, kCtlHot, cudaMemcpyHostToDevice, st));
  // the caller's state (3 planes of m_eta+4 rows, leading dimension ld) into buffer 0, and into
  // buffer 2 so the corner ghosts the sweeps never write carry the caller's values
  for (int b : {0, 2})
    NA_CK(cudaMemcpy2DAsync(base + b * g.bufstride, sizeof(double) * pitch, d_in, sizeof(double) * ld,
                            sizeof(double) * (mx + 4), 3 * (size_t)(my + 4), cudaMemcpyDeviceToDevice, st));
  pcl::launch_timectl(g, pcl::kOpInit, 0, 0.0, st);
  pcl::launch_sweeps_fp64(g, st);
  pcl::launch_timectl(g, pcl::kOpFinalizeSolve, 0, 0.0, st);
  NA_CK(cudaGetLastError());
  NA_CK(cudaMemcpyAsync(&h, g.ctl, kCtlHot, cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  *ierr = h.ierr;
  if (cfl) *cfl = h.CFL;
  rc = status_code(h.status);
  if (rc == PCL_OK && h.ierr == 1) {
    NA_CK(cudaMemcpy2DAsync(d_out, sizeof(double) * ld, base + (long long)h.cur * g.bufstride, sizeof(double) * pitch,
                            sizeof(double) * (mx + 4), 3 * (size_t)(my + 4), cudaMemcpyDeviceToDevice, st));
    NA_CK(cudaStreamSynchronize(st));
  }
done:
  if (prev >= 0) cudaSetDevice(prev);
  return rc;
}
