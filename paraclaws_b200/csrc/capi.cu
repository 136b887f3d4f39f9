// capi.cu -- the C ABI (include/paraclaws_b200.h): contexts, the control.in reader, and the
// per-routine and whole-loop entry points.  Host arithmetic here (mesh tables, snapshot times)
// is built without contraction (-ffp-contract=off) to round as the reference does.
#include <cuda_runtime.h>

#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <string>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/paraclaws_b200.h"
#include "pcl_equations.h"
#include "pcl_launch.h"
#include "pcl_types.h"
#include "pcl_mixed.h"

using namespace pcl;

struct pcl_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  pcl_solver_control cfg{};
  GridDev g{};
  Ctl* ctl_d = nullptr;
  Ctl* ctl_h = nullptr;          // pinned mirror for reads
  double* bufs_d = nullptr;      // 3 state buffers
  double* tables_d = nullptr;    // row + column metric tables
  double* metrics_d = nullptr;   // mapped grids: capacity and face length ratios per cell
  double* staging_d = nullptr;   // AoS staging for upload/download
  StepLogEntry* log_d = nullptr;
  long long log_cap = 0;
  size_t device_bytes = 0;
  cudaGraphExec_t graph = nullptr;
  int graph_chunk = 0;
  void* mixed = nullptr;         // mixed-precision workspace (pcl_mixed.h)
  long long launches = 0;        // kernels launched by this context
  long long graph_launches = 0;  // kernels in one launch of the captured graph
  long long h2d_bytes = 0, d2h_bytes = 0;  // bytes copied across the host boundary
  // snapshot writer: pinned copy of the state, the copy's event, and the formatting thread
  pcl_user_bc_fn user_bc = nullptr;  // hook for sides coded 1
  void* user_bc_data = nullptr;
  pcl_source_fn source = nullptr;     // source-term hook
  void* source_data = nullptr;
  int user_bc_rc = 0;                 // first failure of a hook since the last check
  double* snap_h = nullptr;
  cudaEvent_t snap_ev = nullptr;
  std::thread snap_thread;
  int snap_status = 0;
};

#define CK(call)                                       \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) {                           \
      std::fprintf(stderr, "paraclaws_b200: %s: %s\n", #call, cudaGetErrorString(e_)); \
      return PCL_ERR_CUDA;                             \
    }                                                  \
  } while (0)

static int status_to_code(int st) {
  if (st & kStatusNaN) return PCL_ERR_NAN;
  if (st & kStatusNegDepth) return PCL_ERR_NEG_DEPTH;
  if (st & kStatusTimeout) return PCL_ERR_TIMEOUT;
  if (st & kStatusFatalDt) return PCL_ERR_FATAL_DT;
  return PCL_OK;
}

extern "C" {

int pcl_version(void) { return 100; }

const char* pcl_status_string(int s) {
  switch (s) {
    case PCL_OK: return "ok";
    case PCL_ERR_NAN: return "NaN in a flux Jacobian";
    case PCL_ERR_NEG_DEPTH: return "negative water depth (complex eigenvalues)";
    case PCL_ERR_TIMEOUT: return "device wait timed out";
    case PCL_ERR_OOM: return "out of memory";
    case PCL_ERR_BADARG: return "invalid argument";
    case PCL_ERR_CUDA: return "CUDA error";
    case PCL_ERR_FATAL_DT: return "time step control cannot continue (constant dt violated)";
    case PCL_ERR_IO: return "cannot read a control file or write a snapshot file";
    case PCL_ERR_FULL: return "batch is full or over its memory budget";
    case PCL_ERR_USER: return "a device hook (user boundary condition or source term) failed";
    default: return "unknown status";
  }
}

void pcl_default_control(pcl_solver_control* c) {
  std::memset(c, 0, sizeof(*c));
  c->num_equations = 3;
  c->num_dimensions = 2;
  c->num_ghost = 2;
  c->num_aux = 10;
  c->num_waves = 2;
  c->t_start = 0.0;
  c->t_final = 0.5;
  c->number_of_snapshots = 5;
  c->dt_initial = 1e-10;
  c->adaptive_timestepping = 1;
  c->cfl_limit = 0.1;
  c->dt_min = 1e-10;
  c->dt_max = 5e-5;
  c->dt_max_growth_ratio = 1.2;
  c->dt_min_shrink_ratio = 0.5;
  c->higher_order_flux_correction = 0;
  c->use_limiter = 1;
  c->limiter_method = 1;
  c->m_xi = c->m_eta = 21;
  c->xi_min = -1.0; c->xi_max = 1.0; c->eta_min = -1.0; c->eta_max = 1.0;
  c->bc_xi_lower = c->bc_xi_upper = c->bc_eta_lower = c->bc_eta_upper = 2;
  c->precision_mode = PCL_PREC_FP64;
  c->grav = (double)9.81f;  // examples/2D_dam_break/cartesian/SMOD_setup.f90:21
  c->initial_condition = 1;
  c->dam_radius = 0.5; c->dam_h_in = 2.0; c->dam_h_out = 1.0; c->dam_x0 = 0.0; c->dam_y0 = 0.0;
  c->max_accepted_steps = 0;
}

// ---- list-directed reads (utility/MOD_IO.f90:61-94) ----
static bool first_token(const std::string& rec, std::string& tok) {
  size_t a = rec.find_first_not_of(" \t\r");
  if (a == std::string::npos) return false;
  size_t b = rec.find_first_of(" \t\r,/", a);
  tok = rec.substr(a, b == std::string::npos ? std::string::npos : b - a);
  return !tok.empty();
}
static bool parse_int(const std::string& t, int& v) {
  char* e = nullptr;
  long x = std::strtol(t.c_str(), &e, 10);
  if (e == t.c_str() || *e) return false;
  v = (int)x;
  return true;
}
static bool parse_ll(const std::string& t, long long& v) {
  char* e = nullptr;
  long long x = std::strtoll(t.c_str(), &e, 10);
  if (e == t.c_str() || *e) return false;
  v = x;
  return true;
}
static bool parse_real(std::string t, double& v) {
  for (auto& ch : t)
    if (ch == 'd' || ch == 'D') ch = 'e';
  char* e = nullptr;
  double x = std::strtod(t.c_str(), &e);
  if (e == t.c_str() || *e) return false;
  v = x;
  return true;
}
static bool parse_logical(std::string t, int& v) {
  if (!t.empty() && t[0] == '.') t = t.substr(1);
  if (t.empty()) return false;
  char ch = (char)std::toupper((unsigned char)t[0]);
  if (ch == 'T') { v = 1; return true; }
  if (ch == 'F') { v = 0; return true; }
  return false;
}
static bool read_records(const char* path, std::vector<std::string>& toks) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line, tok;
  while (std::getline(f, line))
    if (first_token(line, tok)) toks.push_back(tok);
  return true;
}

int pcl_read_solver_control(const char* control_in, const char* custom_in, pcl_solver_control* out) {
  if (!control_in || !out) return PCL_ERR_BADARG;
  pcl_default_control(out);
  std::vector<std::string> t;
  if (!read_records(control_in, t)) return PCL_ERR_IO;
  if (t.size() < 28) return PCL_ERR_IO;
  bool ok = true;
  pcl_solver_control& c = *out;
  ok &= parse_int(t[0], c.num_equations);
  ok &= parse_int(t[1], c.num_dimensions);
  ok &= parse_int(t[2], c.num_ghost);
  ok &= parse_int(t[3], c.num_aux);
  ok &= parse_int(t[4], c.num_waves);
  ok &= parse_real(t[5], c.t_start);
  ok &= parse_real(t[6], c.t_final);
  ok &= parse_int(t[7], c.number_of_snapshots);
  ok &= parse_real(t[8], c.dt_initial);
  ok &= parse_logical(t[9], c.adaptive_timestepping);
  ok &= parse_real(t[10], c.cfl_limit);
  ok &= parse_real(t[11], c.dt_min);
  ok &= parse_real(t[12], c.dt_max);
  ok &= parse_real(t[13], c.dt_max_growth_ratio);
  ok &= parse_real(t[14], c.dt_min_shrink_ratio);
  ok &= parse_logical(t[15], c.higher_order_flux_correction);
  ok &= parse_logical(t[16], c.use_limiter);
  ok &= parse_int(t[17], c.limiter_method);
  ok &= parse_int(t[18], c.m_xi);
  ok &= parse_int(t[19], c.m_eta);
  ok &= parse_real(t[20], c.xi_min);
  ok &= parse_real(t[21], c.xi_max);
  ok &= parse_real(t[22], c.eta_min);
  ok &= parse_real(t[23], c.eta_max);
  ok &= parse_int(t[24], c.bc_xi_lower);
  ok &= parse_int(t[25], c.bc_xi_upper);
  ok &= parse_int(t[26], c.bc_eta_lower);
  ok &= parse_int(t[27], c.bc_eta_upper);
  if (!ok) return PCL_ERR_IO;
  if (custom_in) {
    std::vector<std::string> u;
    if (read_records(custom_in, u) && u.size() >= 9) {
      ok &= parse_ll(u[0], c.max_accepted_steps);
      ok &= parse_int(u[1], c.precision_mode);
      ok &= parse_real(u[2], c.grav);
      ok &= parse_int(u[3], c.initial_condition);
      ok &= parse_real(u[4], c.dam_radius);
      ok &= parse_real(u[5], c.dam_h_in);
      ok &= parse_real(u[6], c.dam_h_out);
      ok &= parse_real(u[7], c.dam_x0);
      ok &= parse_real(u[8], c.dam_y0);
      if (!ok) return PCL_ERR_IO;
    }
  }
  return PCL_OK;
}

// num_equations: the state's components, 1 .. PCL_EQ_MAX_EQUATIONS (3 for the shallow-water
// modules, the mixed-precision and batched forms).  num_waves: HLL makes two waves
// (solver/SMOD_approximate_Riemann_solvers.f90:68-100 writes lambda(1:2) and waves(:,1:2)); the
// reference's work arrays hold num_waves of them, zeroed after every sweep
// (solver/MOD_work_arrays.f90:79-109), so waves 3.. stay zero and add nothing to the CFL maximum,
// the split fluxes or the correction: any num_waves >= 2 runs the two-wave step.  num_waves = 1
// would have HLL write past its arrays and is refused.
int validate_control(const pcl_solver_control* c) {
  if (c->num_equations < 1 || c->num_equations > PCL_EQ_MAX_EQUATIONS || c->num_waves < 2 || c->num_ghost != 2)
    return PCL_ERR_BADARG;
  if (c->num_equations != 3 && c->precision_mode != PCL_PREC_FP64) return PCL_ERR_BADARG;
  if (c->m_xi < 2 || c->m_eta < 2) return PCL_ERR_BADARG;
  if (c->m_xi > (1 << 28) || c->m_eta > 16 * 65535) return PCL_ERR_BADARG;  // launch-grid limits
  const int bcs[4] = {c->bc_xi_lower, c->bc_xi_upper, c->bc_eta_lower, c->bc_eta_upper};
  for (int k = 0; k < 4; ++k)
    if (bcs[k] < 1 || bcs[k] > 3) return PCL_ERR_BADARG;
  if (c->higher_order_flux_correction && c->use_limiter && (c->limiter_method < 1 || c->limiter_method > 4))
    return PCL_ERR_BADARG;
  if (c->dt_min > c->dt_max) return PCL_ERR_BADARG;
  if (c->precision_mode != PCL_PREC_FP64 && c->precision_mode != PCL_PREC_MIXED) return PCL_ERR_BADARG;
  if (c->number_of_snapshots > kMaxSnapshots) return PCL_ERR_BADARG;
  if (!(c->xi_max > c->xi_min) || !(c->eta_max > c->eta_min)) return PCL_ERR_BADARG;
  return PCL_OK;
}

// mesh tables in the reference's operation order (domain/SMOD_mesh_manipulation.f90)
void build_tables(const pcl_solver_control* c, double dxi, double deta, std::vector<double>& rowm,
                         std::vector<double>& colm) {
  const int ni = c->m_xi + 4, nj = c->m_eta + 4;
  rowm.assign((size_t)nj * kRowMetrics, 0.0);
  colm.assign((size_t)ni * kColMetrics, 0.0);
  for (int j = -1; j <= c->m_eta + 2; ++j) {
    const double e1 = c->eta_min + (double)(j - 1) * deta;  // eta_corner(1) :43
    const double e3 = e1 + deta;                            // eta_corner(3) :45
    double* r = &rowm[(size_t)(j + 1) * kRowMetrics];
    r[0] = 0.5 * (e1 + e1);
    r[1] = 0.5 * (e3 + e3);
    r[2] = std::fabs(e3 - e1) / deta;  // length_ratio_xi :147-153, NORM2([0, dy]) = |dy|
    r[3] = c->eta_min + (double)(j - 1) * deta + deta / 2;  // eta centre :51
  }
  for (int i = -1; i <= c->m_xi + 2; ++i) {
    const double c1 = c->xi_min + (double)(i - 1) * dxi;  // xi_corner(1) :36
    const double c2 = c1 + dxi;                            // xi_corner(2) :37
    double* r = &colm[(size_t)(i + 1) * kColMetrics];
    r[0] = c1 - c2;
    r[1] = c2 - c1;
    r[2] = std::fabs(c2 - c1) / dxi;  // length_ratio_eta :156-162
    r[3] = c->xi_min + (double)(i - 1) * dxi + dxi / 2;  // xi centre :50
  }
}

// time_control%initialize (MOD_time_control.f90:70-151)
void init_ctl(const pcl_solver_control* c, Ctl& t) {
  std::memset(&t, 0, sizeof(t));
  t.time_initial = c->t_start;
  t.time_final = c->t_final;
  t.time = c->t_start;
  t.dt = c->dt_initial;
  t.dt_previous = c->dt_initial;
  t.dt_max = c->dt_max;
  t.dt_min = c->dt_min;
  t.adaptive = c->adaptive_timestepping ? 1 : 0;
  t.n_snapshots = c->number_of_snapshots < 1 ? 1 : c->number_of_snapshots;
  const double si = (t.time_final - t.time_initial) / t.n_snapshots;
  for (int i = 1; i <= t.n_snapshots; ++i) t.snap_times[i - 1] = t.time_initial + i * si;
  t.snap_times[t.n_snapshots - 1] = t.time_final;
  t.snapshot_index = 1;
  t.CFL = 0.0;
  t.CFL_previous_timestep = 0.0;
  t.CFL_target = c->cfl_limit;
  t.time_precision = 0.01;
  t.growth = c->dt_max_growth_ratio;
  t.shrink = c->dt_min_shrink_ratio;
  t.emergency = 0.25;
  t.cur = 0;
  t.max_accepted = c->max_accepted_steps;
}

static void free_ctx(pcl_ctx* x) {
  if (!x) return;
  if (x->snap_thread.joinable()) x->snap_thread.join();
  if (x->snap_ev) cudaEventDestroy(x->snap_ev);
  if (x->snap_h) cudaFreeHost(x->snap_h);
  if (x->graph) cudaGraphExecDestroy(x->graph);
  if (x->mixed) mixed_free(x->mixed);
  cudaFree(x->bufs_d);
  cudaFree(x->tables_d);
  cudaFree(x->metrics_d);
  cudaFree(x->staging_d);
  cudaFree(x->ctl_d);
  cudaFree(x->log_d);
  if (x->ctl_h) cudaFreeHost(x->ctl_h);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

int pcl_create(const pcl_solver_control* c, int device, pcl_ctx** out) {
  if (!c || !out) return PCL_ERR_BADARG;
  *out = nullptr;
  int v = validate_control(c);
  if (v != PCL_OK) return v;
  CK(cudaSetDevice(device));
  pcl_ctx* x = new pcl_ctx();
  x->device = device;
  x->cfg = *c;
  auto fail = [&](int code) {
    free_ctx(x);
    return code;
  };
  if (cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PCL_ERR_CUDA);
  const int ni = c->m_xi + 4, nj = c->m_eta + 4;
  const int pitch = (ni + 31) / 32 * 32;
  const long long plane = (long long)pitch * nj;
  const int neq = c->num_equations;
  const size_t buf_bytes = sizeof(double) * 3 * (size_t)neq * (size_t)plane;
  const double dxi = (c->xi_max - c->xi_min) / c->m_xi;     // :28
  const double deta = (c->eta_max - c->eta_min) / c->m_eta;  // :29
  std::vector<double> rowm, colm;
  build_tables(c, dxi, deta, rowm, colm);
  const size_t tab_bytes = sizeof(double) * (rowm.size() + colm.size());
  const size_t stg_bytes = sizeof(double) * (size_t)neq * (size_t)ni * nj;
  x->log_cap = 1 << 16;
  if (cudaMalloc(&x->bufs_d, buf_bytes) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&x->tables_d, tab_bytes) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&x->staging_d, stg_bytes) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&x->ctl_d, sizeof(Ctl)) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&x->log_d, sizeof(StepLogEntry) * x->log_cap) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMallocHost(&x->ctl_h, sizeof(Ctl)) != cudaSuccess) return fail(PCL_ERR_OOM);
  x->device_bytes = buf_bytes + tab_bytes + stg_bytes + sizeof(Ctl) + sizeof(StepLogEntry) * x->log_cap;
  if (cudaMemsetAsync(x->bufs_d, 0, buf_bytes, x->stream) != cudaSuccess) return fail(PCL_ERR_CUDA);
  if (cudaMemcpyAsync(x->tables_d, rowm.data(), sizeof(double) * rowm.size(), cudaMemcpyHostToDevice, x->stream) != cudaSuccess)
    return fail(PCL_ERR_CUDA);
  if (cudaMemcpyAsync(x->tables_d + rowm.size(), colm.data(), sizeof(double) * colm.size(), cudaMemcpyHostToDevice,
                      x->stream) != cudaSuccess)
    return fail(PCL_ERR_CUDA);
  init_ctl(c, *x->ctl_h);
  x->ctl_h->log = x->log_d;
  x->ctl_h->log_cap = x->log_cap;
  if (cudaMemcpyAsync(x->ctl_d, x->ctl_h, sizeof(Ctl), cudaMemcpyHostToDevice, x->stream) != cudaSuccess)
    return fail(PCL_ERR_CUDA);
  GridDev& g = x->g;
  g.state = x->bufs_d;
  g.bufstride = (long long)neq * plane;
  g.neq = neq;
  g.eq = neq == 3 ? PCL_EQ_SHALLOW_WATER : -1;  // other sizes need a module (pcl_set_equation)
  g.rowm = x->tables_d;
  g.colm = x->tables_d + rowm.size();
  g.ctl = x->ctl_d;
  g.plane = plane;
  g.mx = c->m_xi;
  g.my = c->m_eta;
  g.pitch = pitch;
  g.bc[0] = c->bc_xi_lower; g.bc[1] = c->bc_xi_upper; g.bc[2] = c->bc_eta_lower; g.bc[3] = c->bc_eta_upper;
  g.second_order = c->higher_order_flux_correction ? 1 : 0;
  g.limiter = c->use_limiter ? c->limiter_method : 0;
  g.dxi = dxi;
  g.deta = deta;
  g.area_scale = dxi * deta;  // d_xi*d_eta (SMOD_mesh_manipulation.f90:173)
  g.grav = c->grav;
  launch_metric_check(g, x->stream);
  if (cudaMemcpyAsync(&x->ctl_h->nonunit_metric, &g.ctl->nonunit_metric, sizeof(int), cudaMemcpyDeviceToHost,
                      x->stream) != cudaSuccess || cudaStreamSynchronize(x->stream) != cudaSuccess)
    return fail(PCL_ERR_CUDA);
  g.metric = x->ctl_h->nonunit_metric ? kMetricTable : kMetricUnit;
  if (c->precision_mode == PCL_PREC_MIXED) {
    int r = mixed_create(g, x->stream, &x->mixed);
    if (r != PCL_OK) return fail(r);
  }
  launch_timectl(g, kOpInit, 0, 0.0, x->stream);
  if (cudaStreamSynchronize(x->stream) != cudaSuccess) return fail(PCL_ERR_CUDA);
  if (cudaGetLastError() != cudaSuccess) return fail(PCL_ERR_CUDA);
  *out = x;
  return PCL_OK;
}

int pcl_destroy(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  cudaSetDevice(x->device);
  cudaStreamSynchronize(x->stream);
  free_ctx(x);
  return PCL_OK;
}

long long pcl_state_doubles(const pcl_ctx* x) {
  return x ? (long long)x->cfg.num_equations * (x->cfg.m_xi + 4) * (x->cfg.m_eta + 4) : 0;
}
long long pcl_device_bytes(const pcl_ctx* x) { return x ? (long long)x->device_bytes : 0; }
void* pcl_get_stream(pcl_ctx* x) { return x ? (void*)x->stream : nullptr; }

// the control block without its snapshot table (which only the host writes)
static const size_t kCtlHotBytes = offsetof(Ctl, snap_times);

static int read_ctl(pcl_ctx* x) {
  x->d2h_bytes += (long long)kCtlHotBytes;
  CK(cudaMemcpyAsync(x->ctl_h, x->ctl_d, kCtlHotBytes, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return PCL_OK;
}

static int check_launch(pcl_ctx* x) {
  CK(cudaGetLastError());
  return PCL_OK;
}

int pcl_synchronize(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  CK(cudaStreamSynchronize(x->stream));
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  return status_to_code(x->ctl_h->status);
}

int pcl_upload_state(pcl_ctx* x, const double* vars) {
  if (!x || !vars) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  x->h2d_bytes += (long long)sizeof(double) * pcl_state_doubles(x);
  CK(cudaMemcpyAsync(x->staging_d, vars, sizeof(double) * pcl_state_doubles(x), cudaMemcpyHostToDevice, x->stream));
  launch_upload(x->g, x->staging_d, x->stream);
  int r = check_launch(x);
  if (r != PCL_OK) return r;
  CK(cudaStreamSynchronize(x->stream));
  return PCL_OK;
}

int pcl_initial_condition(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  if (x->cfg.initial_condition != 1 || x->g.neq != 3) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  const pcl_solver_control& c = x->cfg;
  launch_dam_ic(x->g, c.dam_radius, c.dam_h_in, c.dam_h_out, c.dam_x0, c.dam_y0, x->stream);
  x->launches += 1;
  int r = check_launch(x);
  if (r != PCL_OK) return r;
  CK(cudaStreamSynchronize(x->stream));
  return PCL_OK;
}

int pcl_download_state(pcl_ctx* x, double* vars) {
  if (!x || !vars) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  launch_download(x->g, x->staging_d, x->stream);
  int r = check_launch(x);
  if (r != PCL_OK) return r;
  x->d2h_bytes += (long long)sizeof(double) * pcl_state_doubles(x);
  CK(cudaMemcpyAsync(vars, x->staging_d, sizeof(double) * pcl_state_doubles(x), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  return PCL_OK;
}

static void fill_view(const pcl_ctx* x, pcl_device_view& v) {
  v.state = x->g.state;
  v.buffer_stride = x->g.bufstride;
  v.plane_stride = x->g.plane;
  v.pitch = x->g.pitch;
  v.m_xi = x->g.mx;
  v.m_eta = x->g.my;
  v.centre_stride = kColMetrics;
  v.xi_centre = x->g.colm + 3;
  v.eta_centre = x->g.rowm + 3;
  v.current_buffer = &x->ctl_d->cur;
  v.attempt_accepted = &x->ctl_d->ierr;
  v.step_dt = &x->ctl_d->dt_step;
  v.num_equations = x->g.neq;
}

// The ghost fill: the built-in kernel for every side, then the user hook for sides coded 1.
static void enqueue_ghost(pcl_ctx* x, int force) {
  launch_ghost(x->g, force, x->stream);
  if (!x->user_bc) return;
  int sides = 0;
  for (int s = 0; s < 4; ++s)
    if (x->g.bc[s] == 1) sides |= 1 << s;
  if (!sides) return;
  pcl_device_view v;
  fill_view(x, v);
  const int rc = x->user_bc(&v, sides, force, (void*)x->stream, x->user_bc_data);
  if (rc != 0 && x->user_bc_rc == 0) x->user_bc_rc = PCL_ERR_USER;
}

// integrate_source_term: nothing for phi = 0, else the source hook
static void enqueue_source(pcl_ctx* x, int force) {
  if (!x->source) return;
  pcl_device_view v;
  fill_view(x, v);
  const int rc = x->source(&v, force, (void*)x->stream, x->source_data);
  if (rc != 0 && x->user_bc_rc == 0) x->user_bc_rc = PCL_ERR_USER;
}

int pcl_set_source_hook(pcl_ctx* x, pcl_source_fn fn, void* user) {
  if (!x) return PCL_ERR_BADARG;
  x->source = fn;
  x->source_data = user;
  if (x->graph) {  // the captured graphs hold the previous step
    cudaGraphExecDestroy(x->graph);
    x->graph = nullptr;
    x->graph_chunk = 0;
  }
  return PCL_OK;
}

static int take_user_bc_rc(pcl_ctx* x) {
  const int r = x->user_bc_rc;
  x->user_bc_rc = 0;
  return r;
}

int pcl_update_rank_boundaries(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  enqueue_ghost(x, 1);
  x->launches += 1;
  const int r = take_user_bc_rc(x);
  if (r != PCL_OK) return r;
  return check_launch(x);
}

int pcl_set_user_bc(pcl_ctx* x, pcl_user_bc_fn fn, void* user) {
  if (!x) return PCL_ERR_BADARG;
  x->user_bc = fn;
  x->user_bc_data = user;
  x->g.user_bc = fn ? 1 : 0;
  if (x->graph) {  // the captured graphs hold the previous fill
    cudaGraphExecDestroy(x->graph);
    x->graph = nullptr;
    x->graph_chunk = 0;
  }
  return PCL_OK;
}

static int sweep_kernels(const pcl_ctx* x) { return x->cfg.precision_mode == PCL_PREC_MIXED ? 1 : 2; }

static void launch_sweeps(pcl_ctx* x) {
  if (x->cfg.precision_mode == PCL_PREC_MIXED)
    launch_sweeps_mixed(x->g, x->mixed, x->stream);
  else
    launch_sweeps_fp64(x->g, x->stream);
  x->launches += sweep_kernels(x);
}

int pcl_solve_dimensional_split(pcl_ctx* x, int* ierr) {
  if (!x || !ierr || x->g.eq < 0) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  launch_sweeps(x);
  launch_timectl(x->g, kOpFinalizeSolve, 0, 0.0, x->stream);
  x->launches += 1;
  int r = check_launch(x);
  if (r != PCL_OK) return r;
  r = read_ctl(x);
  if (r != PCL_OK) return r;
  *ierr = x->ctl_h->ierr;
  return status_to_code(x->ctl_h->status);
}

int pcl_restore_solution(pcl_ctx* x) { return x ? PCL_OK : PCL_ERR_BADARG; }
int pcl_integrate_source_term(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  if (!x->source) return PCL_OK;  // phi = 0: q + 0*dt leaves every finite q unchanged
  CK(cudaSetDevice(x->device));
  enqueue_source(x, 1);
  const int r = take_user_bc_rc(x);
  if (r != PCL_OK) return r;
  return check_launch(x);
}

static int timeop(pcl_ctx* x, int op, int arg, double value) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  launch_timectl(x->g, op, arg, value, x->stream);
  x->launches += 1;
  return check_launch(x);
}

int pcl_update_time(pcl_ctx* x, int step_valid) {
  int r = timeop(x, kOpUpdateTime, step_valid ? 1 : 0, 0.0);
  if (r != PCL_OK) return r;
  r = read_ctl(x);
  if (r != PCL_OK) return r;
  return status_to_code(x->ctl_h->status);
}
int pcl_reset_cfl(pcl_ctx* x) { return timeop(x, kOpResetCFL, 0, 0.0); }
int pcl_advance_snapshot_index(pcl_ctx* x) { return timeop(x, kOpAdvanceSnapshot, 0, 0.0); }
int pcl_set_dt(pcl_ctx* x, double dt) { return timeop(x, kOpSetDt, 0, dt); }

#define GETTER(name, type, expr)                 \
  int name(pcl_ctx* x, type* v) {                \
    if (!x || !v) return PCL_ERR_BADARG;         \
    CK(cudaSetDevice(x->device));                \
    int r = read_ctl(x);                         \
    if (r != PCL_OK) return r;                   \
    *v = (expr);                                 \
    return PCL_OK;                               \
  }
GETTER(pcl_get_time, double, x->ctl_h->time)
GETTER(pcl_get_dt, double, x->ctl_h->dt)
GETTER(pcl_get_previous_dt, double, x->ctl_h->dt_previous)
GETTER(pcl_get_cfl, double, x->ctl_h->CFL)
GETTER(pcl_get_snapshot_index, int, x->ctl_h->snapshot_index)
#undef GETTER

int pcl_get_snapshot_time(pcl_ctx* x, int idx, double* t) {
  if (!x || !t) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  if (idx < 1 || idx > x->ctl_h->n_snapshots) return PCL_ERR_BADARG;
  *t = x->ctl_h->snap_times[idx - 1];
  return PCL_OK;
}

static void fill_stats(const Ctl& c, long long launches, pcl_run_stats* s) {
  s->launches = launches;
  s->attempts = c.attempts;
  s->accepted = c.accepted;
  s->rejected = c.attempts - c.accepted;
  s->time = c.time;
  s->dt = c.dt;
  s->dt_previous = c.dt_previous;
  s->cfl = c.CFL;
  s->snapshot_index = c.snapshot_index;
  s->done = c.done;
  s->status = status_to_code(c.status);
  s->last_ierr = c.ierr;
}

int pcl_get_stats(pcl_ctx* x, pcl_run_stats* s) {
  if (!x || !s) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  fill_stats(*x->ctl_h, x->launches, s);
  return PCL_OK;
}

static void enqueue_attempt(pcl_ctx* x) {
  if (x->cfg.precision_mode == PCL_PREC_MIXED && !x->source && !x->user_bc && !mixed_injection_on(x->mixed)) {
    launch_step_mixed(x->g, x->mixed, x->stream);  // sweeps, time control and ghost fill in one launch
    x->launches += 1;
    return;
  }
  launch_sweeps(x);
  launch_timectl(x->g, kOpFullStep, 0, 0.0, x->stream);
  enqueue_source(x, 0);
  enqueue_ghost(x, 0);
  x->launches += 2;
}

static int build_graph(pcl_ctx* x, int chunk) {
  if (x->graph && x->graph_chunk == chunk) return PCL_OK;
  if (x->graph) {
    cudaGraphExecDestroy(x->graph);
    x->graph = nullptr;
  }
  cudaGraph_t gr;
  const long long before = x->launches;
  CK(cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal));
  for (int k = 0; k < chunk; ++k) enqueue_attempt(x);
  CK(cudaStreamEndCapture(x->stream, &gr));
  x->graph_launches = x->launches - before;  // kernels per graph launch
  x->launches = before;
  const int urc = take_user_bc_rc(x);
  if (urc != PCL_OK) {
    cudaGraphDestroy(gr);
    return urc;
  }
  cudaError_t e = cudaGraphInstantiate(&x->graph, gr, 0);
  cudaGraphDestroy(gr);
  if (e != cudaSuccess) return PCL_ERR_CUDA;
  x->graph_chunk = chunk;
  return PCL_OK;
}

static int advance_loop(pcl_ctx* x, long long max_attempts, pcl_run_stats* stats);

int pcl_advance(pcl_ctx* x, long long max_attempts, pcl_run_stats* stats) { return advance_loop(x, max_attempts, stats); }

int pcl_advance_to_snapshot(pcl_ctx* x, pcl_run_stats* stats) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  int r = timeop(x, kOpSetPause, 1, 0.0);
  if (r != PCL_OK) return r;
  const int rc = advance_loop(x, 0, nullptr);
  r = timeop(x, kOpSetPause, 0, 0.0);  // the context steps normally again
  if (r != PCL_OK) return r;
  r = read_ctl(x);
  if (r != PCL_OK) return r;
  if (stats) fill_stats(*x->ctl_h, x->launches, stats);
  return rc;
}

static int advance_loop(pcl_ctx* x, long long max_attempts, pcl_run_stats* stats) {
  if (!x || x->g.eq < 0) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  const int chunk = 32;
  int r = build_graph(x, chunk);
  if (r != PCL_OK) return r;
  r = read_ctl(x);
  if (r != PCL_OK) return r;
  const long long start = x->ctl_h->attempts;
  timeop(x, kOpInit, 0, 0.0);  // refresh done / dt ratios after any host-side change
  r = read_ctl(x);
  if (r != PCL_OK) return r;
  while (!x->ctl_h->done) {
    const long long doneatt = x->ctl_h->attempts - start;
    if (max_attempts > 0 && doneatt >= max_attempts) break;
    if (max_attempts > 0 && max_attempts - doneatt < chunk) {
      for (long long k = doneatt; k < max_attempts; ++k) enqueue_attempt(x);
      r = take_user_bc_rc(x);
      if (r != PCL_OK) return r;
    } else {
      CK(cudaGraphLaunch(x->graph, x->stream));
      x->launches += x->graph_launches;
    }
    r = check_launch(x);
    if (r != PCL_OK) return r;
    r = read_ctl(x);
    if (r != PCL_OK) return r;
  }
  if (stats) fill_stats(*x->ctl_h, x->launches, stats);
  return status_to_code(x->ctl_h->status);
}

int pcl_reset_time_control(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  CK(cudaStreamSynchronize(x->stream));
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  const int cur = x->ctl_h->cur;
  init_ctl(&x->cfg, *x->ctl_h);
  x->ctl_h->cur = cur;
  x->ctl_h->log = x->log_d;
  x->ctl_h->log_cap = x->log_cap;
  CK(cudaMemcpyAsync(x->ctl_d, x->ctl_h, sizeof(Ctl), cudaMemcpyHostToDevice, x->stream));
  launch_timectl(x->g, kOpInit, 0, 0.0, x->stream);
  x->launches += 1;
  CK(cudaStreamSynchronize(x->stream));
  return check_launch(x);
}

int pcl_profile_kernels(pcl_ctx* x, int reps, double* avg_ms, int* nkinds) {
  if (!x || !avg_ms || reps < 1 || x->g.eq < 0) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  const int nk = sweep_kernels(x) + 2;
  cudaEvent_t ev[6];
  for (int k = 0; k < 6; ++k) CK(cudaEventCreate(&ev[k]));
  double acc[5] = {0, 0, 0, 0, 0};
  for (int r = 0; r < reps; ++r) {
    int e = 0;
    CK(cudaEventRecord(ev[e++], x->stream));
    if (x->cfg.precision_mode == PCL_PREC_MIXED) {
      launch_sweeps_mixed(x->g, x->mixed, x->stream);
      CK(cudaEventRecord(ev[e++], x->stream));
    } else {
      launch_xsweep_fp64(x->g, x->stream);
      CK(cudaEventRecord(ev[e++], x->stream));
      launch_ysweep_fp64(x->g, x->stream);
      CK(cudaEventRecord(ev[e++], x->stream));
    }
    launch_timectl(x->g, kOpFullStep, 0, 0.0, x->stream);
    CK(cudaEventRecord(ev[e++], x->stream));
    launch_ghost(x->g, 0, x->stream);
    CK(cudaEventRecord(ev[e++], x->stream));
    x->launches += nk;
    CK(cudaEventSynchronize(ev[e - 1]));
    for (int k = 0; k + 1 < e; ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
      acc[k] += ms;
    }
  }
  for (int k = 0; k < 6; ++k) cudaEventDestroy(ev[k]);
  for (int k = 0; k < nk; ++k) avg_ms[k] = acc[k] / reps;
  if (nkinds) *nkinds = nk;
  return check_launch(x);
}

int pcl_get_step_log(pcl_ctx* x, pcl_step_record* out, long long cap, long long* n) {
  if (!x) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  const long long len = x->ctl_h->log_len;
  if (n) *n = len;
  const long long m = len < cap ? len : cap;
  if (out && m > 0) {
    std::vector<StepLogEntry> tmp((size_t)m);
    CK(cudaMemcpy(tmp.data(), x->log_d, sizeof(StepLogEntry) * m, cudaMemcpyDeviceToHost));
    for (long long k = 0; k < m; ++k) {
      out[k].dt = tmp[k].dt;
      out[k].cfl = tmp[k].cfl;
      out[k].time = tmp[k].time;
      out[k].dt_next = tmp[k].dt_next;
      out[k].ierr = tmp[k].ierr;
      out[k].snapshot_index = tmp[k].snapshot_index;
    }
  }
  return PCL_OK;
}

int pcl_conservation_sums(pcl_ctx* x, double* sums) {
  if (!x || !sums || x->g.neq != 3) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  // the AoS staging buffer (3 doubles per padded cell) holds the 3 partials of each row
  launch_row_sums(x->g, x->staging_d, x->stream);
  x->launches += 1;
  int r = check_launch(x);
  if (r != PCL_OK) return r;
  std::vector<double> part((size_t)3 * x->cfg.m_eta);
  x->d2h_bytes += (long long)(sizeof(double) * part.size());
  CK(cudaMemcpyAsync(part.data(), x->staging_d, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  double s[3] = {0.0, 0.0, 0.0};
  for (int j = 0; j < x->cfg.m_eta; ++j)
    for (int p = 0; p < 3; ++p) s[p] += part[(size_t)j * 3 + p];
  for (int p = 0; p < 3; ++p) sums[p] = s[p];
  return PCL_OK;
}

static void drop_graph(pcl_ctx* x) {
  if (x->graph) {  // the captured launches carry the old kernels
    cudaGraphExecDestroy(x->graph);
    x->graph = nullptr;
    x->graph_chunk = 0;
  }
}

int pcl_set_equation(pcl_ctx* x, int module, const double* params, int nparams) {
  if (!x || module < 0 || module >= PCL_EQ_COUNT || nparams < 0 || (nparams > 0 && !params)) return PCL_ERR_BADARG;
  // the module's num_equations is the context's (control.in): the state has that many planes
  if (pcl_eq_num_equations(module) != x->cfg.num_equations) return PCL_ERR_BADARG;
  if (module != PCL_EQ_SHALLOW_WATER && (x->cfg.precision_mode != PCL_PREC_FP64 || x->g.metric == kMetricMapped))
    return PCL_ERR_BADARG;
  double p[2] = {x->cfg.grav, 0.0};
  if (module == PCL_EQ_ACOUSTICS) {
    if (nparams != 2 || !(params[0] > 0.0) || !(params[1] > 0.0)) return PCL_ERR_BADARG;
    p[0] = params[0];
    p[1] = params[1];
  } else if (module == PCL_EQ_ADVECTION) {
    if (nparams != 2 || !std::isfinite(params[0]) || !std::isfinite(params[1])) return PCL_ERR_BADARG;
    p[0] = params[0];
    p[1] = params[1];
  } else if (module == PCL_EQ_BURGERS) {
    if (nparams != 0) return PCL_ERR_BADARG;
  } else if (nparams >= 1) {  // the shallow-water modules: g
    p[0] = params[0];
  }
  x->g.eq = module;
  x->g.eqp[0] = p[0];
  x->g.eqp[1] = p[1];
  if (module == PCL_EQ_SHALLOW_WATER) x->g.grav = p[0];
  drop_graph(x);
  return PCL_OK;
}

int pcl_set_mesh_metrics(pcl_ctx* x, const double* capacity, const double* lrx, const double* lry) {
  if (!x || !capacity || !lrx || !lry || x->cfg.precision_mode != PCL_PREC_FP64 || x->g.eq != PCL_EQ_SHALLOW_WATER)
    return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  GridDev& g = x->g;
  const size_t ni = (size_t)g.mx + 4, nj = (size_t)g.my + 4;
  if (!x->metrics_d) {
    if (cudaMalloc(&x->metrics_d, sizeof(double) * 3 * (size_t)g.plane) != cudaSuccess) return PCL_ERR_OOM;
    x->device_bytes += sizeof(double) * 3 * (size_t)g.plane;
  }
  const double* src[3] = {capacity, lrx, lry};
  for (int k = 0; k < 3; ++k)  // column-major (m_xi+4) x (m_eta+4) -> rows of `pitch` doubles
    CK(cudaMemcpy2DAsync(x->metrics_d + (size_t)k * g.plane, sizeof(double) * g.pitch, src[k], sizeof(double) * ni,
                         sizeof(double) * ni, nj, cudaMemcpyHostToDevice, x->stream));
  x->h2d_bytes += (long long)(3 * sizeof(double) * ni * nj);
  CK(cudaStreamSynchronize(x->stream));  // the caller's arrays may go away on return
  g.kap = x->metrics_d;
  g.lrx = x->metrics_d + g.plane;
  g.lry = x->metrics_d + 2 * g.plane;
  g.metric = kMetricMapped;
  drop_graph(x);
  return PCL_OK;
}

// NORM2 of a 2-vector (face length); exact whenever one component is zero
static double face_norm(double a, double b) {
  if (b == 0.0) return std::fabs(a);
  if (a == 0.0) return std::fabs(b);
  return std::sqrt(a * a + b * b);
}

int pcl_compute_mesh_metrics(const pcl_solver_control* c, pcl_map_fn map, void* user, double* kap, double* lrx,
                             double* lry) {
  if (!c || !kap || !lrx || !lry || c->m_xi < 1 || c->m_eta < 1) return PCL_ERR_BADARG;
  const double dxi = (c->xi_max - c->xi_min) / c->m_xi;      // SMOD_mesh_manipulation.f90:28
  const double deta = (c->eta_max - c->eta_min) / c->m_eta;  // :29
  const size_t ni = (size_t)c->m_xi + 4;
  for (int j = -1; j <= c->m_eta + 2; ++j) {
    for (int i = -1; i <= c->m_xi + 2; ++i) {
      // corners 1..4 counter-clockwise, 5 = 1 (:36-47)
      double xi[6], eta[6], x[6], y[6];
      xi[1] = c->xi_min + (double)(i - 1) * dxi;
      xi[2] = xi[1] + dxi;
      xi[3] = xi[2];
      xi[4] = xi[1];
      xi[5] = xi[1];
      eta[1] = c->eta_min + (double)(j - 1) * deta;
      eta[2] = eta[1];
      eta[3] = eta[2] + deta;
      eta[4] = eta[3];
      eta[5] = eta[1];
      for (int m = 1; m <= 5; ++m) {  // finalize_mesh :137-140
        if (map)
          map(xi[m], eta[m], &x[m], &y[m], user);
        else
          x[m] = xi[m], y[m] = eta[m];
      }
      const size_t o = (size_t)(j + 1) * ni + (size_t)(i + 1);
      lrx[o] = face_norm(x[4] - x[1], y[4] - y[1]) / deta;  // :147-153
      lry[o] = face_norm(x[2] - x[1], y[2] - y[1]) / dxi;   // :156-162
      double area = 0.0;                                     // :165-170
      for (int m = 1; m <= 4; ++m) area = area + (0.5 * (y[m] + y[m + 1])) * (x[m] - x[m + 1]);
      kap[o] = area / (dxi * deta);                          // :173
    }
  }
  return PCL_OK;
}

int pcl_set_tile_rows(pcl_ctx* x, int rows) {
  if (!x || rows < 4) return PCL_ERR_BADARG;
  if (x->mixed) mixed_set_tile_rows(x->mixed, rows);
  drop_graph(x);  // the captured launches carry the old tiling
  return PCL_OK;
}

int pcl_set_sweep_shape(pcl_ctx* x, int eta_shape) {
  if (!x || eta_shape < PCL_SHAPE_AUTO || eta_shape > PCL_SHAPE_BAND) return PCL_ERR_BADARG;
  static_assert(PCL_SHAPE_WINDOW == kEtaWindow && PCL_SHAPE_BAND == kEtaBand, "shape codes");
  x->g.eta_shape = eta_shape;
  drop_graph(x);  // the captured launches run the other kernel
  return PCL_OK;
}

int pcl_get_sweep_shape(pcl_ctx* x, int* eta_shape) {
  if (!x || !eta_shape) return PCL_ERR_BADARG;
  *eta_shape = eta_shape_of(x->g);
  return PCL_OK;
}

int pcl_inject_copy_stall(pcl_ctx* x, int row, unsigned probes) {
  if (!x || !x->mixed || row < -1 || row > x->cfg.m_eta + 2) return PCL_ERR_BADARG;
  mixed_set_injection(x->mixed, row, probes);
  drop_graph(x);  // the captured launches run the other build
  return PCL_OK;
}

int pcl_get_io_bytes(pcl_ctx* x, long long* h2d, long long* d2h) {
  if (!x) return PCL_ERR_BADARG;
  if (h2d) *h2d = x->h2d_bytes;
  if (d2h) *d2h = x->d2h_bytes;
  return PCL_OK;
}

int pcl_host_alloc(void** p, long long bytes) {
  if (!p || bytes <= 0) return PCL_ERR_BADARG;
  if (cudaMallocHost(p, (size_t)bytes) != cudaSuccess) return PCL_ERR_OOM;
  return PCL_OK;
}
int pcl_host_free(void* p) {
  if (p) cudaFreeHost(p);
  return PCL_OK;
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// snapshot writer (utility/MOD_IO.f90:397-460, writeData)
// ------------------------------------------------------------------------------------------
namespace {

// One value in Fortran's E26.16 edit descriptor: right-justified "[-]0.<16 digits>E+ee" (the
// exponent letter is dropped for |exponent| > 99, as Fortran does), from the correctly rounded
// 16 significant digits that printf's %.15e gives.
void put_e26_16(double v, char* out) {
  char buf[40], field[32];
  int n;
  if (std::isnan(v)) {
    n = std::snprintf(field, sizeof field, "NaN");
  } else if (std::isinf(v)) {
    n = std::snprintf(field, sizeof field, "%s", v < 0 ? "-Infinity" : "Infinity");
  } else {
    std::snprintf(buf, sizeof buf, "%.15e", v);  // [-]d.ddddddddddddddde[+-]XX[X]
    const char* p = buf;
    const bool neg = *p == '-';
    if (neg) ++p;
    char digits[17];
    digits[0] = p[0];
    std::memcpy(digits + 1, p + 2, 15);
    digits[16] = 0;
    const char* e = std::strchr(p, 'e');
    int ex = std::atoi(e + 1) + 1;
    if (v == 0.0) ex = 0;
    const int ax = ex < 0 ? -ex : ex;
    if (ax <= 99)
      n = std::snprintf(field, sizeof field, "%s0.%sE%c%02d", neg ? "-" : "", digits, ex < 0 ? '-' : '+', ax);
    else
      n = std::snprintf(field, sizeof field, "%s0.%s%c%03d", neg ? "-" : "", digits, ex < 0 ? '-' : '+', ax);
  }
  std::memset(out, ' ', 26);
  std::memcpy(out + 26 - n, field, (size_t)n);
}

bool make_dir(const std::string& d) { return ::mkdir(d.c_str(), 0755) == 0 || errno == EEXIST; }

// Format `cells` records of `per` values (3 for qout, num_aux zeros for aout when q is null) in
// parallel row blocks and write them in order.
bool write_records(const std::string& path, const double* q, long long cells, int per) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const size_t line = (size_t)per * 26 + 1;
  const int nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const long long block = 1LL << 16;  // records per thread and round
  std::vector<std::string> parts(nt);
  bool ok = true;
  for (long long base = 0; base < cells && ok; base += block * nt) {
    std::vector<std::thread> ts;
    for (int t = 0; t < nt; ++t) {
      ts.emplace_back([&, t] {
        const long long a = base + (long long)t * block, b = std::min(cells, a + block);
        std::string& s = parts[t];
        s.assign(a < b ? (size_t)(b - a) * line : 0, ' ');
        for (long long c = a; c < b; ++c) {
          char* o = &s[(size_t)(c - a) * line];
          for (int k = 0; k < per; ++k) put_e26_16(q ? q[c * per + k] : 0.0, o + 26 * k);
          o[line - 1] = '\n';
        }
      });
    }
    for (auto& th : ts) th.join();
    for (int t = 0; t < nt && ok; ++t) ok = std::fwrite(parts[t].data(), 1, parts[t].size(), f) == parts[t].size();
  }
  return std::fclose(f) == 0 && ok;
}

}  // namespace

int pcl_write_snapshot(pcl_ctx* x, const char* output_dir, int wait) {
  if (!x || !output_dir) return PCL_ERR_BADARG;
  CK(cudaSetDevice(x->device));
  if (x->snap_thread.joinable()) x->snap_thread.join();  // the previous snapshot owns the buffer
  const long long n = pcl_state_doubles(x);
  if (!x->snap_h && cudaMallocHost(&x->snap_h, sizeof(double) * (size_t)n) != cudaSuccess) return PCL_ERR_OOM;
  if (!x->snap_ev && cudaEventCreateWithFlags(&x->snap_ev, cudaEventDisableTiming) != cudaSuccess) return PCL_ERR_CUDA;
  int r = read_ctl(x);
  if (r != PCL_OK) return r;
  const double time = x->ctl_h->time;
  launch_download(x->g, x->staging_d, x->stream);
  r = check_launch(x);
  if (r != PCL_OK) return r;
  CK(cudaMemcpyAsync(x->snap_h, x->staging_d, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaEventRecord(x->snap_ev, x->stream));
  x->d2h_bytes += (long long)sizeof(double) * n;
  // output/<time F20.10, left-adjusted>/rank_0/{qout,aout}.dat (MOD_IO.f90:420-438)
  char ts[64];
  std::snprintf(ts, sizeof ts, "%.10f", time);
  const std::string dir = std::string(output_dir) + "/" + ts;
  const std::string sub = dir + "/rank_0";
  const long long cells = (long long)(x->cfg.m_xi + 4) * (x->cfg.m_eta + 4);
  const int naux = x->cfg.num_aux;
  const int neq = x->cfg.num_equations;
  x->snap_status = PCL_OK;
  x->snap_thread = std::thread([x, dir, sub, cells, naux, neq] {
    int st = PCL_OK;
    if (cudaEventSynchronize(x->snap_ev) != cudaSuccess) st = PCL_ERR_CUDA;
    if (st == PCL_OK && !(make_dir(dir) && make_dir(sub))) st = PCL_ERR_IO;
    if (st == PCL_OK && !write_records(sub + "/qout.dat", x->snap_h, cells, neq)) st = PCL_ERR_IO;
    // the SWE never sets its aux fields: num_aux zeros per cell
    if (st == PCL_OK && !write_records(sub + "/aout.dat", nullptr, cells, naux)) st = PCL_ERR_IO;
    x->snap_status = st;
  });
  return wait ? pcl_snapshot_wait(x) : PCL_OK;
}

int pcl_snapshot_wait(pcl_ctx* x) {
  if (!x) return PCL_ERR_BADARG;
  if (x->snap_thread.joinable()) x->snap_thread.join();
  return x->snap_status;
}

int pcl_format_e26_16(double v, char* out) {
  if (!out) return PCL_ERR_BADARG;
  put_e26_16(v, out);
  out[26] = 0;
  return PCL_OK;
}
