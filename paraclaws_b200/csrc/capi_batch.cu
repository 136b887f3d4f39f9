// capi_batch.cu -- C ABI of the batching form: many independent grids (instances) of uneven
// size, each with its own time control, advanced together by one persistent kernel launch per
// attempted step (batch_fp64.cu / batch_mixed.cu), in CUDA graphs.  The slot table, the work
// items and their counts live in device memory, so adding or removing an instance between steps
// changes what the captured launches do without capturing them again.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/paraclaws_b200.h"
#include "pcl_batch.h"
#include "pcl_launch.h"
#include "pcl_types.h"

using namespace pcl;

extern "C" int validate_control(const pcl_solver_control* c);
extern "C" void init_ctl(const pcl_solver_control* c, Ctl& t);
extern "C" void build_tables(const pcl_solver_control* c, double dxi, double deta, std::vector<double>& rowm,
                             std::vector<double>& colm);

namespace {

constexpr long long kBatchLogCap = 8192;
constexpr int kMixedStrip = 124;

struct Slot {
  bool used = false;
  pcl_solver_control cfg{};
  GridDev g{};
  double* mem = nullptr;  // one allocation: state buffers, tables, control block, log
  size_t bytes = 0;
};

size_t instance_layout(const pcl_solver_control* c, long long* plane, int* pitch, size_t* off_tab, size_t* off_ctl,
                       size_t* off_log) {
  const int ni = c->m_xi + 4, nj = c->m_eta + 4;
  const int p = (ni + 31) / 32 * 32;
  const long long pl = (long long)p * nj;
  size_t off = sizeof(double) * 9 * (size_t)pl;
  const size_t tab = off;
  off += sizeof(double) * ((size_t)nj * kRowMetrics + (size_t)ni * kColMetrics);
  off = (off + 255) / 256 * 256;
  const size_t ctl = off;
  off += sizeof(Ctl);
  off = (off + 255) / 256 * 256;
  const size_t lg = off;
  off += sizeof(StepLogEntry) * kBatchLogCap;
  if (plane) *plane = pl;
  if (pitch) *pitch = p;
  if (off_tab) *off_tab = tab;
  if (off_ctl) *off_ctl = ctl;
  if (off_log) *off_log = lg;
  return off;
}

}  // namespace

struct pcl_batch {
  int device = 0;
  int precision = PCL_PREC_FP64;
  cudaStream_t stream = nullptr;
  std::vector<Slot> slots;
  GridDev* inst_d = nullptr;
  int4* items_d = nullptr;
  long long items_cap = 0;
  int* scal_d = nullptr;       // [0] n_items, [1] queue head, [2] timeout flags of the last steps
  int* flags_h = nullptr;      // pinned copy of scal_d[2]
  int* counters_d = nullptr;
  int* totals_d = nullptr;
  int* poll_d = nullptr;       // [4*max_slots]: used flags, then done/status/accepted per slot
  double* staging_d = nullptr;
  size_t staging_bytes = 0;
  Ctl* ctl_h = nullptr;
  bool dirty = true;
  int n_items = 0;
  // schedule (the autotuner's knobs)
  // tile_rows 0: chosen per membership.  y_rows: an eta item of c rows takes (c + 4) / 32 steps
  // of its band (the first fills the 4-row halo), so 124 leaves no step half used.
  int x_rows = 8, y_rows = 124, tile_rows = 0, blocks_per_sm = 0;
  int tile_rows_eff = 64;  // rows per mixed item in the current items (a launch parameter)
  int desc_base = -1;  // mixed: first descriptor of this batch in the constant pool (-1: none)
  int mode = -1;       // mixed: the mode every instance shares (the specialised build), or -1
  int item_ghosts = 0;  // edge items fill ghost cells (few items per step), else the finisher does
  int fast_div = 1;     // FP64: every instance's g is inside the shared-reciprocal range
  int launch_ctas = 0;  // CTAs per launch: the persistent grid, or fewer when there are fewer items
  cudaGraphExec_t graph = nullptr;
  int graph_chunk = 0;
  long long launches = 0;
  long long steps = 0;
  unsigned spin_limit = 1u << 24;  // bounded wait of an FP64 eta item (about a second)
  int stall_slot = -1;             // pcl_batch_inject_stall
};

#define BCK(call)                                                                          \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      std::fprintf(stderr, "paraclaws_b200 batch: %s: %s\n", #call, cudaGetErrorString(e_)); \
      return PCL_ERR_CUDA;                                                                 \
    }                                                                                      \
  } while (0)

static int status_code(int st) {
  if (st & kStatusNaN) return PCL_ERR_NAN;
  if (st & kStatusNegDepth) return PCL_ERR_NEG_DEPTH;
  if (st & kStatusTimeout) return PCL_ERR_TIMEOUT;
  if (st & kStatusFatalDt) return PCL_ERR_FATAL_DT;
  return PCL_OK;
}

static void drop_graph(pcl_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_chunk = 0;
}

static BatchView view(const pcl_batch* b) {
  BatchView v;
  v.inst = b->inst_d;
  v.items = b->items_d;
  v.n_items = b->scal_d;
  v.head = reinterpret_cast<unsigned*>(b->scal_d + 1);
  v.counters = b->counters_d;
  v.totals = b->totals_d;
  v.x_rows = b->x_rows;
  v.y_rows = b->y_rows;
  v.tile_rows = b->tile_rows_eff;
  v.desc_base = b->desc_base;
  v.item_ghosts = b->item_ghosts;
  v.spin_limit = b->spin_limit;
  v.flags = b->scal_d + 2;
  v.stall_slot = b->stall_slot;
  v.fast_div = b->fast_div;
  return v;
}

static int grid_size(const pcl_batch* b) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  const int occ =
      b->precision == PCL_PREC_MIXED ? batch_mixed_occupancy(b->desc_base >= 0, b->mode) : batch_fp64_occupancy();
  const int per = b->blocks_per_sm > 0 ? std::min(b->blocks_per_sm, occ) : occ;
  return sms * per;
}

// Rows per mixed item when the schedule leaves it open (tile_rows 0): the height that minimises
// the estimated step time, waves x (rows an item streams + a fixed cost per item), where waves
// is the item count over the persistent CTAs, rounded up, over heights 8 ... 128.  A few small instances get short
// items spread over the SMs (a step takes about one item's time); a large batch gets taller
// items whose four halo rows cost less.
constexpr int kItemFixedRows = 8;

static int auto_tile_rows(const pcl_batch* b, const std::vector<int>& order) {
  const long long ctas = std::max(1, grid_size(b));
  int best = 64;
  double best_cost = 1e300;
  // 256-row items are left out: their rows measured ~12% slower than 128-row items' on large
  // grids, which the wave count does not see
  for (int ty : {8, 16, 32, 64, 128}) {
    long long n = 0;
    for (int s : order) {
      const auto& c = b->slots[s].cfg;
      n += (long long)((c.m_xi + kMixedStrip - 1) / kMixedStrip) * ((c.m_eta + ty - 1) / ty);
    }
    const double cost = (double)((n + ctas - 1) / ctas) * (ty + 4 + kItemFixedRows);
    if (cost <= best_cost) {  // ties: the taller item (fewer of them)
      best_cost = cost;
      best = ty;
    }
  }
  return best;
}

// Work items of every used slot, largest instances first so the long items start early.
static int rebuild_items(pcl_batch* b) {
  std::vector<int> order;
  for (int s = 0; s < (int)b->slots.size(); ++s)
    if (b->slots[s].used) order.push_back(s);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    const auto& A = b->slots[a].cfg;
    const auto& B = b->slots[c].cfg;
    return (long long)A.m_xi * A.m_eta > (long long)B.m_xi * B.m_eta;
  });
  std::vector<int4> items;
  std::vector<int> totals(2 * b->slots.size(), 0);
  if (b->precision == PCL_PREC_MIXED) {
    int mode = -2;
    for (int s : order) {
      const GridDev& g = b->slots[s].g;
      const int m = g.second_order ? 1 + g.limiter : 0;
      mode = mode == -2 ? m : (mode == m ? m : -1);
    }
    // an empty batch keeps its build (and its captured graph) for the next instance
    if (mode != -2) {
      if (mode < 0) mode = -1;
      if (mode != b->mode) drop_graph(b);  // the captured launches run the other build
      b->mode = mode;
    }
    if (!order.empty()) {
      const int ty = b->tile_rows > 0 ? b->tile_rows : auto_tile_rows(b, order);
      if (ty != b->tile_rows_eff) drop_graph(b);  // the captured launches carry the old height
      b->tile_rows_eff = ty;
    }
    for (int s : order) {
      const auto& c = b->slots[s].cfg;
      const int ns = (c.m_xi + kMixedStrip - 1) / kMixedStrip;
      const int nr = (c.m_eta + b->tile_rows_eff - 1) / b->tile_rows_eff;
      for (int r = 0; r < nr; ++r)
        for (int k = 0; k < ns; ++k) items.push_back(make_int4(s, kItemMixed, k, r));
      totals[2 * s + 1] = ns * nr;
    }
  } else {
    for (int s : order) {
      const auto& c = b->slots[s].cfg;
      const int xseg = batch_fp64_segment();
      const int nseg = (c.m_xi + xseg - 1) / xseg;
      int nx = 0;
      for (int j = 1; j <= c.m_eta; j += b->x_rows)
        for (int k = 0; k < nseg; ++k, ++nx) items.push_back(make_int4(s, kItemX, j, 1 + k * xseg));
      totals[2 * s] = nx;
    }
    for (int s : order) {
      const auto& c = b->slots[s].cfg;
      int ny = 0;
      // bands start at column -1 + 4k (sector-aligned rows); the last one holds column m_xi
      for (int j0 = 1; j0 <= c.m_eta; j0 += b->y_rows)
        for (int i0 = -1; i0 <= c.m_xi; i0 += batch_fp64_band(), ++ny) items.push_back(make_int4(s, kItemY, i0, j0));
      totals[2 * s + 1] = totals[2 * s] + ny;
    }
    // the shared-reciprocal quotients' range argument holds for g in [2^-20, 2^20]
    int fd = 1;
    for (int s : order) {
      const double g = b->slots[s].g.grav;
      if (!(g >= 0x1p-20 && g <= 0x1p20)) fd = 0;
    }
    if (!order.empty()) {
      if (fd != b->fast_div) drop_graph(b);  // a launch parameter of the captured launches
      b->fast_div = fd;
    }
  }
  if ((long long)items.size() > b->items_cap) {
    cudaFree(b->items_d);
    b->items_d = nullptr;
    b->items_cap = std::max<long long>((long long)items.size() * 2, 1 << 16);
    BCK(cudaMalloc(&b->items_d, sizeof(int4) * b->items_cap));
    drop_graph(b);  // the captured launches point at the old item array
  }
  b->n_items = (int)items.size();
  if (!items.empty()) {
    // The finishing CTA's ghost fill (8 max(m_xi, m_eta) cells) is hidden only behind other
    // instances' items.  Edge items fill the ghosts instead when a step is up to two waves of
    // items (it lasts a few items) or when one instance holds most of the items (its finisher
    // would run at the end of the step, alone).
    long long largest = 0;
    for (int s : order) largest = std::max<long long>(largest, totals[2 * s + 1]);
    const long long n = (long long)items.size();
    const int ig = n <= 2LL * grid_size(b) || 2 * largest > n ? 1 : 0;
    if (ig != b->item_ghosts) drop_graph(b);  // a launch parameter of the captured launches
    b->item_ghosts = ig;
    // a CTA without an item only sets up its ring and leaves: launch no more CTAs than items
    const int ctas = (int)std::min<long long>(grid_size(b), n);
    if (ctas != b->launch_ctas) drop_graph(b);
    b->launch_ctas = ctas;
  }
  if (!items.empty())
    BCK(cudaMemcpyAsync(b->items_d, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->totals_d, totals.data(), sizeof(int) * totals.size(), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->scal_d, &b->n_items, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemsetAsync(b->counters_d, 0, sizeof(int) * 2 * b->slots.size(), b->stream));
  BCK(cudaStreamSynchronize(b->stream));  // the host vectors go out of scope
  b->dirty = false;
  return PCL_OK;
}

static void enqueue_step(pcl_batch* b) {
  cudaMemsetAsync(b->scal_d + 1, 0, sizeof(int), b->stream);
  const BatchView v = view(b);
  if (b->precision == PCL_PREC_MIXED)
    launch_batch_mixed(v, b->launch_ctas, b->desc_base >= 0, b->mode, b->stream);
  else
    launch_batch_fp64(v, b->launch_ctas, b->stream);
}

extern "C" {

long long pcl_batch_instance_bytes(const pcl_solver_control* c) {
  if (!c) return 0;
  return (long long)instance_layout(c, nullptr, nullptr, nullptr, nullptr, nullptr);
}

int pcl_batch_create(int device, int precision, int max_instances, pcl_batch** out) {
  if (!out || max_instances < 1 || (precision != PCL_PREC_FP64 && precision != PCL_PREC_MIXED)) return PCL_ERR_BADARG;
  *out = nullptr;
  BCK(cudaSetDevice(device));
  auto* b = new pcl_batch();
  b->device = device;
  b->precision = precision;
  b->slots.resize(max_instances);
  auto fail = [&](int code) {
    cudaFree(b->inst_d);
    cudaFree(b->scal_d);
    cudaFree(b->counters_d);
    cudaFree(b->totals_d);
    cudaFree(b->poll_d);
    if (b->ctl_h) cudaFreeHost(b->ctl_h);
    if (b->flags_h) cudaFreeHost(b->flags_h);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return code;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PCL_ERR_CUDA);
  if (cudaMalloc(&b->inst_d, sizeof(GridDev) * max_instances) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&b->scal_d, sizeof(int) * 4) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&b->counters_d, sizeof(int) * 2 * max_instances) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&b->totals_d, sizeof(int) * 2 * max_instances) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMalloc(&b->poll_d, sizeof(int) * 4 * max_instances) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMallocHost(&b->ctl_h, sizeof(Ctl)) != cudaSuccess) return fail(PCL_ERR_OOM);
  if (cudaMallocHost(&b->flags_h, sizeof(int)) != cudaSuccess) return fail(PCL_ERR_OOM);
  *b->flags_h = 0;
  cudaMemsetAsync(b->scal_d, 0, sizeof(int) * 4, b->stream);
  cudaMemsetAsync(b->counters_d, 0, sizeof(int) * 2 * max_instances, b->stream);
  cudaMemsetAsync(b->totals_d, 0, sizeof(int) * 2 * max_instances, b->stream);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return fail(PCL_ERR_CUDA);
  // a mixed batch takes a range of the constant descriptor pool if one is free (else its items
  // read their descriptors from global memory)
  if (precision == PCL_PREC_MIXED) b->desc_base = batch_desc_reserve(max_instances);
  *out = b;
  return PCL_OK;
}

int pcl_batch_destroy(pcl_batch* b) {
  if (!b) return PCL_ERR_BADARG;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (auto& s : b->slots)
    if (s.mem) cudaFree(s.mem);
  cudaFree(b->inst_d);
  cudaFree(b->items_d);
  cudaFree(b->scal_d);
  cudaFree(b->counters_d);
  cudaFree(b->totals_d);
  cudaFree(b->poll_d);
  cudaFree(b->staging_d);
  cudaFreeHost(b->ctl_h);
  cudaFreeHost(b->flags_h);
  cudaStreamDestroy(b->stream);
  if (b->desc_base >= 0) batch_desc_release(b->desc_base, (int)b->slots.size());
  delete b;
  return PCL_OK;
}

int pcl_batch_add(pcl_batch* b, const pcl_solver_control* c, const double* vars, int* slot_out) {
  if (!b || !c || !slot_out) return PCL_ERR_BADARG;
  if (!vars && c->initial_condition != 1) return PCL_ERR_BADARG;
  int v = validate_control(c);
  if (v != PCL_OK) return v;
  if (c->precision_mode != b->precision || c->num_equations != 3) return PCL_ERR_BADARG;
  int s = -1;
  for (int k = 0; k < (int)b->slots.size(); ++k)
    if (!b->slots[k].used) {
      s = k;
      break;
    }
  if (s < 0) return PCL_ERR_FULL;
  BCK(cudaSetDevice(b->device));
  Slot& sl = b->slots[s];
  long long plane;
  int pitch;
  size_t off_tab, off_ctl, off_log;
  const size_t bytes = instance_layout(c, &plane, &pitch, &off_tab, &off_ctl, &off_log);
  char* mem = nullptr;
  if (cudaMalloc(&mem, bytes) != cudaSuccess) return PCL_ERR_OOM;
  const double dxi = (c->xi_max - c->xi_min) / c->m_xi;
  const double deta = (c->eta_max - c->eta_min) / c->m_eta;
  std::vector<double> rowm, colm;
  build_tables(c, dxi, deta, rowm, colm);
  Ctl* h = b->ctl_h;
  init_ctl(c, *h);
  h->log = reinterpret_cast<StepLogEntry*>(mem + off_log);
  h->log_cap = kBatchLogCap;
  GridDev g{};
  g.state = reinterpret_cast<double*>(mem);
  g.bufstride = 3 * plane;
  g.neq = 3;
  g.rowm = reinterpret_cast<double*>(mem + off_tab);
  g.colm = g.rowm + rowm.size();
  g.ctl = reinterpret_cast<Ctl*>(mem + off_ctl);
  g.plane = plane;
  g.mx = c->m_xi;
  g.my = c->m_eta;
  g.pitch = pitch;
  g.bc[0] = c->bc_xi_lower; g.bc[1] = c->bc_xi_upper; g.bc[2] = c->bc_eta_lower; g.bc[3] = c->bc_eta_upper;
  g.second_order = c->higher_order_flux_correction ? 1 : 0;
  g.limiter = c->use_limiter ? c->limiter_method : 0;
  g.dxi = dxi;
  g.deta = deta;
  g.area_scale = dxi * deta;
  g.grav = c->grav;
  const size_t stg = sizeof(double) * 3 * (size_t)(c->m_xi + 4) * (c->m_eta + 4);
  if (vars && stg > b->staging_bytes) {
    cudaFree(b->staging_d);
    b->staging_d = nullptr;
    if (cudaMalloc(&b->staging_d, stg) != cudaSuccess) {
      cudaFree(mem);
      b->staging_bytes = 0;
      return PCL_ERR_OOM;
    }
    b->staging_bytes = stg;
  }
  BCK(cudaMemcpyAsync(const_cast<double*>(g.rowm), rowm.data(), sizeof(double) * rowm.size(), cudaMemcpyHostToDevice,
                      b->stream));
  BCK(cudaMemcpyAsync(const_cast<double*>(g.colm), colm.data(), sizeof(double) * colm.size(), cudaMemcpyHostToDevice,
                      b->stream));
  BCK(cudaMemcpyAsync(g.ctl, h, sizeof(Ctl), cudaMemcpyHostToDevice, b->stream));
  if (vars) {
    BCK(cudaMemcpyAsync(b->staging_d, vars, stg, cudaMemcpyHostToDevice, b->stream));
    launch_upload(g, b->staging_d, b->stream);
  } else {
    launch_dam_ic(g, c->dam_radius, c->dam_h_in, c->dam_h_out, c->dam_x0, c->dam_y0, b->stream);
  }
  launch_ghost(g, 1, b->stream);
  launch_timectl(g, kOpInit, 0, 0.0, b->stream);
  launch_metric_check(g, b->stream);
  b->launches += 4;
  BCK(cudaMemcpyAsync(&h->nonunit_metric, &g.ctl->nonunit_metric, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  g.metric = h->nonunit_metric ? kMetricTable : kMetricUnit;
  BCK(cudaMemcpyAsync(b->inst_d + s, &g, sizeof(GridDev), cudaMemcpyHostToDevice, b->stream));
  if (b->desc_base >= 0) {
    ItemDesc d{};
    d.state = g.state;
    d.bufstride = g.bufstride;
    d.plane = g.plane;
    d.ctl = g.ctl;
    d.grav = g.grav;
    d.mx = g.mx;
    d.my = g.my;
    d.pitch = g.pitch;
    d.mode = g.second_order ? 1 + g.limiter : 0;
    BCK(batch_mixed_set_desc(b->desc_base + s, d, b->stream));
  }
  BCK(cudaGetLastError());
  BCK(cudaStreamSynchronize(b->stream));
  sl.used = true;
  sl.cfg = *c;
  sl.g = g;
  sl.mem = reinterpret_cast<double*>(mem);
  sl.bytes = bytes;
  b->dirty = true;
  *slot_out = s;
  return PCL_OK;
}

int pcl_batch_remove(pcl_batch* b, int s) {
  if (!b || s < 0 || s >= (int)b->slots.size() || !b->slots[s].used) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaStreamSynchronize(b->stream));
  cudaFree(b->slots[s].mem);
  b->slots[s] = Slot();
  b->dirty = true;
  return PCL_OK;
}

int pcl_batch_set_schedule(pcl_batch* b, int tile_rows, int x_rows, int y_rows, int blocks_per_sm) {
  if (!b || (tile_rows != 0 && tile_rows < 4) || x_rows < 1 || y_rows < 1 || blocks_per_sm < 0) return PCL_ERR_BADARG;
  b->tile_rows = tile_rows;
  b->x_rows = x_rows;
  b->y_rows = y_rows;
  b->blocks_per_sm = blocks_per_sm;
  b->dirty = true;
  drop_graph(b);
  return PCL_OK;
}

int pcl_batch_step(pcl_batch* b, int nsteps) {
  if (!b || nsteps < 0) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  if (b->dirty) {
    int r = rebuild_items(b);
    if (r != PCL_OK) return r;
  }
  if (b->n_items == 0 || nsteps == 0) return PCL_OK;
  const int chunk = 16;
  if (nsteps >= chunk && b->graph_chunk != chunk) {
    drop_graph(b);
    cudaGraph_t gr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < chunk; ++k) enqueue_step(b);
    BCK(cudaStreamEndCapture(b->stream, &gr));
    cudaError_t e = cudaGraphInstantiate(&b->graph, gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return PCL_ERR_CUDA;
    b->graph_chunk = chunk;
  }
  int left = nsteps;
  while (left >= chunk) {
    BCK(cudaGraphLaunch(b->graph, b->stream));
    left -= chunk;
  }
  for (; left > 0; --left) enqueue_step(b);
  b->launches += nsteps;
  b->steps += nsteps;
  BCK(cudaGetLastError());
  // did a bounded wait give up during these steps?  (read and cleared in stream order)
  BCK(cudaMemcpyAsync(b->flags_h, b->scal_d + 2, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaMemsetAsync(b->scal_d + 2, 0, sizeof(int), b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return *b->flags_h ? PCL_ERR_TIMEOUT : PCL_OK;
}

int pcl_batch_inject_stall(pcl_batch* b, int slot, unsigned spin_limit) {
  if (!b || slot < -1 || slot >= (int)b->slots.size() || b->precision != PCL_PREC_FP64) return PCL_ERR_BADARG;
  b->stall_slot = slot;
  b->spin_limit = spin_limit > 0 ? spin_limit : (1u << 24);
  drop_graph(b);  // the captured launches carry the old view
  return PCL_OK;
}

int pcl_batch_stats(pcl_batch* b, int s, pcl_run_stats* st) {
  if (!b || !st || s < 0 || s >= (int)b->slots.size() || !b->slots[s].used) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaMemcpyAsync(b->ctl_h, b->slots[s].g.ctl, offsetof(Ctl, snap_times), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  const Ctl& c = *b->ctl_h;
  st->attempts = c.attempts;
  st->accepted = c.accepted;
  st->rejected = c.attempts - c.accepted;
  st->launches = b->launches;
  st->time = c.time;
  st->dt = c.dt;
  st->dt_previous = c.dt_previous;
  st->cfl = c.CFL;
  st->snapshot_index = c.snapshot_index;
  st->done = c.done;
  st->status = status_code(c.status);
  st->last_ierr = c.ierr;
  return PCL_OK;
}

int pcl_batch_download(pcl_batch* b, int s, double* vars) {
  if (!b || !vars || s < 0 || s >= (int)b->slots.size() || !b->slots[s].used) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  const auto& c = b->slots[s].cfg;
  const size_t stg = sizeof(double) * 3 * (size_t)(c.m_xi + 4) * (c.m_eta + 4);
  if (stg > b->staging_bytes) {
    cudaFree(b->staging_d);
    b->staging_d = nullptr;
    b->staging_bytes = 0;
    if (cudaMalloc(&b->staging_d, stg) != cudaSuccess) return PCL_ERR_OOM;
    b->staging_bytes = stg;
  }
  launch_download(b->slots[s].g, b->staging_d, b->stream);
  b->launches += 1;
  BCK(cudaMemcpyAsync(vars, b->staging_d, stg, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return PCL_OK;
}

int pcl_batch_get_step_log(pcl_batch* b, int s, pcl_step_record* out, long long cap, long long* n) {
  if (!b || s < 0 || s >= (int)b->slots.size() || !b->slots[s].used) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  BCK(cudaMemcpyAsync(b->ctl_h, b->slots[s].g.ctl, offsetof(Ctl, snap_times), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  const long long len = b->ctl_h->log_len;
  if (n) *n = len;
  const long long m = std::min(len, cap);
  if (out && m > 0) {
    std::vector<StepLogEntry> tmp((size_t)m);
    BCK(cudaMemcpy(tmp.data(), b->ctl_h->log, sizeof(StepLogEntry) * m, cudaMemcpyDeviceToHost));
    for (long long k = 0; k < m; ++k)
      out[k] = pcl_step_record{tmp[k].dt, tmp[k].cfl, tmp[k].time, tmp[k].dt_next, tmp[k].ierr, tmp[k].snapshot_index};
  }
  return PCL_OK;
}

int pcl_batch_info(pcl_batch* b, int* n_used, int* n_done, long long* cells, long long* device_bytes) {
  if (!b) return PCL_ERR_BADARG;
  int used = 0, dn = 0;
  long long cl = 0, by = 0;
  for (int s = 0; s < (int)b->slots.size(); ++s) {
    if (!b->slots[s].used) continue;
    used++;
    cl += (long long)b->slots[s].cfg.m_xi * b->slots[s].cfg.m_eta;
    by += (long long)b->slots[s].bytes;
  }
  if (n_done) {
    BCK(cudaSetDevice(b->device));
    for (int s = 0; s < (int)b->slots.size(); ++s) {
      if (!b->slots[s].used) continue;
      int d = 0;
      BCK(cudaMemcpyAsync(&d, &b->slots[s].g.ctl->done, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
      BCK(cudaStreamSynchronize(b->stream));
      dn += d != 0;
    }
    *n_done = dn;
  }
  if (n_used) *n_used = used;
  if (cells) *cells = cl;
  if (device_bytes) *device_bytes = by;
  return PCL_OK;
}

void* pcl_batch_get_stream(pcl_batch* b) { return b ? (void*)b->stream : nullptr; }

}  // extern "C"

// one thread per slot: done flag, status bits and accepted-step count of every used slot
__global__ void batch_poll_kernel(const GridDev* inst, const int* used, int n, int* out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  if (!used[s]) {
    out[3 * s] = out[3 * s + 1] = out[3 * s + 2] = -1;
    return;
  }
  const Ctl* c = inst[s].ctl;
  out[3 * s] = c->done;
  out[3 * s + 1] = c->status;
  out[3 * s + 2] = (int)c->accepted;
}

extern "C" {

int pcl_batch_poll(pcl_batch* b, int* done, int* status) {
  if (!b || !done) return PCL_ERR_BADARG;
  BCK(cudaSetDevice(b->device));
  const int n = (int)b->slots.size();
  std::vector<int> used(n), out(3 * (size_t)n);
  for (int s = 0; s < n; ++s) used[s] = b->slots[s].used ? 1 : 0;
  int* used_d = b->poll_d;
  int* res_d = b->poll_d + n;
  BCK(cudaMemcpyAsync(used_d, used.data(), sizeof(int) * n, cudaMemcpyHostToDevice, b->stream));
  batch_poll_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->inst_d, used_d, n, res_d);
  b->launches += 1;
  BCK(cudaGetLastError());
  BCK(cudaMemcpyAsync(out.data(), res_d, sizeof(int) * 3 * n, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  for (int s = 0; s < n; ++s) {
    done[s] = out[3 * s];
    if (status) status[s] = out[3 * s] < 0 ? 0 : status_code(out[3 * s + 1]);
  }
  return PCL_OK;
}

}  // extern "C"
