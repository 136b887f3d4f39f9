// pcl_sweeps_fp64.cuh -- the FP64 parity sweeps as device functions, shared by the per-sweep
// kernels of a single grid (kernels_fp64.cu) and the persistent batched kernel
// (batch_fp64.cu).  Include only from translation units built with --fmad=false.
//
// MK (metric kind, pcl_types.h): kMetricTable rebuilds kappa per cell from the row/column tables
// of the uniform grid; kMetricUnit is a uniform grid whose capacities and length ratios are all
// exactly 1.0 (checked once per grid by the metric-check kernel), so x/kappa, gamma*x and the
// capacity mean of the correction coefficient are identities and are left out (same bits);
// kMetricMapped reads the per-cell capacity and face length ratios of a mapped grid
// (MOD_solve.f90:211-233 reads length_ratio_xi(1,i,j) and (1,i+1,j) for the two faces of a cell).
//
// Buffer rotation replaces solution_old = solution (main.f90:201): the xi sweep reads buffer
// cur and writes the interior rows of buffer (cur+1)%3; the eta sweep reads those rows plus the
// pre-step ghost rows of buffer cur (ghosts are filled once per accepted step, main.f90:246) and
// writes buffer (cur+2)%3.  A rejected attempt never touches buffer cur.
#pragma once
#include <cuda_runtime.h>

#include "pcl_fp64.cuh"
#include "pcl_sm100.cuh"

namespace pcl {


// CFL bookkeeping shared by both sweeps: block max of s2, one atomic per block.
template <int NT>
__device__ __forceinline__ void block_max_to(unsigned long long* dst, double v, double* red) {
  v = warp_max(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double w = lane < NT / 32 ? red[lane] : 0.0;
    w = warp_max(w);
    if (lane == 0) atomic_max_nonneg(dst, w);
  }
}

// ------------------------------------------------------------------------------------------
// xi sweep.  One CTA = one row segment of L = NT-4 cells.  Thread t owns cell i0-2+t (phase A),
// interface i0-1+t (phase B), interface i0+t (phase C) and cell i0+t (phase D).
// ------------------------------------------------------------------------------------------
// Shared memory of one xi-sweep segment (per-slot cell data, waves, correction flux).
template <int NT>
struct XSmem {
  // sq and sk in two copies by row parity: phase D of a row reads them after its last barrier,
  // while phase A of the next row writes them, so consecutive rows need no barrier between them
  double sq[2][3][NT], sf[3][NT], ss[NT], sk[2][NT];
  double sw1[3][NT], sw2[3][NT], ss2[NT], sft[3][NT];
  double red[NT / 32];
  bool sok[NT];  // kOptFastDiv: the cell is in the range of the shared-reciprocal quotients
};

// End of an xi-sweep CTA: the wave-speed maximum and the status bits of all its rows.
template <int NT>
__device__ __forceinline__ void xsweep_finish(const GridDev& g, double smax, int bad, XSmem<NT>& S) {
  block_max_to<NT>(const_cast<unsigned long long*>(&g.ctl->smax_x), smax, S.red);
  if (bad) atomicOr(&g.ctl->status, bad);
}

// The specialised shallow-water module (other modules: pcl_sweeps_gen.cuh).  OPT: the kOpt*
// mask of pcl_fp64.cuh (same results for every value).  The row's wave-speed maximum is
// folded into smax_acc and its status bits into bad_acc; the caller reduces them over the CTA
// once for all the rows it sweeps (xsweep_finish).
// Rows swept one after another alternate `par` (0, 1, 0, ...) and need no barrier between them:
// every shared array phase D reads is either in the row's own parity copy or written by the next
// row only after that row's first barrier.
template <int NT, int LIM, bool SO, int MK = kMetricTable, int OPT = 0>
__device__ __forceinline__ void xsweep_segment(const GridDev& g, int j, int i0, XSmem<NT>& S, double& smax_acc,
                                               int& bad_acc, int par = 0) {
  constexpr bool UM = MK == kMetricUnit, MP = MK == kMetricMapped;
  const Ctl* ctl = g.ctl;
  constexpr int L = NT - 4;
  const int cur = ctl->cur, out = cur == 2 ? 0 : cur + 1;
  const double dtod = ctl->dtod_x;
  const int t = threadIdx.x;
  const int mx = g.mx;
  const long long row = (long long)(j + 1) * g.pitch;
  const double* q0 = buffer(g, cur) + row;
  const double* q1 = q0 + g.plane;
  const double* q2 = q1 + g.plane;

  auto& sq = S.sq[par];
  auto& sf = S.sf;
  auto& ss = S.ss;
  auto& sk = S.sk[par];
  auto& sw1 = S.sw1;
  auto& sw2 = S.sw2;
  auto& ss2 = S.ss2;
  auto& sft = S.sft;

  // phase A: per-cell flux J.q, wave-speed bound and capacity
  int bad = 0;
  {
    const int c = i0 - 2 + t;
    if (c <= mx + 2) {
      const double h = q0[c + 1], hu = q1[c + 1], hv = q2[c + 1];
      int cb = 0;
      const CellFlux F = cell_flux<0, OPT>(h, hu, hv, g.grav, &cb);
      if (c <= mx + 1) bad |= cb;  // getJakobi runs on cells -1 .. m_xi+1 in the xi sweep
      sq[0][t] = h; sq[1][t] = hu; sq[2][t] = hv;
      sf[0][t] = F.f0; sf[1][t] = F.f1; sf[2][t] = F.f2;
      ss[t] = F.s;
      if constexpr ((OPT & kOptFastDiv) != 0) S.sok[t] = F.ok;
      if constexpr (MP)
        sk[t] = __ldg(g.kap + row + c + 1);
      else if constexpr (!UM)
        sk[t] = capacity(g.rowm, g.colm, c, j, g.area_scale);
    }
  }
  __syncthreads();

  // phase B: HLL at interface k = i0-1+t between cells k-1 (slot t) and k (slot t+1)
  double smax = 0.0;
  if (t < NT - 1) {
    const int k = i0 - 1 + t;
    Waves W;
    double s2 = 0.0;
    if (k <= mx + 1) {
      const double qL[3] = {sq[0][t], sq[1][t], sq[2][t]};
      const double qR[3] = {sq[0][t + 1], sq[1][t + 1], sq[2][t + 1]};
      CellFlux FL = {sf[0][t], sf[1][t], sf[2][t], ss[t]};
      CellFlux FR = {sf[0][t + 1], sf[1][t + 1], sf[2][t + 1], ss[t + 1]};
      if constexpr ((OPT & kOptFastDiv) != 0) FL.ok = S.sok[t], FR.ok = S.sok[t + 1];
      s2 = hll<OPT>(qL, FL, qR, FR, W);
      smax = s2;
    } else {
#pragma unroll
      for (int me = 0; me < 3; ++me) W.w1[me] = W.w2[me] = 0.0;
    }
#pragma unroll
    for (int me = 0; me < 3; ++me) {
      sw1[me][t] = W.w1[me];
      sw2[me][t] = W.w2[me];
    }
    ss2[t] = s2;
  }
  smax_acc = fmax(smax_acc, smax);
  bad_acc |= bad;
  __syncthreads();

  // phase C: correction flux at interface k = i0+t (slot t+1); limited for 1 <= k <= m_xi,
  // the wave at k = m_xi+1 stays unlimited (MOD_flux_correction.f90:54-75 vs :159)
  if constexpr (SO) {
    if (t < NT - 3) {
      const int k = i0 + t;
      double ft[3] = {0.0, 0.0, 0.0};
      if (k <= mx + 1) {
        const int s = t + 1;
        const double s2 = ss2[s];
        const double cf = UM ? corr_coef_unit(s2, dtod) : corr_coef(s2, dtod, sk[t + 1], sk[t + 2]);
        if (cf != 0.0) {
          const double w1[3] = {sw1[0][s], sw1[1][s], sw1[2][s]};
          const double w2[3] = {sw2[0][s], sw2[1][s], sw2[2][s]};
          double a[3], b[3];
          if (LIM != 0 && k <= mx) {
            const double w1m[3] = {sw1[0][s - 1], sw1[1][s - 1], sw1[2][s - 1]};
            const double w1p[3] = {sw1[0][s + 1], sw1[1][s + 1], sw1[2][s + 1]};
            const double w2m[3] = {sw2[0][s - 1], sw2[1][s - 1], sw2[2][s - 1]};
            const double w2p[3] = {sw2[0][s + 1], sw2[1][s + 1], sw2[2][s + 1]};
            limit_wave<LIM, OPT>(w1m, w1, w1p, false, a);  // lambda_1 = -s2 <= 0
            limit_wave<LIM, OPT>(w2m, w2, w2p, s2 > 0.0, b);
          } else {
#pragma unroll
            for (int me = 0; me < 3; ++me) {
              a[me] = w1[me];
              b[me] = w2[me];
            }
          }
#pragma unroll
          for (int me = 0; me < 3; ++me) ft[me] = cf * a[me] + cf * b[me];
        }
      }
#pragma unroll
      for (int me = 0; me < 3; ++me) sft[me][t] = ft[me];
    }
    __syncthreads();
  }

  // phase D: update of cell i = i0+t (MOD_solve.f90:207-221 and :268-278)
  if (t < L) {
    const int i = i0 + t;
    if (i <= mx) {
      const int c = t + 2;
      const double gam = (UM || MP) ? 1.0 : __ldg(g.rowm + (j + 1) * kRowMetrics + 2);
      const double gl = MP ? __ldg(g.lrx + row + i + 1) : gam;  // face between cells i-1 and i
      const double gr = MP ? __ldg(g.lrx + row + i + 2) : gam;  // face between cells i and i+1
      const double dtk = UM ? dtod : dtod / sk[c];
      const double sp = ss2[t + 1];       // A+ at interface i:   s2 * W2
      const double sm = -ss2[t + 2];      // A- at interface i+1: s1 * W1
      double* o0 = buffer(g, out) + row;
#pragma unroll
      for (int me = 0; me < 3; ++me) {
        const double ap = sp * sw2[me][t + 1];
        const double am = sm * sw1[me][t + 2];
        double q = UM ? sq[me][c] - dtk * (ap + am) : sq[me][c] - dtk * (gl * ap + gr * am);
        if constexpr (SO) q = q - dtk * (sft[me][t + 1] - sft[me][t]);
        o0[me * g.plane + i + 1] = q;
      }
    }
  }
}

// xi-sweep validity (MOD_solve.f90:107-120), recomputed from the xi sweep's reduction word
__device__ __forceinline__ bool eta_valid(const GridDev& g) {
  const Ctl* ctl = g.ctl;
  // written by atomics of other CTAs in a batched launch: read at L2, not a stale L1 line
  const double sx = __longlong_as_double((long long)__ldcg(&ctl->smax_x));
  const double cflx = sx * ctl->dt / g.dxi;
  const double cfl = fmax(ctl->CFL, cflx);
  return ctl->CFL_target / cfl >= ctl->shrink;
}

// ------------------------------------------------------------------------------------------
// eta sweep.  One thread = one column i, marching over a strip of rows [j0, j1] with a
// register window of three interfaces.  Loads of consecutive threads are consecutive doubles.
// ------------------------------------------------------------------------------------------
struct YCell {
  double q[3];
  CellFlux F;
  double kap;
  double lr;  // mapped grids: length ratio of the eta face below the cell
};

template <int LIM, bool SO, bool UM, int OPT = 0>
__device__ __forceinline__ void y_corr_flux(const Waves& Wm, const Waves& W, const Waves& Wp, double s2,
                                            bool limited, double dtod, double kl, double kr, double ft[3]) {
  const double cf = UM ? corr_coef_unit(s2, dtod) : corr_coef(s2, dtod, kl, kr);
  if (cf == 0.0) {
    ft[0] = ft[1] = ft[2] = 0.0;
    return;
  }
  double a[3], b[3];
  if (LIM != 0 && limited) {
    limit_wave<LIM, OPT>(Wm.w1, W.w1, Wp.w1, false, a);
    limit_wave<LIM, OPT>(Wm.w2, W.w2, Wp.w2, s2 > 0.0, b);
  } else {
#pragma unroll
    for (int me = 0; me < 3; ++me) {
      a[me] = W.w1[me];
      b[me] = W.w2[me];
    }
  }
#pragma unroll
  for (int me = 0; me < 3; ++me) ft[me] = cf * a[me] + cf * b[me];
}

// UNR unrolls the row loop (the window's shift then becomes register renaming); it changes no
// arithmetic.
template <int LIM, bool SO, int MK = kMetricTable, int OPT = 0, int UNR = 1>
__device__ __forceinline__ void ysweep_strip(const GridDev& g, int col0, int j0, int strip_rows) {
  constexpr bool UM = MK == kMetricUnit, MP = MK == kMetricMapped;
  Ctl* ctl = g.ctl;
  if (!eta_valid(g)) return;
  const int cur = ctl->cur;
  const int xb = cur == 2 ? 0 : cur + 1;
  const int yb = cur == 0 ? 2 : cur - 1;
  const double dtod = ctl->dtod_y;
  const int mx = g.mx, my = g.my;
  const int i = col0 + threadIdx.x;
  const bool active = i <= mx;
  const int ic = active ? i : mx;  // inactive lanes shadow a valid column and store nothing
  const int j1 = min(j0 + strip_rows - 1, my);
  const long long P = g.pitch;
  const double* pre = buffer(g, cur);
  const double* xsw = buffer(g, xb);
  double* outp = buffer(g, yb);
  const double gam = (UM || MP) ? 1.0 : __ldg(g.colm + (ic + 1) * kColMetrics + 2);
  int bad = 0;
  double smax = 0.0;

  auto load = [&](int jj, YCell& c) {
    const double* src = (jj >= 1 && jj <= my) ? xsw : pre;
    const long long o = (long long)(jj + 1) * P + (ic + 1);
    c.q[0] = src[o];
    c.q[1] = src[o + g.plane];
    c.q[2] = src[o + 2 * g.plane];
    int cb = 0;
    c.F = cell_flux<1, OPT>(c.q[0], c.q[1], c.q[2], g.grav, &cb);
    if (jj <= my + 1) bad |= cb;  // getJakobi runs on rows -1 .. m_eta+1 in the eta sweep
    if constexpr (MP) {
      c.kap = __ldg(g.kap + o);
      c.lr = __ldg(g.lry + o);
    } else {
      c.kap = (SO && !UM) ? capacity(g.rowm, g.colm, ic, jj, g.area_scale) : 1.0;
      c.lr = gam;
    }
  };
  auto iface = [&](int k, const YCell& L, const YCell& R, Waves& W) -> double {
    if (k > my + 1) {
#pragma unroll
      for (int me = 0; me < 3; ++me) W.w1[me] = W.w2[me] = 0.0;
      return 0.0;
    }
    const double s2 = hll<OPT>(L.q, L.F, R.q, R.F, W);
    smax = fmax(smax, s2);
    return s2;
  };

  // prologue: cells j0-2 .. j0+1, interfaces j0-1 .. j0+1, correction flux at j0
  YCell cA, cB, cC;  // cells jj, jj+1, jj+2 of the window
  Waves W0, W1, W2;  // interfaces jj, jj+1, jj+2
  double s0, s1, s2w;
  double ft0[3] = {0.0, 0.0, 0.0}, ft1[3] = {0.0, 0.0, 0.0};
  {
    YCell cm2, cm1;
    Waves Wm;
    load(j0 - 2, cm2);
    load(j0 - 1, cm1);
    const double sm = iface(j0 - 1, cm2, cm1, Wm);
    (void)sm;
    load(j0, cA);
    s0 = iface(j0, cm1, cA, W0);
    load(j0 + 1, cB);
    s1 = iface(j0 + 1, cA, cB, W1);
    if constexpr (SO) y_corr_flux<LIM, SO, UM, OPT>(Wm, W0, W1, s0, true, dtod, cm1.kap, cA.kap, ft0);
  }
#pragma unroll UNR
  for (int jj = j0; jj <= j1; ++jj) {
    load(jj + 2, cC);
    s2w = iface(jj + 2, cB, cC, W2);
    if constexpr (SO) y_corr_flux<LIM, SO, UM, OPT>(W0, W1, W2, s1, jj + 1 <= my, dtod, cA.kap, cB.kap, ft1);
    const double kap = (SO || UM || MP) ? cA.kap : capacity(g.rowm, g.colm, ic, jj, g.area_scale);
    const double gl = MP ? cA.lr : gam, gr = MP ? cB.lr : gam;  // faces below and above the cell
    const double dtk = UM ? dtod : dtod / kap;
    const long long o = (long long)(jj + 1) * P + (ic + 1);
#pragma unroll
    for (int me = 0; me < 3; ++me) {
      const double ap = s0 * W0.w2[me];
      const double am = (-s1) * W1.w1[me];
      double q = UM ? cA.q[me] - dtk * (ap + am) : cA.q[me] - dtk * (gl * ap + gr * am);
      if constexpr (SO) q = q - dtk * (ft1[me] - ft0[me]);
      if (active) outp[o + me * g.plane] = q;
    }
    // slide the window
    cA = cB;
    cB = cC;
    W0 = W1;
    W1 = W2;
    s0 = s1;
    s1 = s2w;
#pragma unroll
    for (int me = 0; me < 3; ++me) ft0[me] = ft1[me];
  }
  // Carry the pre-step ghost cells into the new buffer: until update_rank_boundaries runs, the
  // reference's solution keeps the ghosts of the previous fill (main.f90:210 vs :246).
  if (active) {
    auto copy_cell = [&](int ci, int cj) {
      const long long o = (long long)(cj + 1) * P + (ci + 1);
#pragma unroll
      for (int me = 0; me < 3; ++me) outp[o + me * g.plane] = pre[o + me * g.plane];
    };
    if (j0 == 1) copy_cell(i, -1), copy_cell(i, 0);
    if (j1 == my) copy_cell(i, my + 1), copy_cell(i, my + 2);
    if (i == 1)
      for (int jj = j0; jj <= j1; ++jj) copy_cell(-1, jj), copy_cell(0, jj);
    if (i == mx)
      for (int jj = j0; jj <= j1; ++jj) copy_cell(mx + 1, jj), copy_cell(mx + 2, jj);
  }
  if (!active) smax = 0.0, bad = 0;
  smax = warp_max(smax);
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&ctl->smax_y, smax);
  if (bad) atomicOr(&ctl->status, bad);
}

// ------------------------------------------------------------------------------------------
// eta sweep in bands (the default shape at every grid size; the batch's eta items).  A CTA
// walks down a band of TX columns over rows j0 .. j1 in steps of L = NT/TX rows, running the xi
// sweep's four shared-memory phases along the columns: slot (r, c) = (row, column in the band),
// so a warp's loads are TX*8 contiguous bytes on each of 32/TX rows.  The last two cells, the last
// two interfaces and the last correction flux of a step stay in history slots (rows 0, 1) for the
// next step, so only the four rows in front of j0 are computed twice.  Bands start at column
// i = -1 + TX*k (a 32-byte sector boundary, the pitch being a multiple of 32 doubles); columns
// outside 1 .. m_xi are computed on a clamped column and written nowhere.
//
// PB (parity buffers): three CTA barriers per step (after phases A, B and C).  The cell states,
// capacities and face ratios, which phase D reads while faster threads already fill the next
// step's phase A, are kept per step parity; the next step's cells are staged (PF: cp.async,
// right after the barrier that ends this step's phase A) or loaded into the other parity.
// History rows move at two points: the phase-A arrays right after the phase-B barrier (nothing
// of this step reads their rows 0, 1 after it; the next phase A writes rows 2 and up only), the
// phase-B and C arrays after phase D in the warp that reads their rows 0, 1 (the next step
// writes them only after its phase-A barrier).  Without PB (less shared memory: the batch's
// items, whose kernel keeps a stack in L1) one copy of each array, every history row moved after
// phase D, and a fourth barrier closes the step.
//
// Semantics of ysweep_strip: rows 1 .. m_eta from the xi-swept buffer, the ghost rows from the
// pre-step buffer (main.f90:210 runs before the ghost fill at :246); getJakobi's status over rows
// -1 .. m_eta+1; waves of interfaces beyond m_eta+1 are zero and the interface m_eta+1 is
// unlimited; the pre-step ghost cells carried into the new buffer.  The first step of a CTA starts at s = j0-2 with empty history: its interface
// s and the correction fluxes and updates that would read the history are never used (updates
// start at row j0).  The caller checks the xi-sweep validity (eta_valid) and reduces smax and
// the status bits over the CTA.
// ------------------------------------------------------------------------------------------
template <int SLOTS, int NP, bool MP>
struct YBMapped {
  double slr[NP][SLOTS];  // mapped grids: length ratio of the eta face below the cell
};
template <int SLOTS, int NP>
struct YBMapped<SLOTS, NP, false> {};

// MP: mapped-grid metrics (the batch and uniform grids leave them out, for shared memory);
// PB: parity buffers.
template <int NT, int TX, bool MP = true, bool PB = true>
struct YBSmem : YBMapped<(NT / TX + 2) * TX, PB ? 2 : 1, MP> {
  static constexpr int L = NT / TX, SL = (L + 2) * TX, NP = PB ? 2 : 1;
  double sq[NP][3][SL], sk[NP][SL];  // cell states and capacities (by step parity with PB)
  double sf[3][SL], ss[SL];
  double sw1[3][SL], sw2[3][SL], ss2[SL];
  double sft[3][(L + 1) * TX];
  double red[NT / 32];
  bool sok[SL];
};

// PF: each thread stages its cell of the next step into shared memory (cp.async) while this
// step's phases B .. D run, so the global loads do not open the step.
template <int NT, int TX, int LIM, bool SO, int MK = kMetricTable, int OPT = 0, bool PF = false, bool PB = true>
__device__ __forceinline__ void ysweep_band(const GridDev& g, int i0, int j0, int j1,
                                            YBSmem<NT, TX, MK == kMetricMapped, PB>& S, double& smax_acc,
                                            int& bad_acc) {
  constexpr bool UM = MK == kMetricUnit, MP = MK == kMetricMapped;
  constexpr int L = NT / TX;
  static_assert(NT % 32 == 0 && TX <= 16 && L >= 4, "band shape: rows 0, 1 within warp 0");
  static_assert(PB || !PF, "staging fills the other parity");
  const Ctl* ctl = g.ctl;
  const int cur = ctl->cur;
  const int xb = cur == 2 ? 0 : cur + 1;
  const int yb = cur == 0 ? 2 : cur - 1;
  const double dtod = ctl->dtod_y;
  const int mx = g.mx, my = g.my;
  const long long P = g.pitch;
  const int t = threadIdx.x;
  const int cx = t % TX, r = t / TX;
  const int i = i0 + cx;
  const bool active = i >= 1 && i <= mx;
  const int ic = i < 1 ? 1 : (i > mx ? mx : i);
  const double* pre = buffer(g, cur);
  const double* xsw = buffer(g, xb);
  double* outp = buffer(g, yb);
  const double gam = (UM || MP) ? 1.0 : __ldg(g.colm + (ic + 1) * kColMetrics + 2);
  double smax = 0.0;
  int bad = 0;
  const int jlast = min(j1, my);
  const int sa = (r + 2) * TX + cx;  // this thread's phase-A and phase-B slot
  // cell j = s + r of this thread's column into its slot of parity p (rows past m_eta+2: nothing)
  auto stage = [&](int s_, int p_) {
    if constexpr (PF) {
      const int j = s_ + r;
      if (j <= my + 2) {
        const double* src = (j >= 1 && j <= my) ? xsw : pre;
        const long long o = (long long)(j + 1) * P + (ic + 1);
        cp_async8(&S.sq[p_][0][sa], src + o);
        cp_async8(&S.sq[p_][1][sa], src + o + g.plane);
        cp_async8(&S.sq[p_][2][sa], src + o + 2 * g.plane);
      }
      cp_async_commit();
    }
  };
  if constexpr (PF) stage(j0 - 2, 0);

  int p = 0;  // step parity (0 throughout without PB)
  for (int s = j0 - 2; s - 2 <= jlast; s += L, p = PB ? p ^ 1 : 0) {
    if constexpr (PF) cp_async_wait<0>();
    {  // phase A: cell j = s + r into slot (r+2)TX + c
      const int j = s + r;
      if (j <= my + 2) {
        const long long o = (long long)(j + 1) * P + (ic + 1);
        double h, hu, hv;
        if constexpr (PF) {
          h = S.sq[p][0][sa], hu = S.sq[p][1][sa], hv = S.sq[p][2][sa];
        } else {
          const double* src = (j >= 1 && j <= my) ? xsw : pre;
          h = src[o], hu = src[o + g.plane], hv = src[o + 2 * g.plane];
          S.sq[p][0][sa] = h; S.sq[p][1][sa] = hu; S.sq[p][2][sa] = hv;
        }
        int cb = 0;
        const CellFlux F = cell_flux<1, OPT>(h, hu, hv, g.grav, &cb);
        if (j <= my + 1 && active) bad |= cb;
        S.sf[0][sa] = F.f0; S.sf[1][sa] = F.f1; S.sf[2][sa] = F.f2;
        S.ss[sa] = F.s;
        if constexpr ((OPT & kOptFastDiv) != 0) S.sok[sa] = F.ok;
        if constexpr (MP) {
          S.sk[p][sa] = __ldg(g.kap + o);
          S.slr[p][sa] = __ldg(g.lry + o);
        } else if constexpr (!UM) {
          S.sk[p][sa] = capacity(g.rowm, g.colm, ic, j, g.area_scale);
        }
      }
    }
    __syncthreads();
    if constexpr (PF) {  // the next step's cells into the other parity, read last by the previous phase D
      if (s + L - 2 <= jlast) stage(s + L, p ^ 1);
    }
    {  // phase B: interface k = s + r (cells k-1, k) into slot (r+2)TX + c
      const int k = s + r;
      const int sl = sa, sm = sl - TX;
      Waves W;
      double s2 = 0.0;
      if (k <= my + 1 && k >= j0 - 1) {
        const double qL[3] = {S.sq[p][0][sm], S.sq[p][1][sm], S.sq[p][2][sm]};
        const double qR[3] = {S.sq[p][0][sl], S.sq[p][1][sl], S.sq[p][2][sl]};
        CellFlux FL = {S.sf[0][sm], S.sf[1][sm], S.sf[2][sm], S.ss[sm]};
        CellFlux FR = {S.sf[0][sl], S.sf[1][sl], S.sf[2][sl], S.ss[sl]};
        if constexpr ((OPT & kOptFastDiv) != 0) FL.ok = S.sok[sm], FR.ok = S.sok[sl];
        s2 = hll<OPT>(qL, FL, qR, FR, W);
        if (active) smax = fmax(smax, s2);
      } else {
#pragma unroll
        for (int me = 0; me < 3; ++me) W.w1[me] = W.w2[me] = 0.0;
      }
#pragma unroll
      for (int me = 0; me < 3; ++me) {
        S.sw1[me][sl] = W.w1[me];
        S.sw2[me][sl] = W.w2[me];
      }
      S.ss2[sl] = s2;
    }
    __syncthreads();
    // history of the phase-A arrays: rows L, L+1 -> 0, 1 (states and metrics: of parity p ^ 1)
    auto history_a = [&](int pn) {
      if (r < 2) {
        const int from = (L + r) * TX + cx, to = r * TX + cx;
#pragma unroll
        for (int me = 0; me < 3; ++me) {
          S.sq[pn][me][to] = S.sq[p][me][from];
          S.sf[me][to] = S.sf[me][from];
        }
        S.ss[to] = S.ss[from];
        if constexpr ((OPT & kOptFastDiv) != 0) S.sok[to] = S.sok[from];
        if constexpr (MP) S.slr[pn][to] = S.slr[p][from];
        if constexpr (MP || !UM) S.sk[pn][to] = S.sk[p][from];
      }
    };
    if constexpr (PB) history_a(p ^ 1);
    if constexpr (SO) {  // phase C: correction flux at interface k = s - 1 + r into ft slot (r+1)TX + c
      const int k = s - 1 + r;
      const int w = (r + 1) * TX + cx;  // interface k's slot; k-1 at w - TX, k+1 at w + TX
      double ft[3] = {0.0, 0.0, 0.0};
      if (k <= my + 1) {
        const double s2 = S.ss2[w];
        const double cf = UM ? corr_coef_unit(s2, dtod) : corr_coef(s2, dtod, S.sk[p][w - TX], S.sk[p][w]);
        if (cf != 0.0) {
          const double w1[3] = {S.sw1[0][w], S.sw1[1][w], S.sw1[2][w]};
          const double w2[3] = {S.sw2[0][w], S.sw2[1][w], S.sw2[2][w]};
          double a[3], b[3];
          if (LIM != 0 && k <= my) {
            const double w1m[3] = {S.sw1[0][w - TX], S.sw1[1][w - TX], S.sw1[2][w - TX]};
            const double w1p[3] = {S.sw1[0][w + TX], S.sw1[1][w + TX], S.sw1[2][w + TX]};
            const double w2m[3] = {S.sw2[0][w - TX], S.sw2[1][w - TX], S.sw2[2][w - TX]};
            const double w2p[3] = {S.sw2[0][w + TX], S.sw2[1][w + TX], S.sw2[2][w + TX]};
            limit_wave<LIM, OPT>(w1m, w1, w1p, false, a);
            limit_wave<LIM, OPT>(w2m, w2, w2p, s2 > 0.0, b);
          } else {
#pragma unroll
            for (int me = 0; me < 3; ++me) {
              a[me] = w1[me];
              b[me] = w2[me];
            }
          }
#pragma unroll
          for (int me = 0; me < 3; ++me) ft[me] = cf * a[me] + cf * b[me];
        }
      }
#pragma unroll
      for (int me = 0; me < 3; ++me) S.sft[me][(r + 1) * TX + cx] = ft[me];
    }
    __syncthreads();
    {  // phase D: update of cell j = s - 2 + r (cell and interface slot rTX + c)
      const int j = s - 2 + r;
      if (active && j >= j0 && j <= jlast) {
        const int c = r * TX + cx;
        double gl = gam, gr = gam;  // faces below and above the cell
        if constexpr (MP) gl = S.slr[p][c], gr = S.slr[p][c + TX];
        const double dtk = UM ? dtod : dtod / S.sk[p][c];
        const double sp = S.ss2[c];
        const double sm = -S.ss2[c + TX];
        const long long o = (long long)(j + 1) * P + (i + 1);
#pragma unroll
        for (int me = 0; me < 3; ++me) {
          const double ap = sp * S.sw2[me][c];
          const double am = sm * S.sw1[me][c + TX];
          double q = UM ? S.sq[p][me][c] - dtk * (ap + am) : S.sq[p][me][c] - dtk * (gl * ap + gr * am);
          if constexpr (SO) q = q - dtk * (S.sft[me][c + TX] - S.sft[me][c]);
          outp[o + me * g.plane] = q;
        }
        if (i == 1 || i == mx) {  // the pre-step ghost columns beside the edge columns
          const long long ob = (long long)(j + 1) * P;
          const int g0 = i == 1 ? -1 : mx + 1;
#pragma unroll
          for (int gcol = g0; gcol <= g0 + 1; ++gcol)
#pragma unroll
            for (int me = 0; me < 3; ++me) outp[ob + gcol + 1 + me * g.plane] = pre[ob + gcol + 1 + me * g.plane];
        }
      }
    }
    // History of the interfaces (rows L, L+1 -> 0, 1) and the correction flux (L -> 0), and
    // without PB of the phase-A arrays too.  Phase D reads rows 0 and 1 of those arrays only in
    // threads r = 0, 1 (row 2 and up belong to later rows), which share warp 0 with the copying
    // threads (32/TX >= 2 rows per warp): a warp barrier orders them.  The rows copied from were
    // final before phase D.  With PB the next step writes these arrays only after its phase-A
    // barrier, which this warp reaches after the copy: no closing CTA barrier.
    if (threadIdx.x < 32) __syncwarp();
    if constexpr (!PB) history_a(0);
    if (r < 2) {
      const int from = (L + r) * TX + cx, to = r * TX + cx;
#pragma unroll
      for (int me = 0; me < 3; ++me) {
        S.sw1[me][to] = S.sw1[me][from];
        S.sw2[me][to] = S.sw2[me][from];
      }
      S.ss2[to] = S.ss2[from];
      if (r == 0) {
#pragma unroll
        for (int me = 0; me < 3; ++me) S.sft[me][cx] = S.sft[me][L * TX + cx];
      }
    }
    if constexpr (!PB) __syncthreads();
  }
  if constexpr (PB) __syncthreads();  // the last step's phase D has read S before the caller reuses it
  if (active && r < 4) {  // the pre-step ghost rows of the band's columns
    auto copy_cell = [&](int ci, int cj) {
      const long long o = (long long)(cj + 1) * P + (ci + 1);
#pragma unroll
      for (int me = 0; me < 3; ++me) outp[o + me * g.plane] = pre[o + me * g.plane];
    };
    if (r < 2 && j0 == 1) copy_cell(i, -1 + r);
    if (r >= 2 && jlast == my) copy_cell(i, my + r - 1);
  }
  smax_acc = fmax(smax_acc, smax);
  bad_acc |= bad;
}

}  // namespace pcl
