// kernels_mixed.cu -- the precision form: both sweeps of one attempted step fused into one
// row-streaming kernel, with the flux, HLL and limiter arithmetic in FP32 and the state update,
// the wave-speed reduction and the time control in FP64.
//
// Work item: a strip of TXI = 124 columns x a segment of TY rows.  The CTA streams the rows
// j0-2 .. j1+2 of its strip (plus two halo columns each side) through a four-slot shared-memory
// ring filled by bulk copies (cp.async.bulk, completion on an mbarrier), two rows ahead.  For each
// row: the xi sweep of that row runs in shared memory (per-cell flux data, HLL per interface,
// limited correction flux, update); thread t keeps the x-swept FP64 value of its own column
// i0+t in registers and advances its eta-sweep register window (interfaces j-2 .. j) by one
// row, writing the finished cell j-2.  The x-swept state never leaves the SM, so an accepted
// step moves 24 B in and 24 B out per cell instead of twice that.
//
// Precision: differences of the state (dq) are taken in FP64 and rounded once to FP32, and the
// flux jump is written in terms of them, so its rounding error scales with the jump and not with
// the state:  for the reference's flux J(q).q = (n, n^2/h + g h^2, n t/h) (normal momentum n,
// transverse t),
//   d(n^2/h) = u_R dn + n_L du,  du = (dn h_L - n_L dh) / (h_L h_R),  d(g h^2) = g (h_L+h_R) dh,
//   d(n t/h) = u_R dt + t_L du.
// The capacity and length ratios of the uniform grid round to exactly 1 in FP32 and drop out.
// Each cell's increment is accumulated in FP32 and applied to the FP64 state as dt/delta * sum.
#include <cuda_runtime.h>

#include "../../include/paraclaws_b200.h"
#include "pcl_mixed.h"
#include "pcl_sm100.cuh"
#include "pcl_types.h"

namespace pcl {
namespace mixed {

constexpr int NT = 128;      // threads per CTA = slots of a streamed row
constexpr int TXI = NT - 4;  // interior columns of a strip
constexpr int RING = 4;      // row slots
constexpr int AHEAD = 2;     // rows in flight ahead of the one being processed
constexpr float kEps = 1e-10f;

struct CellM {
  float h, n, t, ih, un, s;
};

__device__ __forceinline__ CellM cell_m(double h, double n, double t, float g) {
  CellM c;
  c.h = (float)h;
  c.n = (float)n;
  c.t = (float)t;
  c.ih = __frcp_rn(c.h);
  c.un = c.n * c.ih;
  const float gh = g * c.h;
  c.s = fabsf(c.un) + gh * rsqrtf(gh);
  return c;
}

__device__ __forceinline__ int cell_bad(double h, double n, double t) {
  int b = 0;
  if (isnan(h) || isnan(n) || isnan(t) || h == 0.0) b |= kStatusNaN;
  if (h < 0.0) b |= kStatusNegDepth;
  return b;
}

struct WF {
  float w1[3], w2[3];
};

// HLL in jump form; components in (h, n, t) order.  Returns s2 (0 for a degenerate interface).
__device__ __forceinline__ float hll_m(const CellM& L, const CellM& R, const float dq[3], float g, WF& W) {
  const float s2 = fmaxf(L.s, R.s);
  if (!(s2 > kEps)) {
#pragma unroll
    for (int k = 0; k < 3; ++k) W.w1[k] = W.w2[k] = 0.f;
    return 0.f;
  }
  const float du = (dq[1] * L.h - L.n * dq[0]) * L.ih * R.ih;
  const float df[3] = {dq[1], R.un * dq[1] + L.n * du + g * (L.h + R.h) * dq[0], R.un * dq[2] + L.t * du};
  const float ql[3] = {L.h, L.n, L.t};
  const float rden = __frcp_rn((kEps - s2) - s2);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    W.w1[k] = (df[k] - s2 * dq[k] - kEps * ql[k]) * rden;
    W.w2[k] = dq[k] - W.w1[k];
  }
  return s2;
}

template <int LIM>
__device__ __forceinline__ float phi_f(float r) {
  if (LIM == 1) return fmaxf(0.f, fminf(1.f, r));
  if (LIM == 2) return fmaxf(fmaxf(0.f, fminf(1.f, 2.f * r)), fminf(2.f, r));
  if (LIM == 3) return __fdividef(r + fabsf(r), 1.f + fabsf(r));
  return fmaxf(0.f, fminf(fminf(0.5f * (1.f + r), 2.f), 2.f * r));
}

__device__ __forceinline__ float dot3f(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

template <int LIM>
__device__ __forceinline__ void limit_f(const float wm[3], const float w[3], const float wp[3], bool pos, float o[3]) {
  const float wn2 = dot3f(w, w);
  float ph = 1.f;
  if (wn2 > kEps) ph = phi_f<LIM>(__fdividef(pos ? dot3f(wm, w) : dot3f(w, wp), wn2));
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = ph * w[k];
}

// correction flux of one interface from its wave and its neighbours' (same family)
template <int LIM, bool SO>
__device__ __forceinline__ void corr_f(const WF& Wm, const WF& W, const WF& Wp, float s2, bool limited, float dtodf,
                                       float ft[3]) {
  if (!SO || s2 == 0.f) {
    ft[0] = ft[1] = ft[2] = 0.f;
    return;
  }
  const float cf = (0.5f * s2) * (1.f - s2 * dtodf);
  float a[3], b[3];
  if (LIM != 0 && limited) {
    limit_f<LIM>(Wm.w1, W.w1, Wp.w1, false, a);
    limit_f<LIM>(Wm.w2, W.w2, Wp.w2, true, b);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      a[k] = W.w1[k];
      b[k] = W.w2[k];
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) ft[k] = cf * (a[k] + b[k]);
}

struct __align__(16) Smem {
  double ring[RING][3][NT];   // streamed rows (h, hu, hv), cells i0-2 .. i0+TXI+1
  float cell[6][NT];          // xi sweep per cell: h, n, t, 1/h, u, s
  float w1[3][NT], w2[3][NT];
  float s2[NT];
  float ft[3][NT];
  float red[2][NT / 32];
  uint64_t bar[RING];
};

template <int LIM, bool SO>
__global__ void __launch_bounds__(NT) fused_mixed_kernel(GridDev g, int TY, int nstrips) {
  __shared__ Smem S;
  Ctl* ctl = g.ctl;
  if (ctl->done) return;
  const int t = threadIdx.x;
  const int cur = ctl->cur;
  const int ob = cur == 0 ? 2 : cur - 1;  // the buffer a full step writes
  const double dtodx = ctl->dtod_x, dtody = ctl->dtod_y;
  const float dtodxf = (float)dtodx, dtodyf = (float)dtody;
  const float gf = (float)g.grav;
  const int mx = g.mx, my = g.my;
  const long long P = g.pitch, PL = g.plane;
  const int strip = blockIdx.x % nstrips, seg = blockIdx.x / nstrips;
  const int i0 = 1 + strip * TXI;
  const int j0 = 1 + seg * TY;
  const int j1 = min(j0 + TY - 1, my);
  const int c0 = i0 - 1;  // storage column of cell i0-2 (even: 16-byte aligned)
  const int ncopy = min(NT, (int)(P - c0));
  const double* in = buffer(g, cur);
  double* outp = buffer(g, ob);
  const int jfirst = j0 - 2, nrows = (j1 + 2) - jfirst + 1;
  const int icol = i0 + t;                    // this thread's column in the eta sweep
  const bool ycol = t < TXI && icol <= mx;

  if (t == 0) {
    for (int s = 0; s < RING; ++s) mbar_init(&S.bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](int row, int slot) {
    if (t == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&S.bar[slot], 3u * ncopy * 8u);
      const double* src = in + (long long)(row + 1) * P + c0;
      for (int p = 0; p < 3; ++p) bulk_g2s(&S.ring[slot][p][0], src + p * PL, ncopy * 8u, &S.bar[slot]);
    }
  };
  for (int k = 0; k < AHEAD && k < nrows; ++k) issue(jfirst + k, k);

  int bad = 0;
  float smx = 0.f, smy = 0.f;
  // eta-sweep window (own column).  Entering step k (newest row jr): qb, qc = x-swept FP64 state
  // (h, hu, hv) of rows jr-2, jr-1; cprev = FP32 cell data of row jr-1; (Wa, Wb, Wc) = waves of
  // interfaces jr-3, jr-2, jr-1 (shifted to jr-2, jr-1, jr once interface jr is solved);
  // fta = correction flux at interface jr-2.
  double qb[3] = {0, 0, 0}, qc[3] = {0, 0, 0};
  CellM cprev{};
  WF Wa{}, Wb{}, Wc{};
  float sa = 0.f, sb = 0.f, sc = 0.f;
  float fta[3] = {0.f, 0.f, 0.f};
  bool timed_out = false;
  int issued = min(AHEAD, nrows), consumed = 0;

  for (int k = 0; k < nrows; ++k) {
    const int jr = jfirst + k;
    const int slot = k & (RING - 1);
    if (k + AHEAD < nrows) {
      issue(jr + AHEAD, (k + AHEAD) & (RING - 1));
      issued++;
    }
    const bool ok = mbar_wait_bounded(&S.bar[slot], (uint32_t)((k / RING) & 1));
    if (__syncthreads_or(!ok)) {
      timed_out = true;
      break;
    }
    consumed++;
    const double* r0 = S.ring[slot][0];
    const double* r1 = S.ring[slot][1];
    const double* r2 = S.ring[slot][2];
    double xs[3] = {r0[t + 2 < NT ? t + 2 : NT - 1], r1[t + 2 < NT ? t + 2 : NT - 1], r2[t + 2 < NT ? t + 2 : NT - 1]};

    if (jr >= 1 && jr <= my) {
      // ---- xi sweep of row jr ----
      {  // phase A: cell i0-2+t
        const int c = i0 - 2 + t;
        if (c <= mx + 2) {
          const double h = r0[t], hu = r1[t], hv = r2[t];
          if (c <= mx + 1) bad |= cell_bad(h, hu, hv);
          const CellM m = cell_m(h, hu, hv, gf);
          S.cell[0][t] = m.h; S.cell[1][t] = m.n; S.cell[2][t] = m.t;
          S.cell[3][t] = m.ih; S.cell[4][t] = m.un; S.cell[5][t] = m.s;
        }
      }
      __syncthreads();
      if (t < NT - 1) {  // phase B: interface i0-1+t between slots t and t+1
        const int kf = i0 - 1 + t;
        WF W;
        float s2 = 0.f;
        if (kf <= mx + 1) {
          const CellM L = {S.cell[0][t], S.cell[1][t], S.cell[2][t], S.cell[3][t], S.cell[4][t], S.cell[5][t]};
          const CellM R = {S.cell[0][t + 1], S.cell[1][t + 1], S.cell[2][t + 1], S.cell[3][t + 1], S.cell[4][t + 1],
                           S.cell[5][t + 1]};
          const float dq[3] = {(float)(r0[t + 1] - r0[t]), (float)(r1[t + 1] - r1[t]), (float)(r2[t + 1] - r2[t])};
          s2 = hll_m(L, R, dq, gf, W);
          smx = fmaxf(smx, s2);
        } else {
#pragma unroll
          for (int q = 0; q < 3; ++q) W.w1[q] = W.w2[q] = 0.f;
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          S.w1[q][t] = W.w1[q];
          S.w2[q][t] = W.w2[q];
        }
        S.s2[t] = s2;
      }
      __syncthreads();
      if (SO && t < NT - 3) {  // phase C: correction flux at interface i0+t (slot t+1)
        const int kf = i0 + t;
        float ft[3] = {0.f, 0.f, 0.f};
        if (kf <= mx + 1) {
          const int s = t + 1;
          const WF Wm = {{S.w1[0][s - 1], S.w1[1][s - 1], S.w1[2][s - 1]}, {S.w2[0][s - 1], S.w2[1][s - 1], S.w2[2][s - 1]}};
          const WF W0 = {{S.w1[0][s], S.w1[1][s], S.w1[2][s]}, {S.w2[0][s], S.w2[1][s], S.w2[2][s]}};
          const WF Wp = {{S.w1[0][s + 1], S.w1[1][s + 1], S.w1[2][s + 1]}, {S.w2[0][s + 1], S.w2[1][s + 1], S.w2[2][s + 1]}};
          corr_f<LIM, SO>(Wm, W0, Wp, S.s2[s], kf <= mx, dtodxf, ft);
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) S.ft[q][t] = ft[q];
      }
      if (SO) __syncthreads();
      if (t < TXI && i0 + t <= mx) {  // phase D: x-swept value of this thread's column
        const float sp = S.s2[t + 1], sm = -S.s2[t + 2];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          float fs = sp * S.w2[q][t + 1] + sm * S.w1[q][t + 2];
          if (SO) fs += S.ft[q][t + 1] - S.ft[q][t];
          xs[q] = xs[q] - dtodx * (double)fs;
        }
      }
    }

    // ---- eta sweep: advance this column's window by row jr (components (h, n = hv, t = hu)) ----
    {
      if (ycol && jr <= my + 1) bad |= cell_bad(xs[0], xs[2], xs[1]);
      const CellM cn = cell_m(xs[0], xs[2], xs[1], gf);
      if (k >= 1) {
        WF Wn;
        float sn = 0.f;
        if (jr <= my + 1) {
          const float dq[3] = {(float)(xs[0] - qc[0]), (float)(xs[2] - qc[2]), (float)(xs[1] - qc[1])};
          sn = hll_m(cprev, cn, dq, gf, Wn);
          smy = fmaxf(smy, sn);
        } else {
#pragma unroll
          for (int q = 0; q < 3; ++q) Wn.w1[q] = Wn.w2[q] = 0.f;
        }
        Wa = Wb; sa = sb;
        Wb = Wc; sb = sc;
        Wc = Wn; sc = sn;
      }
      float ftb[3] = {0.f, 0.f, 0.f};
      if (k >= 3) corr_f<LIM, SO>(Wa, Wb, Wc, sb, jr - 1 <= my, dtodyf, ftb);  // interface jr-1
      if (k >= 4 && jr - 2 <= j1 && ycol) {                                   // update cell jr-2
        // A+ at jr-2 is s(jr-2) W2(jr-2), A- at jr-1 is -s(jr-1) W1(jr-1); the window holds
        // interfaces (jr-2, jr-1, jr) as (Wa, Wb, Wc) after the shift above.
        float fs[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) fs[q] = sa * Wa.w2[q] + (-sb) * Wb.w1[q] + (ftb[q] - fta[q]);
        const long long o = (long long)(jr - 2 + 1) * P + (icol + 1);
        outp[o] = qb[0] - dtody * (double)fs[0];
        outp[o + PL] = qb[1] - dtody * (double)fs[2];
        outp[o + 2 * PL] = qb[2] - dtody * (double)fs[1];
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        fta[q] = ftb[q];
        qb[q] = qc[q];
        qc[q] = xs[q];
      }
      cprev = cn;
    }
    __syncthreads();  // slot k&3 is refilled two rows from now
  }

  if (timed_out && t == 0) {
    // drain the copies this CTA still has in flight before its shared memory goes away
    for (int k = consumed; k < issued; ++k) mbar_wait_bounded(&S.bar[k & (RING - 1)], (uint32_t)((k / RING) & 1));
  }
  // eta-sweep speeds count only real columns
  if (!ycol) smy = 0.f;
  // block max of the two wave speeds, one atomic each
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    smx = fmaxf(smx, __shfl_xor_sync(0xffffffffu, smx, o));
    smy = fmaxf(smy, __shfl_xor_sync(0xffffffffu, smy, o));
  }
  if ((t & 31) == 0) {
    S.red[0][t >> 5] = smx;
    S.red[1][t >> 5] = smy;
  }
  __syncthreads();
  if (t == 0) {
    float a = 0.f, b = 0.f;
    for (int w = 0; w < NT / 32; ++w) {
      a = fmaxf(a, S.red[0][w]);
      b = fmaxf(b, S.red[1][w]);
    }
    if (a > 0.f) atomicMax(&ctl->smax_x, (unsigned long long)__double_as_longlong((double)a));
    if (b > 0.f) atomicMax(&ctl->smax_y, (unsigned long long)__double_as_longlong((double)b));
    if (timed_out) atomicOr(&ctl->status, kStatusTimeout);
  }
  if (bad) atomicOr(&ctl->status, bad);
}

struct Workspace {
  int ty;
};

}  // namespace mixed

int mixed_create(const GridDev&, cudaStream_t, void** ws) {
  auto* w = new mixed::Workspace();
  w->ty = 64;
  *ws = w;
  return PCL_OK;
}

void mixed_free(void* ws) { delete static_cast<mixed::Workspace*>(ws); }

void mixed_set_tile_rows(void* ws, int ty) {
  if (ws && ty >= 4) static_cast<mixed::Workspace*>(ws)->ty = ty;
}

namespace {
template <int LIM, bool SO>
void launch_t(const GridDev& g, int ty, cudaStream_t st) {
  const int nstrips = (g.mx + mixed::TXI - 1) / mixed::TXI;
  const int nseg = (g.my + ty - 1) / ty;
  mixed::fused_mixed_kernel<LIM, SO><<<nstrips * nseg, mixed::NT, 0, st>>>(g, ty, nstrips);
}
}  // namespace

void launch_sweeps_mixed(const GridDev& g, void* ws, cudaStream_t st) {
  const int ty = ws ? static_cast<mixed::Workspace*>(ws)->ty : 64;
  if (!g.second_order) return launch_t<0, false>(g, ty, st);
  switch (g.limiter) {
    case 1: return launch_t<1, true>(g, ty, st);
    case 2: return launch_t<2, true>(g, ty, st);
    case 3: return launch_t<3, true>(g, ty, st);
    case 4: return launch_t<4, true>(g, ty, st);
    default: return launch_t<0, true>(g, ty, st);
  }
}

}  // namespace pcl
