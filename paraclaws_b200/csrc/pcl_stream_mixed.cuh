// pcl_stream_mixed.cuh -- the precision form: both sweeps of one attempted step fused into one
// row-streaming kernel, with the flux, HLL and limiter arithmetic in FP32 and the state update,
// the wave-speed reduction and the time control in FP64.
//
// Work item: a strip of TXI = 124 columns x a segment of TY rows.  The CTA streams the rows
// j0-2 .. j1+2 of its strip (plus two halo columns each side) through a five-slot shared-memory
// ring filled by bulk copies (cp.async.bulk, completion on an mbarrier), three rows ahead.  For each
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
// Multiply-adds are written out (__fmaf_rn, fma) and the translation units that include this
// header are built with --fmad=false, so the arithmetic cannot change with the kernel it is
// inlined into: a grid gives the same bits alone and inside a batch.
#pragma once
#include <cuda_runtime.h>

#include "pcl_sm100.cuh"
#include "pcl_types.h"

namespace pcl {
namespace mixed {

constexpr int NT = 128;      // threads per CTA = slots of a streamed row
constexpr int TXI = NT - 4;  // interior columns of a strip
// Row slots: the copy issued at the start of row k refills the slot of row k+AHEAD-RING = k-2,
// which every thread finished before it passed row k-1's copy-wait vote, so a row needs no
// barrier after its last read of the ring.
constexpr int RING = 5;
constexpr int AHEAD = 3;     // rows in flight ahead of the one being processed
static_assert(RING >= AHEAD + 2, "the refilled slot must be two rows old");
constexpr float kEps = 1e-10f;

struct CellM {
  float h, n, t, ih, un, s;
};

__device__ __forceinline__ CellM cell_m(double h, double n, double t, float g) {
  CellM c;
  c.h = (float)h;
  c.n = (float)n;
  c.t = (float)t;
  c.ih = __fdividef(1.f, c.h);
  c.un = c.n * c.ih;
  const float gh = g * c.h;
  c.s = __fmaf_rn(gh, rsqrtf(gh), fabsf(c.un));
  return c;
}

// getJakobi's NaN trap and dgeev's complex-eigenvalue abort as status bits: a cell is bad when
// its wave speed is not finite (h <= 0, or h or n NaN or infinite) or its transverse momentum
// is NaN.  Only the rare bad path looks at h again to tell the two apart.
__device__ __forceinline__ int bad_m(const CellM& m, double h) {
  if ((m.s < __int_as_float(0x7f800000)) && !isnan(m.t)) return 0;
  return h < 0.0 ? kStatusNegDepth : kStatusNaN;
}

struct WF {
  float w1[3], w2[3];
};

// HLL in jump form; components in (h, n, t) order.  Returns s2 (0 for a degenerate interface,
// whose waves are 0).  Branch-free: the degenerate case is selected after the arithmetic.
__device__ __forceinline__ float hll_m(const CellM& L, const CellM& R, const float dq[3], float g, WF& W) {
  const float s2 = fmaxf(L.s, R.s);
  const bool live = s2 > kEps;
  const float du = __fmaf_rn(dq[1], L.h, -(L.n * dq[0])) * (L.ih * R.ih);
  const float gsum = g * (L.h + R.h);
  const float df[3] = {dq[1], __fmaf_rn(R.un, dq[1], __fmaf_rn(L.n, du, gsum * dq[0])),
                       __fmaf_rn(R.un, dq[2], L.t * du)};
  const float ql[3] = {L.h, L.n, L.t};
  const float rden = __fdividef(1.f, (kEps - s2) - s2);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float w1 = __fmaf_rn(-kEps, ql[k], __fmaf_rn(-s2, dq[k], df[k])) * rden;
    W.w1[k] = live ? w1 : 0.f;
    W.w2[k] = live ? dq[k] - w1 : 0.f;
  }
  return live ? s2 : 0.f;
}

template <int LIM>
__device__ __forceinline__ float phi_f(float r) {
  if (LIM == 1) return fmaxf(0.f, fminf(1.f, r));
  if (LIM == 2) return fmaxf(fmaxf(0.f, fminf(1.f, 2.f * r)), fminf(2.f, r));
  if (LIM == 3) return __fdividef(r + fabsf(r), 1.f + fabsf(r));
  return fmaxf(0.f, fminf(fminf(0.5f * (1.f + r), 2.f), 2.f * r));
}

__device__ __forceinline__ float dot3f(const float a[3], const float b[3]) {
  return __fmaf_rn(a[0], b[0], __fmaf_rn(a[1], b[1], a[2] * b[2]));
}

// wave limited by phi(theta), theta = upstream / |W|^2; phi = 1 where |W|^2 <= eps or where the
// interface is not limited (1 * w == w).  Branch-free.
template <int LIM>
__device__ __forceinline__ void limit_f(const float wm[3], const float w[3], const float wp[3], bool pos, bool limited,
                                        float o[3]) {
  const float wn2 = dot3f(w, w);
  const float r = __fdividef(pos ? dot3f(wm, w) : dot3f(w, wp), wn2);
  const float ph = limited && wn2 > kEps ? phi_f<LIM>(r) : 1.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) o[k] = ph * w[k];
}

// correction flux of one interface from its wave and its neighbours' (same family)
template <int LIM, bool SO>
__device__ __forceinline__ void corr_f(const WF& Wm, const WF& W, const WF& Wp, float s2, bool limited, float dtodf,
                                       float ft[3]) {
  if (!SO) {
    ft[0] = ft[1] = ft[2] = 0.f;
    return;
  }
  const float cf = (0.5f * s2) * __fmaf_rn(-s2, dtodf, 1.f);
  float a[3], b[3];
  if (LIM != 0) {
    limit_f<LIM>(Wm.w1, W.w1, Wp.w1, false, limited, a);
    limit_f<LIM>(Wm.w2, W.w2, Wp.w2, true, limited, b);
  } else {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      a[k] = W.w1[k];
      b[k] = W.w2[k];
    }
  }
  const bool live = s2 != 0.f;
#pragma unroll
  for (int k = 0; k < 3; ++k) ft[k] = live ? cf * (a[k] + b[k]) : 0.f;
}

// Shared memory of one CTA.  Per-slot data of the xi sweep is packed in float4 so a neighbour's
// record is two or three 128-bit loads; a thread's own slot stays in registers between phases.
struct __align__(16) Smem {
  double ring[RING][3][NT];   // streamed rows (h, hu, hv), cells i0-2 .. i0+TXI+1
  float4 cA[NT];              // cell: h, n, t, 1/h
  float2 cB[NT];              // cell: u, s
  float4 wA[NT];              // interface: W1 (3), s2
  float4 wB[NT];              // interface: W2 (3), -
  float4 ft[NT];              // correction flux (3), -
  float red[2][NT / 32];
  uint64_t bar[RING];
};

__device__ __forceinline__ WF load_wf(const Smem& S, int s) {
  const float4 a = S.wA[s], b = S.wB[s];
  return WF{{a.x, a.y, a.z}, {b.x, b.y, b.z}};
}

// One work item (strip x row segment) of one grid.  `rows` counts the rows this CTA has
// streamed through the ring before this item (slot and mbarrier parity continue across items);
// the item's wave-speed maxima and status bits go to g.ctl before it returns.  All threads of
// the CTA call it together.  Returns false if a bulk copy did not arrive in time.
// UNROLL unrolls the row loop (the single-grid kernel: 2, letting the eta window shift by
// renaming; the batched kernel: 1, which keeps its register count at four CTAs per SM).  It
// changes no arithmetic.
// G is GridDev or any descriptor with its fields ctl, grav, mx, my, pitch, plane, state and
// bufstride (the batch keeps a compact one in constant memory).
// INJ (a separate build, used only by the test of the timeout path): the bulk copy of row
// inj_row is never issued, so the wait for it runs out after `probes` probes; the copies that
// were issued are drained as after any timeout.
template <int LIM, bool SO, int UNROLL = 1, bool INJ = false, class G>
__device__ __forceinline__ bool mixed_item(const G& g, int strip, int seg, int TY, Smem& S, unsigned& rows,
                                           int inj_row = -1, unsigned probes = 1u << 22) {
  Ctl* ctl = g.ctl;
  const int t = threadIdx.x;
  const int cur = ctl->cur;
  const int ob = cur == 0 ? 2 : cur - 1;  // the buffer a full step writes
  const double dtodx = ctl->dtod_x, dtody = ctl->dtod_y;
  const float dtodxf = (float)dtodx, dtodyf = (float)dtody;
  const float gf = (float)g.grav;
  const int mx = g.mx, my = g.my;
  const long long P = g.pitch, PL = g.plane;
  const int i0 = 1 + strip * TXI;
  const int j0 = 1 + seg * TY;
  const int j1 = min(j0 + TY - 1, my);
  const int c0 = i0 - 1;  // storage column of cell i0-2 (even: 16-byte aligned)
  const int ncopy = min(NT, (int)(P - c0));
  const double* in = g.state + (long long)cur * g.bufstride;
  const int jfirst = j0 - 2, nrows = (j1 + 2) - jfirst + 1;
  const int icol = i0 + t;                    // this thread's column in the eta sweep
  const bool ycol = t < TXI && icol <= mx;
  double* outp = g.state + (long long)ob * g.bufstride + (icol + 1);

  const unsigned base = rows;
  auto issue = [&](int row, int slot) {
    if (INJ && row == inj_row) return;
    if (t == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&S.bar[slot], 3u * ncopy * 8u);
      const double* src = in + (long long)(row + 1) * P + c0;
      for (int p = 0; p < 3; ++p) bulk_g2s(&S.ring[slot][p][0], src + p * PL, ncopy * 8u, &S.bar[slot]);
    }
  };
  for (int k = 0; k < AHEAD && k < nrows; ++k) issue(jfirst + k, (base + k) % RING);

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
  const int tc = t + 2 < NT ? t + 2 : NT - 1;  // ring slot of this thread's column
  const int t1 = t + 1 < NT ? t + 1 : NT - 1;  // next slot (clamped)
  const int t2 = tc;                           // slot after next (clamped)

#pragma unroll UNROLL
  for (int k = 0; k < nrows; ++k) {
    const int jr = jfirst + k;
    const unsigned kk = base + k;
    const int slot = kk % RING;
    if (k + AHEAD < nrows) {
      issue(jr + AHEAD, (kk + AHEAD) % RING);
      issued++;
    }
    const bool ok = INJ ? mbar_wait_bounded(&S.bar[slot], (kk / RING) & 1u, probes)
                        : mbar_wait_bounded(&S.bar[slot], (kk / RING) & 1u);
    if (__syncthreads_or(!ok)) {
      timed_out = true;
      break;
    }
    consumed++;
    const double* r0 = S.ring[slot][0];
    const double* r1 = S.ring[slot][1];
    const double* r2 = S.ring[slot][2];
    double xs[3] = {r0[tc], r1[tc], r2[tc]};

    if (jr >= 1 && jr <= my) {
      // ---- xi sweep of row jr ----
      // Branch-free phases: every thread computes, results outside the valid range are
      // selected to zero (or never read); slot indices past the row are clamped.
      const int c = i0 - 2 + t;  // phase A: this thread's cell (slot t)
      const double qm[3] = {r0[t], r1[t], r2[t]};
      const CellM me = cell_m(qm[0], qm[1], qm[2], gf);
      if (c <= mx + 1) bad |= bad_m(me, qm[0]);
      S.cA[t] = make_float4(me.h, me.n, me.t, me.ih);
      S.cB[t] = make_float2(me.un, me.s);
      __syncthreads();
      WF Wme;  // phase B: interface i0-1+t between slots t (own) and t+1
      float s2me;
      {
        const float4 a = S.cA[t1];
        const float2 b = S.cB[t1];
        const CellM R = {a.x, a.y, a.z, a.w, b.x, b.y};
        const float dq[3] = {(float)(r0[t1] - qm[0]), (float)(r1[t1] - qm[1]), (float)(r2[t1] - qm[2])};
        s2me = hll_m(me, R, dq, gf, Wme);
        const bool v = t < NT - 1 && i0 - 1 + t <= mx + 1;
        s2me = v ? s2me : 0.f;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          Wme.w1[q] = v ? Wme.w1[q] : 0.f;
          Wme.w2[q] = v ? Wme.w2[q] : 0.f;
        }
        smx = fmaxf(smx, s2me);
        S.wA[t] = make_float4(Wme.w1[0], Wme.w1[1], Wme.w1[2], s2me);
        S.wB[t] = make_float4(Wme.w2[0], Wme.w2[1], Wme.w2[2], 0.f);
      }
      __syncthreads();
      float ftme[3] = {0.f, 0.f, 0.f};  // phase C: correction flux at interface i0+t (slot t+1)
      if (SO) {
        const int kf = i0 + t;
        const WF W0 = load_wf(S, t1);
        const WF Wp = load_wf(S, t2);
        corr_f<LIM, SO>(Wme, W0, Wp, S.wA[t1].w, kf <= mx, dtodxf, ftme);
        const bool v = t < NT - 3 && kf <= mx + 1;
#pragma unroll
        for (int q = 0; q < 3; ++q) ftme[q] = v ? ftme[q] : 0.f;
        S.ft[t] = make_float4(ftme[0], ftme[1], ftme[2], 0.f);
        __syncthreads();
      }
      {  // phase D: x-swept value of this thread's column (used only where ycol)
        const float4 a = S.wA[t1], b = S.wB[t1], d = S.wA[t2];
        const float sp = a.w, sm = -d.w;
        float fs[3] = {__fmaf_rn(sp, b.x, sm * d.x), __fmaf_rn(sp, b.y, sm * d.y), __fmaf_rn(sp, b.z, sm * d.z)};
        if (SO) {
          const float4 f1 = S.ft[t1];
          fs[0] += f1.x - ftme[0];
          fs[1] += f1.y - ftme[1];
          fs[2] += f1.z - ftme[2];
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) xs[q] = fma(-dtodx, (double)fs[q], xs[q]);
      }
    }

    // ---- eta sweep: advance this column's window by row jr (components (h, n = hv, t = hu)) ----
    {
      const CellM cn = cell_m(xs[0], xs[2], xs[1], gf);
      if (ycol && jr <= my + 1) bad |= bad_m(cn, xs[0]);
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
        for (int q = 0; q < 3; ++q) fs[q] = __fmaf_rn(sa, Wa.w2[q], __fmaf_rn(-sb, Wb.w1[q], ftb[q] - fta[q]));
        double* o = outp + (long long)(jr - 1) * P;
        o[0] = fma(-dtody, (double)fs[0], qb[0]);
        o[PL] = fma(-dtody, (double)fs[2], qb[1]);
        o[2 * PL] = fma(-dtody, (double)fs[1], qb[2]);
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        fta[q] = ftb[q];
        qb[q] = qc[q];
        qc[q] = xs[q];
      }
      cprev = cn;
    }
  }

  if (timed_out && t == 0) {
    // drain the copies this CTA still has in flight before its shared memory goes away
    for (int k = consumed; k < issued; ++k) {
      if (INJ)
        mbar_wait_bounded(&S.bar[(base + k) % RING], ((base + k) / RING) & 1u, probes);
      else
        mbar_wait_bounded(&S.bar[(base + k) % RING], ((base + k) / RING) & 1u);
    }
  }
  rows = base + issued;
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
  __syncthreads();  // S.red is reused by the next item
  return !timed_out;
}


__device__ __forceinline__ void init_ring(Smem& S) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < RING; ++s) mbar_init(&S.bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
}

}  // namespace mixed
}  // namespace pcl
