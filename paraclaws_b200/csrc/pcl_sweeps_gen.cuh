// pcl_sweeps_gen.cuh -- the FP64 sweeps for any equation module (pcl_equations.h) with N
// equations: the reference's step written for num_equations = N (solver/MOD_solve.f90:23-293,
// solver/SMOD_approximate_Riemann_solvers.f90:15-102 with arrays sized by num_equations at
// :34-44, solver/MOD_flux_correction.f90:17-187 looping over num_equations).  Same structure and
// boundary semantics as the specialised shallow-water sweeps (pcl_sweeps_fp64.cuh): the xi sweep
// in four shared-memory phases per row segment, the eta sweep as a register window per column,
// buffer rotation, the last interface of a row or column unlimited, ghosts filled once per step.
// The cell flux is J(q).q from the module in BLAS dgemv order and the wave speed max |eigenvalue|
// of both cells.  Capacities come from the row/column tables of the uniform grid (on grids
// whose capacities are all 1 this gives the same bits as leaving them out).  Include only from
// translation units built with --fmad=false.
#pragma once
#include <cuda_runtime.h>

#include "pcl_fp64.cuh"
#include "pcl_sweeps_fp64.cuh"

namespace pcl {
namespace gen {

template <int N>
struct Cell {
  double f[N];
  double s;
};

template <int N>
struct WavesN {
  double w1[N], w2[N];
};

// Flux J(q).q and wave-speed bound of a cell for module `module` (N equations), sweep DIR.
template <int N, int DIR>
__device__ __forceinline__ Cell<N> cell_flux(int module, const double q[N], const double* prm, int* bad) {
  Cell<N> c;
  if (pcl_eq_num_equations(module) != N) {  // the host pairs modules with contexts of their size
    *bad |= kStatusNaN;
#pragma unroll
    for (int r = 0; r < N; ++r) c.f[r] = 0.0;
    c.s = 0.0;
    return c;
  }
  double J[N * N];
  if (pcl_eq_jacobian(module, DIR + 1, q, prm, J)) *bad |= kStatusNaN;
#pragma unroll
  for (int r = 0; r < N; ++r) c.f[r] = 0.0;
#pragma unroll
  for (int col = 0; col < N; ++col) {  // dgemv 'N': y = 0; y += x(col) * A(:, col)
    const double temp = q[col];
#pragma unroll
    for (int r = 0; r < N; ++r) c.f[r] = c.f[r] + temp * J[col * N + r];
  }
  double lam[N];
  if (pcl_eq_eigenvalues(module, DIR + 1, q, prm, lam)) *bad |= kStatusNegDepth;
  double s = fabs(lam[0]);
#pragma unroll
  for (int k = 1; k < N; ++k) s = fabs(lam[k]) > s ? fabs(lam[k]) : s;
  c.s = s;
  return c;
}

// HLL two-wave solve at one interface, N components (pcl_fp64.cuh: hll).
template <int N>
__device__ __forceinline__ double hll(const double qL[N], const Cell<N>& fL, const double qR[N], const Cell<N>& fR,
                                      WavesN<N>& W) {
  const double smax = fmax(fL.s, fR.s);
  const double s1 = -smax;
  if (fabs(s1) > kUdPrecision && fabs(smax) > kUdPrecision) {
    const double den = (kUdPrecision + s1) - smax;
#pragma unroll
    for (int me = 0; me < N; ++me) {
      const double qs = div_neg_den(((fR.f[me] - fL.f[me]) - smax * qR[me]) + s1 * qL[me], den);
      W.w1[me] = qs - qL[me];
      W.w2[me] = qR[me] - qs;
    }
    return smax;
  }
#pragma unroll
  for (int me = 0; me < N; ++me) W.w1[me] = W.w2[me] = 0.0;
  return 0.0;
}

template <int N>
__device__ __forceinline__ double dot(const double a[N], const double b[N]) {
  double s = a[0] * b[0];
#pragma unroll
  for (int k = 1; k < N; ++k) s = s + a[k] * b[k];
  return s;
}

// limited wave of one family (pcl_fp64.cuh: limit_wave), N components
template <int N, int LIM>
__device__ __forceinline__ void limit_wave(const double wm[N], const double w[N], const double wp[N], bool lambda_pos,
                                           double out[N]) {
  const double wn2 = dot<N>(w, w);
  if (fabs(wn2) <= kUdPrecision) {
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = w[k];
    return;
  }
  const double up = lambda_pos ? dot<N>(wm, w) : dot<N>(w, wp);
  const double phi = limiter_phi<LIM>(div_pos_den(up, wn2));
#pragma unroll
  for (int k = 0; k < N; ++k) out[k] = phi * w[k];
}

template <int N, int LIM>
__device__ __forceinline__ void corr_flux(const WavesN<N>& Wm, const WavesN<N>& W, const WavesN<N>& Wp, double s2,
                                          bool limited, double dtod, double kl, double kr, double ft[N]) {
  const double cf = corr_coef(s2, dtod, kl, kr);
  if (cf == 0.0) {
#pragma unroll
    for (int k = 0; k < N; ++k) ft[k] = 0.0;
    return;
  }
  double a[N], b[N];
  if (LIM != 0 && limited) {
    limit_wave<N, LIM>(Wm.w1, W.w1, Wp.w1, false, a);
    limit_wave<N, LIM>(Wm.w2, W.w2, Wp.w2, s2 > 0.0, b);
  } else {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      a[k] = W.w1[k];
      b[k] = W.w2[k];
    }
  }
#pragma unroll
  for (int k = 0; k < N; ++k) ft[k] = cf * a[k] + cf * b[k];
}

// ------------------------------------------------------------------------------------------
// xi sweep of one row segment of NT-4 cells (pcl_sweeps_fp64.cuh: xsweep_segment)
// ------------------------------------------------------------------------------------------
template <int NT, int N>
struct XSmem {
  double sq[N][NT], sf[N][NT], ss[NT], sk[NT];
  double sw1[N][NT], sw2[N][NT], ss2[NT], sft[N][NT];
  double red[NT / 32];
};

template <int NT, int N, int LIM, bool SO>
__device__ __forceinline__ void xsweep_segment(const GridDev& g, int j, int i0, XSmem<NT, N>& S, double& smax_acc,
                                               int& bad_acc) {
  const Ctl* ctl = g.ctl;
  constexpr int L = NT - 4;
  const int cur = ctl->cur, out = cur == 2 ? 0 : cur + 1;
  const double dtod = ctl->dtod_x;
  const int t = threadIdx.x;
  const int mx = g.mx;
  const long long row = (long long)(j + 1) * g.pitch;
  const double* q0 = buffer(g, cur) + row;

  int bad = 0;
  {  // phase A: per-cell flux, wave-speed bound and capacity
    const int c = i0 - 2 + t;
    if (c <= mx + 2) {
      double q[N];
#pragma unroll
      for (int me = 0; me < N; ++me) q[me] = q0[me * g.plane + c + 1];
      int cb = 0;
      const Cell<N> F = cell_flux<N, 0>(g.eq, q, g.eqp, &cb);
      if (c <= mx + 1) bad |= cb;  // getJakobi runs on cells -1 .. m_xi+1 in the xi sweep
#pragma unroll
      for (int me = 0; me < N; ++me) {
        S.sq[me][t] = q[me];
        S.sf[me][t] = F.f[me];
      }
      S.ss[t] = F.s;
      S.sk[t] = capacity(g.rowm, g.colm, c, j, g.area_scale);
    }
  }
  __syncthreads();

  double smax = 0.0;
  if (t < NT - 1) {  // phase B: HLL at interface k = i0-1+t (slots t, t+1)
    const int k = i0 - 1 + t;
    WavesN<N> W;
    double s2 = 0.0;
    if (k <= mx + 1) {
      double qL[N], qR[N];
      Cell<N> FL, FR;
#pragma unroll
      for (int me = 0; me < N; ++me) {
        qL[me] = S.sq[me][t];
        qR[me] = S.sq[me][t + 1];
        FL.f[me] = S.sf[me][t];
        FR.f[me] = S.sf[me][t + 1];
      }
      FL.s = S.ss[t];
      FR.s = S.ss[t + 1];
      s2 = hll<N>(qL, FL, qR, FR, W);
      smax = s2;
    } else {
#pragma unroll
      for (int me = 0; me < N; ++me) W.w1[me] = W.w2[me] = 0.0;
    }
#pragma unroll
    for (int me = 0; me < N; ++me) {
      S.sw1[me][t] = W.w1[me];
      S.sw2[me][t] = W.w2[me];
    }
    S.ss2[t] = s2;
  }
  smax_acc = fmax(smax_acc, smax);
  bad_acc |= bad;
  __syncthreads();

  if constexpr (SO) {  // phase C: correction flux at interface k = i0+t (slot t+1)
    if (t < NT - 3) {
      const int k = i0 + t;
      double ft[N];
#pragma unroll
      for (int me = 0; me < N; ++me) ft[me] = 0.0;
      if (k <= mx + 1) {
        const int s = t + 1;
        WavesN<N> Wm, W0, Wp;
#pragma unroll
        for (int me = 0; me < N; ++me) {
          Wm.w1[me] = S.sw1[me][s - 1], Wm.w2[me] = S.sw2[me][s - 1];
          W0.w1[me] = S.sw1[me][s], W0.w2[me] = S.sw2[me][s];
          Wp.w1[me] = S.sw1[me][s + 1], Wp.w2[me] = S.sw2[me][s + 1];
        }
        corr_flux<N, LIM>(Wm, W0, Wp, S.ss2[s], k <= mx, dtod, S.sk[t + 1], S.sk[t + 2], ft);
      }
#pragma unroll
      for (int me = 0; me < N; ++me) S.sft[me][t] = ft[me];
    }
    __syncthreads();
  }

  if (t < L) {  // phase D: update of cell i = i0+t (MOD_solve.f90:207-221 and :268-278)
    const int i = i0 + t;
    if (i <= mx) {
      const int c = t + 2;
      const double gam = __ldg(g.rowm + (j + 1) * kRowMetrics + 2);
      const double dtk = dtod / S.sk[c];
      const double sp = S.ss2[t + 1];   // A+ at interface i:   s2 * W2
      const double sm = -S.ss2[t + 2];  // A- at interface i+1: s1 * W1
      double* o0 = buffer(g, out) + row;
#pragma unroll
      for (int me = 0; me < N; ++me) {
        const double ap = sp * S.sw2[me][t + 1];
        const double am = sm * S.sw1[me][t + 2];
        double q = S.sq[me][c] - dtk * (gam * ap + gam * am);
        if constexpr (SO) q = q - dtk * (S.sft[me][t + 1] - S.sft[me][t]);
        o0[me * g.plane + i + 1] = q;
      }
    }
  }
}

template <int NT, int N>
__device__ __forceinline__ void xsweep_finish(const GridDev& g, double smax, int bad, XSmem<NT, N>& S) {
  block_max_to<NT>(const_cast<unsigned long long*>(&g.ctl->smax_x), smax, S.red);
  if (bad) atomicOr(&g.ctl->status, bad);
}

// ------------------------------------------------------------------------------------------
// eta sweep of one column over a strip of rows (pcl_sweeps_fp64.cuh: ysweep_strip)
// ------------------------------------------------------------------------------------------
template <int N>
struct YCell {
  double q[N];
  Cell<N> F;
  double kap;
};

template <int N, int LIM, bool SO>
__device__ __forceinline__ void ysweep_strip(const GridDev& g, int col0, int j0, int strip_rows) {
  Ctl* ctl = g.ctl;
  {  // xi-sweep validity (MOD_solve.f90:107-120) from the reduction word
    const double sx = __longlong_as_double((long long)__ldcg(&ctl->smax_x));
    const double cflx = sx * ctl->dt / g.dxi;
    const double cfl = fmax(ctl->CFL, cflx);
    if (!(ctl->CFL_target / cfl >= ctl->shrink)) return;
  }
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
  const double gam = __ldg(g.colm + (ic + 1) * kColMetrics + 2);
  int bad = 0;
  double smax = 0.0;

  auto load = [&](int jj, YCell<N>& c) {
    const double* src = (jj >= 1 && jj <= my) ? xsw : pre;
    const long long o = (long long)(jj + 1) * P + (ic + 1);
#pragma unroll
    for (int me = 0; me < N; ++me) c.q[me] = src[o + me * g.plane];
    int cb = 0;
    c.F = cell_flux<N, 1>(g.eq, c.q, g.eqp, &cb);
    if (jj <= my + 1) bad |= cb;  // getJakobi runs on rows -1 .. m_eta+1 in the eta sweep
    c.kap = capacity(g.rowm, g.colm, ic, jj, g.area_scale);
  };
  auto iface = [&](int k, const YCell<N>& L, const YCell<N>& R, WavesN<N>& W) -> double {
    if (k > my + 1) {
#pragma unroll
      for (int me = 0; me < N; ++me) W.w1[me] = W.w2[me] = 0.0;
      return 0.0;
    }
    const double s2 = hll<N>(L.q, L.F, R.q, R.F, W);
    smax = fmax(smax, s2);
    return s2;
  };

  YCell<N> cA, cB, cC;      // cells jj, jj+1, jj+2 of the window
  WavesN<N> W0, W1, W2;     // interfaces jj, jj+1, jj+2
  double s0, s1, s2w;
  double ft0[N], ft1[N];
#pragma unroll
  for (int me = 0; me < N; ++me) ft0[me] = ft1[me] = 0.0;
  {  // prologue: cells j0-2 .. j0+1, interfaces j0-1 .. j0+1, correction flux at j0
    YCell<N> cm2, cm1;
    WavesN<N> Wm;
    load(j0 - 2, cm2);
    load(j0 - 1, cm1);
    iface(j0 - 1, cm2, cm1, Wm);
    load(j0, cA);
    s0 = iface(j0, cm1, cA, W0);
    load(j0 + 1, cB);
    s1 = iface(j0 + 1, cA, cB, W1);
    if constexpr (SO) corr_flux<N, LIM>(Wm, W0, W1, s0, true, dtod, cm1.kap, cA.kap, ft0);
  }
  for (int jj = j0; jj <= j1; ++jj) {
    load(jj + 2, cC);
    s2w = iface(jj + 2, cB, cC, W2);
    if constexpr (SO) corr_flux<N, LIM>(W0, W1, W2, s1, jj + 1 <= my, dtod, cA.kap, cB.kap, ft1);
    const double dtk = dtod / cA.kap;
    const long long o = (long long)(jj + 1) * P + (ic + 1);
#pragma unroll
    for (int me = 0; me < N; ++me) {
      const double ap = s0 * W0.w2[me];
      const double am = (-s1) * W1.w1[me];
      double q = cA.q[me] - dtk * (gam * ap + gam * am);
      if constexpr (SO) q = q - dtk * (ft1[me] - ft0[me]);
      if (active) outp[o + me * g.plane] = q;
    }
    cA = cB;
    cB = cC;
    W0 = W1;
    W1 = W2;
    s0 = s1;
    s1 = s2w;
#pragma unroll
    for (int me = 0; me < N; ++me) ft0[me] = ft1[me];
  }
  // the pre-step ghost cells carried into the new buffer (main.f90:210 vs :246)
  if (active) {
    auto copy_cell = [&](int ci, int cj) {
      const long long o = (long long)(cj + 1) * P + (ci + 1);
#pragma unroll
      for (int me = 0; me < N; ++me) outp[o + me * g.plane] = pre[o + me * g.plane];
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
// eta sweep in bands (pcl_sweeps_fp64.cuh: ysweep_band), N components: a CTA walks its chunk of
// rows down a band of TX columns in steps of L = NT/TX rows, the four phases of the xi sweep
// running along the columns, the last two cells, two interfaces and one correction flux of a
// step carried into the next in history slots, and each thread's cell of the next step staged
// by cp.async while the phases of this one run.  Slot (r, c) = row r of the step (+2 history
// rows), column c of the band.  Same semantics as ysweep_strip; the caller checks the xi-sweep
// validity and reduces smax and the status bits over the CTA.
// ------------------------------------------------------------------------------------------
template <int NT, int TX, int N>
struct YBSmem {
  static constexpr int L = NT / TX;
  static constexpr int CS = (L + 2) * TX;
  double sq[N][CS], sf[N][CS], ss[CS], sk[CS];
  double sw1[N][CS], sw2[N][CS], ss2[CS];
  double sft[N][(L + 1) * TX];
  double stg[2][N][NT];
  double red[NT / 32];
};

template <int NT, int TX, int N, int LIM, bool SO>
__device__ __forceinline__ void ysweep_band(const GridDev& g, int i0, int j0, int j1, YBSmem<NT, TX, N>& S,
                                            double& smax_acc, int& bad_acc) {
  constexpr int L = NT / TX;
  static_assert(NT % 32 == 0 && TX <= 16 && L >= 4, "band shape: rows 0, 1 within warp 0");
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
  const double gam = __ldg(g.colm + (ic + 1) * kColMetrics + 2);
  double smax = 0.0;
  int bad = 0;
  const int jlast = min(j1, my);
  auto stage = [&](int s_, int b_) {  // cell s_ + r of this thread's column (none past m_eta+2)
    const int j = s_ + r;
    if (j <= my + 2) {
      const double* src = (j >= 1 && j <= my) ? xsw : pre;
      const long long o = (long long)(j + 1) * P + (ic + 1);
#pragma unroll
      for (int me = 0; me < N; ++me) cp_async8(&S.stg[b_][me][t], src + o + me * g.plane);
    }
    cp_async_commit();
  };
  stage(j0 - 2, 0);

  int sb = 0;
  for (int s = j0 - 2; s - 2 <= jlast; s += L, sb ^= 1) {
    if (s + L - 2 <= jlast) {
      stage(s + L, sb ^ 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    {  // phase A: cell j = s + r into slot (r+2)TX + c
      const int j = s + r;
      const int sl = (r + 2) * TX + cx;
      if (j <= my + 2) {
        double q[N];
#pragma unroll
        for (int me = 0; me < N; ++me) q[me] = S.stg[sb][me][t];
        int cb = 0;
        const Cell<N> F = cell_flux<N, 1>(g.eq, q, g.eqp, &cb);
        if (j <= my + 1 && active) bad |= cb;  // getJakobi runs on rows -1 .. m_eta+1
#pragma unroll
        for (int me = 0; me < N; ++me) {
          S.sq[me][sl] = q[me];
          S.sf[me][sl] = F.f[me];
        }
        S.ss[sl] = F.s;
        S.sk[sl] = capacity(g.rowm, g.colm, ic, j, g.area_scale);
      }
    }
    __syncthreads();
    {  // phase B: interface k = s + r (cells k-1, k) into slot (r+2)TX + c
      const int k = s + r;
      const int sl = (r + 2) * TX + cx, sm = sl - TX;
      WavesN<N> W;
      double s2 = 0.0;
      if (k <= my + 1 && k >= j0 - 1) {
        double qL[N], qR[N];
        Cell<N> FL, FR;
#pragma unroll
        for (int me = 0; me < N; ++me) {
          qL[me] = S.sq[me][sm];
          qR[me] = S.sq[me][sl];
          FL.f[me] = S.sf[me][sm];
          FR.f[me] = S.sf[me][sl];
        }
        FL.s = S.ss[sm];
        FR.s = S.ss[sl];
        s2 = hll<N>(qL, FL, qR, FR, W);
        if (active) smax = fmax(smax, s2);
      } else {
#pragma unroll
        for (int me = 0; me < N; ++me) W.w1[me] = W.w2[me] = 0.0;
      }
#pragma unroll
      for (int me = 0; me < N; ++me) {
        S.sw1[me][sl] = W.w1[me];
        S.sw2[me][sl] = W.w2[me];
      }
      S.ss2[sl] = s2;
    }
    __syncthreads();
    if constexpr (SO) {  // phase C: correction flux at interface k = s - 1 + r into flux slot (r+1)TX + c
      const int k = s - 1 + r;
      const int w = (r + 1) * TX + cx;  // interface k; k-1 at w - TX, k+1 at w + TX
      double ft[N];
#pragma unroll
      for (int me = 0; me < N; ++me) ft[me] = 0.0;
      if (k <= my + 1) {
        WavesN<N> Wm, W, Wp;
#pragma unroll
        for (int me = 0; me < N; ++me) {
          Wm.w1[me] = S.sw1[me][w - TX], Wm.w2[me] = S.sw2[me][w - TX];
          W.w1[me] = S.sw1[me][w], W.w2[me] = S.sw2[me][w];
          Wp.w1[me] = S.sw1[me][w + TX], Wp.w2[me] = S.sw2[me][w + TX];
        }
        // cells k-1 and k sit in the slots of interfaces k-1 and k
        corr_flux<N, LIM>(Wm, W, Wp, S.ss2[w], k <= my, dtod, S.sk[w - TX], S.sk[w], ft);
      }
#pragma unroll
      for (int me = 0; me < N; ++me) S.sft[me][(r + 1) * TX + cx] = ft[me];
      __syncthreads();
    }
    {  // phase D: update of cell j = s - 2 + r (cell and interface slot rTX + c)
      const int j = s - 2 + r;
      if (active && j >= j0 && j <= jlast) {
        const int c = r * TX + cx;
        const double dtk = dtod / S.sk[c];
        const double sp = S.ss2[c];
        const double sm = -S.ss2[c + TX];
        const long long o = (long long)(j + 1) * P + (i + 1);
#pragma unroll
        for (int me = 0; me < N; ++me) {
          const double ap = sp * S.sw2[me][c];
          const double am = sm * S.sw1[me][c + TX];
          double q = S.sq[me][c] - dtk * (gam * ap + gam * am);
          if constexpr (SO) q = q - dtk * (S.sft[me][c + TX] - S.sft[me][c]);
          outp[o + me * g.plane] = q;
        }
        if (i == 1 || i == mx) {  // the pre-step ghost columns beside the edge columns
          const long long ob = (long long)(j + 1) * P;
          const int g0 = i == 1 ? -1 : mx + 1;
#pragma unroll
          for (int gcol = g0; gcol <= g0 + 1; ++gcol)
#pragma unroll
            for (int me = 0; me < N; ++me) outp[ob + gcol + 1 + me * g.plane] = pre[ob + gcol + 1 + me * g.plane];
        }
      }
    }
    // History: rows L, L+1 -> 0, 1 (cells, interfaces) and flux row L -> 0.  Only threads of
    // rows 0 and 1 read those rows in phase D, and they share warp 0 with the copying threads.
    if (threadIdx.x < 32) __syncwarp();
    if (r < 2) {
      const int from = (L + r) * TX + cx, to = r * TX + cx;
#pragma unroll
      for (int me = 0; me < N; ++me) {
        S.sq[me][to] = S.sq[me][from];
        S.sf[me][to] = S.sf[me][from];
        S.sw1[me][to] = S.sw1[me][from];
        S.sw2[me][to] = S.sw2[me][from];
      }
      S.ss[to] = S.ss[from];
      S.sk[to] = S.sk[from];
      S.ss2[to] = S.ss2[from];
      if (r == 0) {
#pragma unroll
        for (int me = 0; me < N; ++me) S.sft[me][cx] = S.sft[me][L * TX + cx];
      }
    }
    __syncthreads();
  }
  if (active && r < 4) {  // the pre-step ghost rows of the band's columns
    auto copy_cell = [&](int cj) {
      const long long o = (long long)(cj + 1) * P + (i + 1);
#pragma unroll
      for (int me = 0; me < N; ++me) outp[o + me * g.plane] = pre[o + me * g.plane];
    };
    if (r < 2 && j0 == 1) copy_cell(-1 + r);
    if (r >= 2 && jlast == my) copy_cell(my + r - 1);
  }
  smax_acc = fmax(smax_acc, smax);
  bad_acc |= bad;
}


}  // namespace gen
}  // namespace pcl
