// pcl_fp64.cuh -- FP64 arithmetic of the wave-propagation step, bit-compatible with the
// reference's operation order.  Every translation unit that includes this header is compiled
// with --fmad=false so no multiply-add is contracted (the reference's rounding points are kept).
//
// Sweep direction DIR: 0 = xi sweep (normal momentum hu), 1 = eta sweep (normal momentum hv).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "pcl_equations.h"
#include "pcl_types.h"

namespace pcl {

// Flux Jacobian of the shallow-water equation module and its product with q
// (examples/2D_dam_break/cartesian/SMOD_jakobian.f90:44-53; utility/SMOD_matrix_operations.f90:22
// through BLAS dgemv 'N', which accumulates y = ((0 + q1*J(:,1)) + q2*J(:,2)) + q3*J(:,3)).
// Non-constant Jacobian entries (both sweeps share them):
//   jn = -(n*n)/(h*h) + g*h,  d2 = (2n)/h,  jt = -(hu*hv)/(h*h),  d4 = hv/h,  d5 = hu/h
// Flux components in (h, hu, hv) order:
//   xi : (hu, h*jn + hu*d2, (h*jt + hu*d4) + hv*d5)
//   eta: (hv, (h*jt + hu*d4) + hv*d5, h*jn + hv*d2)
// Wave speed bound of the cell: the eigenvalues of J are u-c, u, u+c with u = n/h and
// c = sqrt(g*h), whose largest magnitude is fl(|u| + c) in round-to-nearest
// (solver/SMOD_approximate_Riemann_solvers.f90:186-190 takes maxval of |eig| over both cells).
struct CellFlux {
  double f0, f1, f2, s;
  bool ok;  // h, hu, hv inside the range of the shared-reciprocal quotients (kOptFastDiv)
};

// IEEE division with the zero-numerator case answered without dividing.  CUDA's correctly
// rounded double division leaves its fast path for a zero (or tiny) numerator, and a warp pays
// that path when any lane takes it; quiescent cells (zero momentum) make such numerators
// common.  For a = +-0 the quotient is an exact signed zero: a / b = a for b > 0 (+inf
// included) and -a for b < 0.  Every other case divides, so the result is the same bits as
// a / b for all inputs (b = 0 or NaN still divides and gives NaN).  The numerator select is
// inline PTX so that the optimiser cannot fold it back into the division.
__device__ __forceinline__ double numerator_or_one(double a, bool use_one) {
  double r;
  asm("{\n\t.reg .pred p;\n\tsetp.ne.s32 p, %2, 0;\n\tselp.f64 %0, 0d3FF0000000000000, %1, p;\n\t}"
      : "=d"(r)
      : "d"(a), "r"((int)use_one));
  return r;
}
__device__ __forceinline__ double div_pos_den(double a, double b) {  // quotient for b > 0
  const bool z = a == 0.0 && b > 0.0;
  const double q = numerator_or_one(a, z) / b;
  return z ? a : q;
}
__device__ __forceinline__ double div_neg_den(double a, double b) {  // quotient for b < 0
  const bool z = a == 0.0 && b < 0.0;
  const double q = numerator_or_one(a, z) / b;
  return z ? -a : q;
}

// ---- correctly rounded quotients that share a denominator ----
// Markstein's correction step (P. W. Markstein, "Computation of elementary functions on the IBM
// RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990): when y = RN(1/b) and q is
// within one ulp of a/b, the remainder r = a - b*q is exactly representable (one FMA gives it)
// and RN(q + r*y) = RN(a/b).  q0 = RN(a*y) can be up to 1.5 ulp off, so one correction first
// brings it within one ulp and a second gives the correctly rounded quotient: the same bits as
// IEEE division, in one multiply and four FMAs per quotient after one reciprocal
// (__drcp_rn, correctly rounded) per denominator.  The remainders are exact and nothing
// underflows or overflows while a, b and a/b lie in [2^-960, 2^960] in magnitude; a = 0 takes
// q0 = a*y, the exactly signed zero.  Callers establish the range once per cell (mag_ok) and
// use IEEE division for cells outside it.
struct Den {
  double b, y;
};
__device__ __forceinline__ Den den_of(double b) { return Den{b, __drcp_rn(b)}; }
__device__ __forceinline__ double quot(double a, const Den& d) {
  const double q0 = __dmul_rn(a, d.y);
  const double q1 = __fma_rn(__fma_rn(-q0, d.b, a), d.y, q0);
  const double q2 = __fma_rn(__fma_rn(-q1, d.b, a), d.y, q1);
  return a == 0.0 ? q0 : q2;
}
// |x| is 0 or in [2^-64, 2^64) (biased exponent 959 .. 1086)
__device__ __forceinline__ bool mag_ok(double x) {
  const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7ffu;
  return e - 959u <= 127u || x == 0.0;
}
// x > 0 and in [2^-64, 2^64): the sign bit sits above the exponent, so one compare does both
__device__ __forceinline__ bool pos_ok(double x) { return ((unsigned)__double2hiint(x) >> 20) - 959u <= 127u; }

// Sweep-kernel options (template bit mask, results identical for every value):
//   kOptFastDiv  cell flux and HLL quotients from shared reciprocals (Markstein, above) for
//                cells whose h, hu, hv pass pos_ok/mag_ok, with g in [2^-20, 2^20] (the host
//                picks the build).  Every quotient of the flux and of the HLL solve then stays
//                inside the method's range: a non-zero sum of two doubles is at least 2^-53
//                times the smaller one, which bounds every non-zero flux below by 2^-426 and
//                every non-zero HLL numerator by 2^-585, with |den| in [2^-34, 2^130], so all
//                quotients lie in [2^-716, 2^356] and their remainders stay normal.
//   kOptLimSat   the limiter ratio theta = up/|W|^2 is only divided out where the limiter
//                function does not saturate (see limit_wave)
enum : int { kOptFastDiv = 1, kOptLimSat = 2 };

template <int DIR, int OPT = 0>
__device__ __forceinline__ CellFlux cell_flux(double h, double hu, double hv, double g, int* bad) {
  const double n = DIR == 0 ? hu : hv;
  const double hh = h * h;
  double d1, d3, d4, d5, d2;
  bool fast = false;
  if constexpr ((OPT & kOptFastDiv) != 0) fast = pos_ok(h) && mag_ok(hu) && mag_ok(hv);
  if (fast) {
    // h, |hu|, |hv| in [2^-64, 2^64) (or momenta 0): n/h is 0 or normal, so (2n)/h = 2*(n/h)
    const Den rh = den_of(h), rhh = den_of(hh);
    d1 = quot(n * n, rhh);
    d3 = quot(hu * hv, rhh);
    d4 = quot(hv, rh);
    d5 = quot(hu, rh);
    d2 = 2.0 * (DIR == 0 ? d5 : d4);
  } else {
    d1 = div_pos_den(n * n, hh);
    d3 = div_pos_den(hu * hv, hh);
    d4 = div_pos_den(hv, h);
    d5 = div_pos_den(hu, h);
    const double u = DIR == 0 ? d5 : d4;
    // (2n)/h == 2*(n/h) exactly unless n/h is subnormal (scaling by 2 commutes with rounding);
    // a branch, so the rare division is not evaluated for every cell
    if (fabs(u) >= 0x1p-1000)
      d2 = 2.0 * u;
    else
      d2 = div_pos_den(2.0 * n, h);
  }
  const double un = DIR == 0 ? d5 : d4;
  const double gh = g * h;
  const double jn = -d1 + gh;
  const double jt = -d3;
  CellFlux c;
  c.f0 = n;
  const double fnorm = h * jn + n * d2;
  const double ftran = (h * jt + hu * d4) + hv * d5;
  c.f1 = DIR == 0 ? fnorm : ftran;
  c.f2 = DIR == 0 ? ftran : fnorm;
  c.s = fabs(un) + sqrt(gh);
  c.ok = fast;
  // getJakobi's NaN trap (SMOD_jakobian.f90:55-70) and dgeev's complex-eigenvalue abort
  // (utility/SMOD_eigenvalue_problem.f90:72-83, h < 0) become status bits.  A cell in the
  // fast range has h > 0 and finite Jacobian entries.
  if (!fast) {
    if (isnan(jn) || isnan(d2) || isnan(jt) || isnan(d4) || isnan(d5)) *bad |= kStatusNaN;
    if (h < 0.0) *bad |= kStatusNegDepth;
  }
  return c;
}

// HLL two-wave solve at one interface (SMOD_approximate_Riemann_solvers.f90:189-224):
// s2 = max(sL, sR), s1 = -s2; if |s1| > eps and |s2| > eps:
//   q* = (((fR - fL) - s2*qR) + s1*qL) / ((eps + s1) - s2),  W1 = q* - qL,  W2 = qR - q*
// else lambda = 0 and W = 0.  Returns s2 (0 for the degenerate interface).
struct Waves {
  double w1[3], w2[3];
};

template <int OPT = 0>
__device__ __forceinline__ double hll(const double qL[3], const CellFlux& fL, const double qR[3],
                                      const CellFlux& fR, Waves& W) {
  const double smax = fmax(fL.s, fR.s);
  const double s1 = -smax;
  if (fabs(s1) > kUdPrecision && fabs(smax) > kUdPrecision) {
    const double den = (kUdPrecision + s1) - smax;
    const double fl[3] = {fL.f0, fL.f1, fL.f2};
    const double fr[3] = {fR.f0, fR.f1, fR.f2};
    double num[3];
#pragma unroll
    for (int me = 0; me < 3; ++me) num[me] = ((fr[me] - fl[me]) - smax * qR[me]) + s1 * qL[me];
    double qs[3];
    if ((OPT & kOptFastDiv) != 0 && fL.ok && fR.ok) {  // both cells in range: one reciprocal
      const Den d = den_of(den);
#pragma unroll
      for (int me = 0; me < 3; ++me) qs[me] = quot(num[me], d);
    } else {
#pragma unroll
      for (int me = 0; me < 3; ++me) qs[me] = div_neg_den(num[me], den);
    }
#pragma unroll
    for (int me = 0; me < 3; ++me) {
      W.w1[me] = qs[me] - qL[me];
      W.w2[me] = qR[me] - qs[me];
    }
    return smax;
  }
#pragma unroll
  for (int me = 0; me < 3; ++me) {
    W.w1[me] = 0.0;
    W.w2[me] = 0.0;
  }
  return 0.0;
}

// limiter function phi(theta) by code (solver/MOD_flux_correction.f90:101-112)
template <int LIM>
__device__ __forceinline__ double limiter_phi(double r) {
  if (LIM == 1) return fmax(0.0, fmin(1.0, r));
  if (LIM == 2) return fmax(fmax(0.0, fmin(1.0, 2.0 * r)), fmin(2.0, r));
  if (LIM == 3) return div_pos_den(r + fabs(r), 1.0 + fabs(r));  // zero numerator for every r <= 0
  return fmax(0.0, fmin(fmin((1.0 + r) / 2.0, 2.0), 2.0 * r));
}

__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
  return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

// Limited wave for one family p at interface k (MOD_flux_correction.f90:74-123).  All three
// waves are the unlimited ones: the reference's carried wnorm2r is the dot product of the
// original waves at k and k+1, taken before wave k is limited in place.
//   upstream = lambda_p > 0 ? W_{k-1}.W_k : W_k.W_{k+1};  theta = upstream / |W_k|^2
//   W~ = |W_k|^2 <= eps ? W_k : phi(theta) * W_k
//
// kOptLimSat leaves the division out where phi is known without it (wn2 > eps > 0 here):
//   up >= K*wn2 means theta >= K, where phi saturates: minmod (K = 1) and superbee (K = 2) give
//     phi = K, MC (K = 4, a power of two so K*wn2 is exact) gives 2; van Leer never saturates;
//   up < -2^-900 with wn2 < 2^100 means theta is a negative normal number (it cannot underflow
//     to -0), where every limiter gives +0 (fmax(0, negative) = +0; van Leer: (t + |t|) = +0).
// Everything else divides, so phi has the same bits either way.
template <int LIM, int OPT = 0>
__device__ __forceinline__ void limit_wave(const double wm[3], const double w[3], const double wp[3],
                                           bool lambda_pos, double out[3]) {
  const double wn2 = dot3(w, w);
  if (fabs(wn2) <= kUdPrecision) {
    out[0] = w[0];
    out[1] = w[1];
    out[2] = w[2];
    return;
  }
  const double up = lambda_pos ? dot3(wm, w) : dot3(w, wp);
  double phi;
  if constexpr ((OPT & kOptLimSat) != 0) {
    constexpr double K = LIM == 1 ? 1.0 : LIM == 2 ? 2.0 : 4.0;
    constexpr double SAT = LIM == 1 ? 1.0 : 2.0;
    if (LIM != 3 && up >= K * wn2)
      phi = SAT;
    else if (up < -0x1p-900 && wn2 < 0x1p100)
      phi = 0.0;
    else
      phi = limiter_phi<LIM>(div_pos_den(up, wn2));
  } else {
    phi = limiter_phi<LIM>(div_pos_den(up, wn2));
  }
  out[0] = phi * w[0];
  out[1] = phi * w[1];
  out[2] = phi * w[2];
}

// Correction coefficient of one interface, the same for both waves because |s1| = |s2|
// (MOD_flux_correction.f90:162-165): (0.5*|l|) * (1 - (|l|*dt/delta) / (0.5*(kap_{k-1}+kap_k)))
__device__ __forceinline__ double corr_coef(double s2, double dtod, double kap_l, double kap_r) {
  if (s2 == 0.0) return 0.0;
  const double kb = 0.5 * (kap_l + kap_r);
  return (0.5 * s2) * (1.0 - (s2 * dtod) / kb);
}

// corr_coef with kap_l = kap_r = 1: 0.5*(1+1) = 1 and (s2*dtod)/1 = s2*dtod exactly
__device__ __forceinline__ double corr_coef_unit(double s2, double dtod) {
  if (s2 == 0.0) return 0.0;
  return (0.5 * s2) * (1.0 - s2 * dtod);
}

// Capacity kappa(i,j) of the uniform identity-mapped grid: the shoelace area
// (domain/SMOD_mesh_manipulation.f90:165-173) reduces to (p1*d + p3*d') / (d_xi*d_eta) with
// p1 = 0.5*(e1+e1), p3 = 0.5*(e3+e3) per row and d = c1-c2, d' = c2-c1 per column; the two
// vanishing shoelace terms are signed zeros that leave a non-zero sum unchanged.
__device__ __forceinline__ double capacity(const double* rowm, const double* colm, int i, int j,
                                           double area_scale) {
  const double p1 = __ldg(rowm + (j + 1) * kRowMetrics + 0);
  const double p3 = __ldg(rowm + (j + 1) * kRowMetrics + 1);
  const double d = __ldg(colm + (i + 1) * kColMetrics + 0);
  const double dp = __ldg(colm + (i + 1) * kColMetrics + 1);
  return (p1 * d + p3 * dp) / area_scale;
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double v) {
  if (v > 0.0) atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace pcl
