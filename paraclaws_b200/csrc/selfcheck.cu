// selfcheck.cu -- device self-checks of the arithmetic shortcuts the FP64 sweeps rely on.  Each
// one runs the shortcut and the plain IEEE operations side by side on the GPU and counts the
// inputs whose results differ in any bit.  Built with --fmad=false like the sweeps.
//
//  * pcl_check_quotients / pcl_check_quotients_random: quot(a, den_of(b)) (a correctly rounded
//    quotient from a shared reciprocal by Markstein's correction, pcl_fp64.cuh) against a / b,
//    for pairs inside the method's range: |a|, |b| and |a/b| in [2^-960, 2^960], or a = 0.
//  * pcl_check_flux_paths: the cell flux and HLL solve of both sweep directions with the
//    shared-reciprocal quotients (kOptFastDiv) against the same code with IEEE division, on
//    random cells across the range the sweeps admit to the fast path (h, |hu|, |hv| in
//    [2^-64, 2^64) or momenta 0), and the limiter with and without kOptLimSat.
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "../../include/paraclaws_b200.h"
#include "pcl_fp64.cuh"

using namespace pcl;

namespace {

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// a double with random sign and mantissa and a biased exponent uniform in [elo, ehi]
__device__ __forceinline__ double rand_double(unsigned long long r, unsigned long long r2, int elo, int ehi) {
  const unsigned long long e = (unsigned long long)(elo + (int)(r2 % (unsigned long long)(ehi - elo + 1)));
  const unsigned long long bits = (r & 0x800FFFFFFFFFFFFFull) | (e << 52);
  return __longlong_as_double((long long)bits);
}

// |x| == 0 or its biased exponent in [63, 1983] (2^-960 .. 2^960)
__device__ __forceinline__ bool in_method_range(double x) {
  const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7ffu;
  return e - 63u <= 1920u;
}

__device__ __forceinline__ bool same_bits(double x, double y) {
  return __double_as_longlong(x) == __double_as_longlong(y);
}

__device__ int check_pair(double a, double b) {  // 0: equal, 1: differ, 2: outside the range
  if (!in_method_range(b) || b == 0.0) return 2;
  if (a != 0.0 && !in_method_range(a)) return 2;
  const double q = a / b;
  if (a != 0.0 && !in_method_range(q)) return 2;
  return same_bits(quot(a, den_of(b)), q) ? 0 : 1;
}

__global__ void quot_pairs_kernel(const double* a, const double* b, long long n, unsigned long long* counts) {
  unsigned long long bad = 0, used = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const int r = check_pair(a[k], b[k]);
    bad += r == 1;
    used += r != 2;
  }
  atomicAdd(&counts[0], bad);
  atomicAdd(&counts[1], used);
}

// Random pairs in four families: (0) both operands over the whole method range, (1) both in
// [2^-64, 2^64) as in the sweeps, (2) a = 0 or a power of two, b with an all-ones mantissa,
// (3) quotients near 1 (a = b * (1 + small)).
__global__ void quot_random_kernel(long long n, unsigned long long seed, unsigned long long* counts) {
  unsigned long long bad = 0, used = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    const unsigned long long r0 = mix64(seed ^ (2 * (unsigned long long)k)), r1 = mix64(r0), r2 = mix64(r1),
                             r3 = mix64(r2);
    double a, b;
    switch (k & 3) {
      case 0:
        a = rand_double(r0, r1, 100, 1946);
        b = rand_double(r2, r3, 100, 1946);
        break;
      case 1:
        a = rand_double(r0, r1, 959, 1086);
        b = rand_double(r2, r3, 959, 1086);
        break;
      case 2:
        a = (r0 & 1) ? 0.0 : ldexp(1.0, (int)(r1 % 200) - 100);
        if (r0 & 2) a = -a;
        b = __longlong_as_double((long long)((r2 & 0x8000000000000000ull) | ((900ull + r3 % 250) << 52) |
                                             0x000FFFFFFFFFFFFFull));
        break;
      default: {
        b = rand_double(r0, r1, 959, 1086);
        const double eps = ldexp((double)(r2 & 0xFFFF) - 32768.0, -(int)(40 + r3 % 12));
        a = b * (1.0 + eps);
      }
    }
    const int r = check_pair(a, b);
    bad += r == 1;
    used += r != 2;
  }
  atomicAdd(&counts[0], bad);
  atomicAdd(&counts[1], used);
}

// a value for a cell component: 0 with probability 1/8 (momenta only), else random sign,
// exponent in [-64, 63] weighted towards O(1) and the range ends
__device__ double rand_component(unsigned long long r, unsigned long long r2, bool positive, bool allow_zero) {
  if (allow_zero && (r2 & 7) == 0) return (r2 & 8) ? -0.0 : 0.0;
  int e;
  switch ((r2 >> 4) & 3) {
    case 0: e = 959; break;                               // 2^-64 ..
    case 1: e = 1086; break;                              // .. 2^63
    default: e = 1013 + (int)((r2 >> 8) % 21);            // 2^-10 .. 2^10
  }
  if ((r2 >> 6) & 1) e = 959 + (int)((r2 >> 16) % 128);  // anywhere in the range
  double x = rand_double(r, 0, e, e);
  if (positive) x = fabs(x);
  return x;
}

template <int DIR>
__device__ int flux_pair_differs(const double qL[3], const double qR[3], double g) {
  int b0 = 0, b1 = 0;
  const CellFlux L0 = cell_flux<DIR, 0>(qL[0], qL[1], qL[2], g, &b0);
  const CellFlux R0 = cell_flux<DIR, 0>(qR[0], qR[1], qR[2], g, &b0);
  const CellFlux L1 = cell_flux<DIR, kOptFastDiv>(qL[0], qL[1], qL[2], g, &b1);
  const CellFlux R1 = cell_flux<DIR, kOptFastDiv>(qR[0], qR[1], qR[2], g, &b1);
  int d = b0 != b1;
  d |= !same_bits(L0.f0, L1.f0) || !same_bits(L0.f1, L1.f1) || !same_bits(L0.f2, L1.f2) || !same_bits(L0.s, L1.s);
  d |= !same_bits(R0.f0, R1.f0) || !same_bits(R0.f1, R1.f1) || !same_bits(R0.f2, R1.f2) || !same_bits(R0.s, R1.s);
  Waves W0, W1;
  const double s0 = hll<0>(qL, L0, qR, R0, W0);
  const double s1 = hll<kOptFastDiv>(qL, L1, qR, R1, W1);
  d |= !same_bits(s0, s1);
#pragma unroll
  for (int k = 0; k < 3; ++k) d |= !same_bits(W0.w1[k], W1.w1[k]) || !same_bits(W0.w2[k], W1.w2[k]);
  return d;
}

template <int LIM>
__device__ int limiter_differs(const double wm[3], const double w[3], const double wp[3], bool pos) {
  double a[3], b[3];
  limit_wave<LIM, 0>(wm, w, wp, pos, a);
  limit_wave<LIM, kOptLimSat>(wm, w, wp, pos, b);
  return !same_bits(a[0], b[0]) || !same_bits(a[1], b[1]) || !same_bits(a[2], b[2]);
}

__global__ void flux_paths_kernel(long long n, unsigned long long seed, double g, unsigned long long* counts) {
  unsigned long long bad_flux = 0, fast = 0, bad_lim = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
    unsigned long long r = mix64(seed ^ (0x5151ull + 2 * (unsigned long long)k));
    double qL[3], qR[3];
    for (int c = 0; c < 3; ++c) {
      const unsigned long long x = mix64(r), y = mix64(x);
      qL[c] = rand_component(x, y, c == 0, c != 0);
      r = mix64(y);
      const unsigned long long x2 = mix64(r), y2 = mix64(x2);
      // the right cell: independent, or the left one nudged by a few ulps (small jumps)
      qR[c] = (y2 & 0x300) == 0x300 || qL[c] == 0.0
                  ? rand_component(x2, y2, c == 0, c != 0)
                  : __longlong_as_double(__double_as_longlong(qL[c]) + (long long)(x2 % 9) - 4);
      if (c == 0) qR[c] = fabs(qR[c]);
      r = mix64(y2);
    }
    int dummy = 0;
    fast += cell_flux<0, kOptFastDiv>(qL[0], qL[1], qL[2], g, &dummy).ok &&
            cell_flux<0, kOptFastDiv>(qR[0], qR[1], qR[2], g, &dummy).ok;
    bad_flux += flux_pair_differs<0>(qL, qR, g) | flux_pair_differs<1>(qL, qR, g);
    // limiter: three waves from differences of the cells, scaled, with either wave direction
    double wm[3], w[3], wp[3];
    for (int c = 0; c < 3; ++c) {
      const unsigned long long x = mix64(r);
      r = mix64(x);
      const double s = ldexp(1.0, (int)(x % 80) - 40);
      w[c] = (qR[c] - qL[c]) * s;
      wm[c] = (x & 0x100000) ? w[c] * ((double)((x >> 24) & 0xFFF) / 1024.0 - 2.0) : qL[c] * s;
      wp[c] = (x & 0x200000) ? w[c] * ((double)((x >> 40) & 0xFFF) / 512.0 - 4.0) : qR[c] * s;
    }
    const bool pos = r & 1;
    bad_lim += limiter_differs<1>(wm, w, wp, pos) | limiter_differs<2>(wm, w, wp, pos) |
               limiter_differs<3>(wm, w, wp, pos) | limiter_differs<4>(wm, w, wp, pos);
  }
  atomicAdd(&counts[0], bad_flux);
  atomicAdd(&counts[1], fast);
  atomicAdd(&counts[2], bad_lim);
}

template <class F>
int run_counts(F launch, int ncounts, long long* out) {
  unsigned long long* d = nullptr;
  if (cudaMalloc(&d, sizeof(unsigned long long) * 4) != cudaSuccess) return PCL_ERR_OOM;
  cudaMemset(d, 0, sizeof(unsigned long long) * 4);
  launch(d);
  unsigned long long h[4] = {0, 0, 0, 0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "paraclaws_b200 self-check: %s\n", cudaGetErrorString(e));
    return PCL_ERR_CUDA;
  }
  for (int k = 0; k < ncounts; ++k) out[k] = (long long)h[k];
  return PCL_OK;
}

}  // namespace

extern "C" {

int pcl_check_quotients(const double* a, const double* b, long long n, long long* mismatches, long long* checked) {
  if (!a || !b || n < 0 || !mismatches) return PCL_ERR_BADARG;
  double *da = nullptr, *db = nullptr;
  if (cudaMalloc(&da, sizeof(double) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) return PCL_ERR_OOM;
  if (cudaMalloc(&db, sizeof(double) * (size_t)(n > 0 ? n : 1)) != cudaSuccess) {
    cudaFree(da);
    return PCL_ERR_OOM;
  }
  cudaMemcpy(da, a, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice);
  cudaMemcpy(db, b, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice);
  long long c[2] = {0, 0};
  const int r = run_counts([&](unsigned long long* d) { quot_pairs_kernel<<<1184, 256>>>(da, db, n, d); }, 2, c);
  cudaFree(da);
  cudaFree(db);
  *mismatches = c[0];
  if (checked) *checked = c[1];
  return r;
}

int pcl_check_quotients_random(long long n, unsigned long long seed, long long* mismatches, long long* checked) {
  if (n < 0 || !mismatches) return PCL_ERR_BADARG;
  long long c[2] = {0, 0};
  const int r = run_counts([&](unsigned long long* d) { quot_random_kernel<<<2368, 256>>>(n, seed, d); }, 2, c);
  *mismatches = c[0];
  if (checked) *checked = c[1];
  return r;
}

int pcl_check_flux_paths(long long n, unsigned long long seed, double grav, long long* flux_mismatches,
                         long long* fast_pairs, long long* limiter_mismatches) {
  if (n < 0 || !flux_mismatches) return PCL_ERR_BADARG;
  long long c[3] = {0, 0, 0};
  const int r =
      run_counts([&](unsigned long long* d) { flux_paths_kernel<<<2368, 128>>>(n, seed, grav, d); }, 3, c);
  *flux_mismatches = c[0];
  if (fast_pairs) *fast_pairs = c[1];
  if (limiter_mismatches) *limiter_mismatches = c[2];
  return r;
}

}  // extern "C"
