// pcl_ghost.cuh -- ghost fill of update_rank_boundaries -> apply_physical_boundaries
// (user_subroutines/SMOD_boundary_conditions.f90:58-213) for one grid, as a device function
// over item indices so a whole kernel or one CTA of a batched kernel can run it.
// Items: 4 sides x 2 layers x max(m_xi, m_eta) positions; corners are never written.
// Code 1 (BC_USER, which aborts in the reference) is a reflective wall here: the two ghost
// layers mirror the two nearest interior cells with the normal momentum (or velocity) of the
// equation module negated (pcl_eq_wall_component); a module without one mirrors every component.
// N: the context's number of equations (planes).
#pragma once
#include <cuda_runtime.h>

#include "pcl_equations.h"
#include "pcl_types.h"

namespace pcl {

__device__ __forceinline__ int ghost_items(const GridDev& g) { return 8 * max(g.mx, g.my); }

// One ghost cell's N values and where they go (plane 0; plane p at dst + p * plane).
template <int N = 3>
struct GhostVal {
  double* dst;
  double v[N];
};

// the component a wall negates on the xi (dir 1) or eta (dir 2) sides; -1: none
__device__ __forceinline__ int wall_component(const GridDev& g, int dir) {
  return g.eq == PCL_EQ_SHALLOW_WATER ? dir : pcl_eq_wall_component(g.eq, dir);
}

// Loads only: no ghost item reads a cell that another one writes (sources are interior cells
// and the metric tables), so the planes of an item are all loaded before any is stored
// (one memory round trip per item, not one per plane).  Returns false where it writes nothing.
template <int N = 3>
__device__ __forceinline__ bool ghost_value(const GridDev& g, double* b, int tid, GhostVal<N>& o) {
  const int mx = g.mx, my = g.my;
  const int n = max(mx, my);
  const int side = tid / (2 * n);
  const int rem = tid - side * 2 * n;
  const int layer = rem / n;
  const int idx = 1 + rem - layer * n;  // 1-based position along the side
  if (side >= 4) return false;
  const long long P = g.pitch;
  const int bc = g.bc[side];
  if (bc == 1 && g.user_bc) return false;  // the user boundary hook fills this side
  if (side < 2) {  // xi boundaries, rows j = 1 .. m_eta
    const int j = idx;
    if (j > my) return false;
    const int i = side == 0 ? -1 + layer : mx + 1 + layer;
    const int i1 = side == 0 ? 1 : mx;          // nearest interior cell
    const int i2 = side == 0 ? 2 : mx - 1;      // second interior cell
    const int im = side == 0 ? 1 - i : 2 * mx + 1 - i;
    const double xg = __ldg(g.colm + (i + 1) * kColMetrics + 3);
    const double x1 = __ldg(g.colm + (i1 + 1) * kColMetrics + 3);
    const double x2 = __ldg(g.colm + (i2 + 1) * kColMetrics + 3);
    o.dst = b + (long long)(j + 1) * P + (i + 1);
    const int wc = bc == 1 ? wall_component(g, 1) : -1;
#pragma unroll
    for (int me = 0; me < N; ++me) {
      const double* p = b + me * g.plane + (long long)(j + 1) * P;
      double v;
      if (bc == 2) {
        v = p[i1 + 1];
      } else if (bc == 3) {
        // deriv_2p(x_a, x_b, y_a, y_b) = (y_b - y_a)/(x_b - x_a) with (a, b) = (ilow, ilow+1)
        // on the left and (ihigh-1, ihigh) on the right (SMOD_boundary_conditions.f90:101-104)
        const double ya = side == 0 ? p[i1 + 1] : p[i2 + 1];
        const double yb = side == 0 ? p[i2 + 1] : p[i1 + 1];
        const double xa = side == 0 ? x1 : x2;
        const double xb = side == 0 ? x2 : x1;
        v = p[i1 + 1] + (yb - ya) / (xb - xa) * (xg - x1);
      } else {
        v = me == wc ? -p[im + 1] : p[im + 1];
      }
      o.v[me] = v;
    }
  } else {  // eta boundaries, columns i = 1 .. m_xi
    const int i = idx;
    if (i > mx) return false;
    const int j = side == 2 ? -1 + layer : my + 1 + layer;
    const int j1 = side == 2 ? 1 : my;
    const int j2 = side == 2 ? 2 : my - 1;
    const int jm = side == 2 ? 1 - j : 2 * my + 1 - j;
    const double yg = __ldg(g.rowm + (j + 1) * kRowMetrics + 3);
    const double y1 = __ldg(g.rowm + (j1 + 1) * kRowMetrics + 3);
    const double y2 = __ldg(g.rowm + (j2 + 1) * kRowMetrics + 3);
    o.dst = b + (long long)(j + 1) * P + (i + 1);
    const int wc = bc == 1 ? wall_component(g, 2) : -1;
#pragma unroll
    for (int me = 0; me < N; ++me) {
      const double* p = b + me * g.plane + (i + 1);
      double v;
      if (bc == 2) {
        v = p[(long long)(j1 + 1) * P];
      } else if (bc == 3) {
        const double va = side == 2 ? p[(long long)(j1 + 1) * P] : p[(long long)(j2 + 1) * P];
        const double vb = side == 2 ? p[(long long)(j2 + 1) * P] : p[(long long)(j1 + 1) * P];
        const double ya = side == 2 ? y1 : y2;
        const double yb = side == 2 ? y2 : y1;
        v = p[(long long)(j1 + 1) * P] + (vb - va) / (yb - ya) * (yg - y1);
      } else {
        v = me == wc ? -p[(long long)(jm + 1) * P] : p[(long long)(jm + 1) * P];
      }
      o.v[me] = v;
    }
  }
  return true;
}

template <int N = 3>
__device__ __forceinline__ void ghost_store(const GridDev& g, const GhostVal<N>& o) {
#pragma unroll
  for (int me = 0; me < N; ++me) o.dst[me * g.plane] = o.v[me];
}

template <int N = 3>
__device__ __forceinline__ void ghost_item(const GridDev& g, double* b, int tid) {
  GhostVal<N> o;
  if (ghost_value<N>(g, b, tid, o)) ghost_store<N>(g, o);
}

// Ghost cells next to a block of interior cells [i0, i1] x [j0, j1] of buffer b that the calling
// CTA has just written (batched kernels, before the step's accept decision: a rejected step
// leaves b unused).  A ghost value reads interior cells within two cells of its side, so the
// block fills a side along its own rows (xi) or columns (eta) when it holds both source cells:
// always on the low sides (cells 1 and 2 lie in the first block of a grid at least two cells
// wide), on a high side when the block is at least two cells deep there.  All threads of the CTA.
__device__ __forceinline__ void ghost_fill_block(const GridDev& g, double* b, int i0, int i1, int j0, int j1) {
  const int mx = g.mx, my = g.my, n = max(mx, my);
  const int nc = i1 - i0 + 1, nr = j1 - j0 + 1;
  const int c0 = i0 == 1 ? 2 * nr : 0;               // xi low: sources i = 1, 2
  const int c1 = i1 == mx && nc >= 2 ? 2 * nr : 0;   // xi high: i = mx, mx - 1
  const int c2 = j0 == 1 ? 2 * nc : 0;               // eta low: j = 1, 2
  const int c3 = j1 == my && nr >= 2 ? 2 * nc : 0;   // eta high: j = my, my - 1
  const int total = c0 + c1 + c2 + c3;
  for (int k = threadIdx.x; k < total; k += blockDim.x) {
    int side = 0, r = k;
    if (r >= c0) {
      r -= c0;
      side = 1;
      if (r >= c1) {
        r -= c1;
        side = 2;
        if (r >= c2) {
          r -= c2;
          side = 3;
        }
      }
    }
    const int len = side < 2 ? nr : nc;
    const int layer = r / len;
    const int pos = (side < 2 ? j0 : i0) + (r - layer * len);  // 1-based along the side
    ghost_item(g, b, side * 2 * n + layer * n + (pos - 1));
  }
}

// The high sides ghost_fill_block leaves to whoever runs after all blocks: xi high when the last
// block column is one cell wide, eta high when the last block row is one cell deep.
__device__ __forceinline__ void ghost_fill_open_sides(const GridDev& g, double* b, bool xi_hi, bool eta_hi) {
  const int n = max(g.mx, g.my);
  for (int k = threadIdx.x; k < 2 * n; k += blockDim.x) {
    if (xi_hi) ghost_item(g, b, 2 * n + k);
    if (eta_hi) ghost_item(g, b, 6 * n + k);
  }
}

}  // namespace pcl
