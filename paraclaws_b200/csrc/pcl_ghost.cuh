// pcl_ghost.cuh -- ghost fill of update_rank_boundaries -> apply_physical_boundaries
// (user_subroutines/SMOD_boundary_conditions.f90:58-213) for one grid, as a device function
// over item indices so a whole kernel or one CTA of a batched kernel can run it.
// Items: 4 sides x 2 layers x max(m_xi, m_eta) positions; corners are never written.
// Code 1 (BC_USER, which aborts in the reference) is a reflective wall here: the two ghost
// layers mirror the two nearest interior cells with the normal momentum negated.
#pragma once
#include <cuda_runtime.h>

#include "pcl_types.h"

namespace pcl {

__device__ __forceinline__ int ghost_items(const GridDev& g) { return 8 * max(g.mx, g.my); }

// One ghost cell's three values and where they go (plane 0; plane p at dst + p * plane).
struct GhostVal {
  double* dst;
  double v[3];
};

// Loads only: no ghost item reads a cell that another one writes (sources are interior cells
// and the metric tables), so the three planes of an item are all loaded before any is stored
// (one memory round trip per item, not one per plane).  Returns false where it writes nothing.
__device__ __forceinline__ bool ghost_value(const GridDev& g, double* b, int tid, GhostVal& o) {
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
#pragma unroll
    for (int me = 0; me < 3; ++me) {
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
        v = me == 1 ? -p[im + 1] : p[im + 1];
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
#pragma unroll
    for (int me = 0; me < 3; ++me) {
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
        v = me == 2 ? -p[(long long)(jm + 1) * P] : p[(long long)(jm + 1) * P];
      }
      o.v[me] = v;
    }
  }
  return true;
}

__device__ __forceinline__ void ghost_store(const GridDev& g, const GhostVal& o) {
  o.dst[0] = o.v[0];
  o.dst[g.plane] = o.v[1];
  o.dst[2 * g.plane] = o.v[2];
}

__device__ __forceinline__ void ghost_item(const GridDev& g, double* b, int tid) {
  GhostVal o;
  if (ghost_value(g, b, tid, o)) ghost_store(g, o);
}

}  // namespace pcl
