// Warp-level building blocks shared by the pair kernels (refinement, distance, erosion): local edge lists,
// crossing parity, containment probes. Restating engine/engine.cuh:322-412 of landstats-us/postgis-cuda.
#pragma once
#include "geom.cuh"

namespace gsj {

__device__ __forceinline__ EList carve(unsigned char* base, int cap) {
  EList L;
  L.x0 = reinterpret_cast<double*>(base);
  L.y0 = L.x0 + cap; L.x1 = L.y0 + cap; L.y1 = L.x1 + cap;
  L.fl = reinterpret_cast<uint32_t*>(L.y1 + cap);
  return L;
}
__device__ __forceinline__ EList carve_f(unsigned char* base, int cap) { return carve(base, cap); }
// edge (x0, y0)-(x1, y1) entirely outside box [bx0, bx1] x [by0, by1], by comparisons only
__device__ __forceinline__ bool out_cmp(double x0, double y0, double x1, double y1, double bx0, double by0, double bx1, double by1) {
  return (x0 < bx0 && x1 < bx0) || (x0 > bx1 && x1 > bx1) || (y0 < by0 && y1 < by0) || (y0 > by1 && y1 > by1);
}
__device__ __forceinline__ bool edge_outside(double px, double py, double qx, double qy, const Box& o) {
  return fmax(px, qx) < o.x0 || fmin(px, qx) > o.x1 || fmax(py, qy) < o.y0 || fmin(py, qy) > o.y1;
}

// all edges of geometry A meeting the overlap box, compacted in ring order with a warp ballot (engine.cuh:358-377).
// PIP: the same pass also takes the crossing parity of the segment (A's bbox left edge - 1, my) -> (mx, my) over
// every edge of A, as pip_full_warp does (an XOR over the edges, so the order is free), into *inside.
template <bool F, bool PIP = false, bool S32 = false>
static __device__ int collect(const Frame& A, const Box& ov, EList L, int cap, int lane, double mx = 0, double my = 0, bool* inside = nullptr) {
  const DLayer& S = *A.L;
  const unsigned lt = (1u << lane) - 1;
  const double ox = A.shx - (double)1, oy = my;
  bool par = false;
  int cnt = 0;
  for (uint32_t ra = A.r0; ra < A.r1; ra++) {
    const uint64_t s = S.rvo[ra], e = S.rvo[ra + 1];
    for (uint64_t base = s; base + 1 < e; base += 32) {
      const uint64_t i = base + lane;
      bool in = false;
      double x0 = 0, y0 = 0, x1 = 0, y1 = 0; uint32_t fl = 0;
      if (i + 1 < e) {
        A.v(i, x0, y0); A.v(i + 1, x1, y1);
        if (S.synb) {
          fl = (uint32_t)S.syn(i) | (S.syn(i > s ? i - 1 : e - 2) ? 2u : 0u) | (S.syn(i + 2 < e ? i + 1 : s) ? 4u : 0u);
        }
        in = F ? !out_cmp(x0, y0, x1, y1, ov.x0, ov.y0, ov.x1, ov.y1) : !edge_outside(x0, y0, x1, y1, ov);
        if (PIP && !((y0 > my) == (y1 > my) && y0 != my && y1 != my)) {
          if (S32) {   // the same signs through the certified FP32 filter
            const bool so = left_of32(x0, y0, x1, y1, ox, oy), sc = left_of32(x0, y0, x1, y1, mx, my);
            if (so != sc) {
              const bool su = orient_sign32(ox, oy, mx, my, x0, y0) > 0, sv = orient_sign32(ox, oy, mx, my, x1, y1) > 0;
              if (su != sv) par = !par;
            }
          } else {
            const bool so = left_of(x0, y0, x1, y1, ox, oy), sc = left_of(x0, y0, x1, y1, mx, my);
            if (so != sc) {
              const bool su = orient(ox, oy, mx, my, x0, y0) > 0, sv = orient(ox, oy, mx, my, x1, y1) > 0;
              if (su != sv) par = !par;
            }
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, in);
      const int pos = cnt + __popc(m & lt);
      if (in && pos < cap) {
        L.x0[pos] = x0; L.y0[pos] = y0; L.x1[pos] = x1; L.y1[pos] = y1; L.fl[pos] = fl;
      }
      cnt += __popc(m);
    }
  }
  if (PIP) *inside = (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
  return cnt;
}

// crossing parity of segment (B's bbox left edge - 1, my) -> (mx, my) over all of B's edges (engine.cuh:382-397)
static __device__ bool pip_full_warp(const Frame& B, double mx, double my, int lane) {
  const DLayer& S = *B.L;
  const double ox = B.shx - (double)1, oy = my;
  bool par = false;
  for (uint32_t r = B.r0; r < B.r1; r++) {
    const uint64_t s = S.rvo[r], e = S.rvo[r + 1];
    for (uint64_t j = s + 1 + lane; j < e; j += 32) {
      double x0, y0, x1, y1; B.v(j - 1, x0, y0); B.v(j, x1, y1);
      if ((y0 > my) == (y1 > my) && y0 != my && y1 != my) continue;
      bool so = left_of(x0, y0, x1, y1, ox, oy), sc = left_of(x0, y0, x1, y1, mx, my);
      if (so == sc) continue;
      bool su = orient(ox, oy, mx, my, x0, y0) > 0, sv = orient(ox, oy, mx, my, x1, y1) > 0;
      if (su != sv) par = !par;
    }
  }
  return (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
}

// inside(x) = inside(c) xor crossings of c -> x with the local edges (engine.cuh:400-412)
// S32: the four orientation signs through the certified FP32 filter (the same booleans)
template <bool F, bool S32 = false>
__device__ __forceinline__ bool inside_from_c(const EList& L, int cnt, double cx, double cy, bool in_c, double x, double y) {
  bool in = in_c;
  const double sx0 = fmin(cx, x), sx1 = fmax(cx, x), sy0 = fmin(cy, y), sy1 = fmax(cy, y);
  auto step = [&](int k) {
    const double ex0 = L.x0[k], ey0 = L.y0[k], ex1 = L.x1[k], ey1 = L.y1[k];
    if (F ? out_cmp(ex0, ey0, ex1, ey1, sx0, sy0, sx1, sy1)
          : (fmax(ex0, ex1) < sx0 || fmin(ex0, ex1) > sx1 || fmax(ey0, ey1) < sy0 || fmin(ey0, ey1) > sy1)) return false;
    if constexpr (S32) {
      const bool sc = left_of32(ex0, ey0, ex1, ey1, cx, cy), sx = left_of32(ex0, ey0, ex1, ey1, x, y);
      if (sc == sx) return false;
      const bool su = orient_sign32(cx, cy, x, y, ex0, ey0) > 0, sv = orient_sign32(cx, cy, x, y, ex1, ey1) > 0;
      if (su != sv) in = !in;
    } else {
      bool sc = left_of(ex0, ey0, ex1, ey1, cx, cy), sx = left_of(ex0, ey0, ex1, ey1, x, y);
      if (sc == sx) return false;
      bool su = orient(cx, cy, x, y, ex0, ey0) > 0, sv = orient(cx, cy, x, y, ex1, ey1) > 0;
      if (su != sv) in = !in;
    }
    return false;
  };
  for (int k = 0; k < cnt; k++) step(k);
  return in;
}

// The same parity for one query point shared by the whole warp: lanes split the edges, a ballot counts crossings
// (the parity does not depend on the order of the edges).
template <bool S32 = false>
static __device__ bool inside_from_c_warp(const EList& L, int cnt, double cx, double cy, bool in_c, double x, double y, int lane) {
  const double sx0 = fmin(cx, x), sx1 = fmax(cx, x), sy0 = fmin(cy, y), sy1 = fmax(cy, y);
  bool par = false;
  for (int k = lane; k < cnt; k += 32) {
    const double ex0 = L.x0[k], ey0 = L.y0[k], ex1 = L.x1[k], ey1 = L.y1[k];
    if (out_cmp(ex0, ey0, ex1, ey1, sx0, sy0, sx1, sy1)) continue;
    const bool sc = S32 ? left_of32(ex0, ey0, ex1, ey1, cx, cy) : left_of(ex0, ey0, ex1, ey1, cx, cy);
    const bool sx = S32 ? left_of32(ex0, ey0, ex1, ey1, x, y) : left_of(ex0, ey0, ex1, ey1, x, y);
    if (sc == sx) continue;
    const bool su = (S32 ? orient_sign32(cx, cy, x, y, ex0, ey0) : orient(cx, cy, x, y, ex0, ey0)) > 0;
    const bool sv = (S32 ? orient_sign32(cx, cy, x, y, ex1, ey1) : orient(cx, cy, x, y, ex1, ey1)) > 0;
    if (su != sv) par = !par;
  }
  const bool odd = (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
  return in_c != odd;
}

__device__ __forceinline__ bool probe_vertex(const Frame& A, uint32_t r, double& x, double& y) {   // engine.cuh:322-327
  const DLayer& S = *A.L;
  uint64_t v = S.rvo[r], e = S.rvo[r + 1];
  if (S.synb) { while (v + 1 < e && S.syn(v)) v++; if (v + 1 >= e) return false; }
  A.v(v, x, y);
  return true;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gsj
