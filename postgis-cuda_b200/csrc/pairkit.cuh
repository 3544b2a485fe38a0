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
template <bool F, bool PIP = false>
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
          const bool so = left_of(x0, y0, x1, y1, ox, oy), sc = left_of(x0, y0, x1, y1, mx, my);
          if (so != sc) {
            const bool su = orient(ox, oy, mx, my, x0, y0) > 0, sv = orient(ox, oy, mx, my, x1, y1) > 0;
            if (su != sv) par = !par;
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

// Both geometries of a pair at once: each iteration a lane takes one edge of A and one of B (32 of each per
// iteration), so the two polygons' load chains are in flight together; each list is compacted in ring order with its
// own ballot, and each polygon's crossing parity for the probe point (mx, my) is taken in the same pass, as collect
// does for one geometry. Returns the counts in na / nb (a count above cap: that list was not fully kept).
struct RingWalk {   // the warp's position in one geometry's rings (the same in every lane)
  uint32_t r, r1; uint64_t s, e, base; bool done;
  __device__ __forceinline__ void start(const Frame& G) {
    const DLayer& S = *G.L;
    r = G.r0; r1 = G.r1; done = r >= r1; s = e = base = 0;
    if (!done) { s = S.rvo[r]; e = S.rvo[r + 1]; base = s; }
    skip(G);
  }
  __device__ __forceinline__ void skip(const Frame& G) {   // to the next ring with an edge left
    const DLayer& S = *G.L;
    while (!done && base + 1 >= e) {
      if (++r >= r1) { done = true; break; }
      s = S.rvo[r]; e = S.rvo[r + 1]; base = s;
    }
  }
};
template <bool F>
__device__ __forceinline__ bool take_edge(const Frame& G, const RingWalk& w, const Box& ov, int lane, double mx, double my, bool& par,
                                          double& x0, double& y0, double& x1, double& y1, uint32_t& fl) {
  if (w.done) return false;
  const DLayer& S = *G.L;
  const uint64_t i = w.base + lane, s = w.s, e = w.e;
  if (i + 1 >= e) return false;
  G.v(i, x0, y0); G.v(i + 1, x1, y1);
  fl = 0;
  if (S.synb) fl = (uint32_t)S.syn(i) | (S.syn(i > s ? i - 1 : e - 2) ? 2u : 0u) | (S.syn(i + 2 < e ? i + 1 : s) ? 4u : 0u);
  if (!((y0 > my) == (y1 > my) && y0 != my && y1 != my)) {
    const double ox = G.shx - (double)1, oy = my;
    const bool so = left_of(x0, y0, x1, y1, ox, oy), sc = left_of(x0, y0, x1, y1, mx, my);
    if (so != sc) {
      const bool su = orient(ox, oy, mx, my, x0, y0) > 0, sv = orient(ox, oy, mx, my, x1, y1) > 0;
      if (su != sv) par = !par;
    }
  }
  return F ? !out_cmp(x0, y0, x1, y1, ov.x0, ov.y0, ov.x1, ov.y1) : !edge_outside(x0, y0, x1, y1, ov);
}
template <bool F>
static __device__ void collect_both(const Frame& A, const Frame& B, const Box& ov, EList LA, EList LB, int cap, int lane, double mx, double my,
                                    int& na, int& nb, bool& inA, bool& inB) {
  const unsigned lt = (1u << lane) - 1;
  RingWalk wa, wb;
  wa.start(A); wb.start(B);
  bool pa = false, pb = false;
  int ca = 0, cb = 0;
  while (!wa.done || !wb.done) {
    double ax0 = 0, ay0 = 0, ax1 = 0, ay1 = 0, bx0 = 0, by0 = 0, bx1 = 0, by1 = 0;
    uint32_t fa = 0, fb = 0;
    const bool ka = take_edge<F>(A, wa, ov, lane, mx, my, pa, ax0, ay0, ax1, ay1, fa);
    const bool kb = take_edge<F>(B, wb, ov, lane, mx, my, pb, bx0, by0, bx1, by1, fb);
    const unsigned ma = __ballot_sync(0xffffffffu, ka), mb = __ballot_sync(0xffffffffu, kb);
    const int qa = ca + __popc(ma & lt), qb = cb + __popc(mb & lt);
    if (ka && qa < cap) { LA.x0[qa] = ax0; LA.y0[qa] = ay0; LA.x1[qa] = ax1; LA.y1[qa] = ay1; LA.fl[qa] = fa; }
    if (kb && qb < cap) { LB.x0[qb] = bx0; LB.y0[qb] = by0; LB.x1[qb] = bx1; LB.y1[qb] = by1; LB.fl[qb] = fb; }
    ca += __popc(ma); cb += __popc(mb);
    if (!wa.done) { wa.base += 32; wa.skip(A); }
    if (!wb.done) { wb.base += 32; wb.skip(B); }
  }
  na = ca; nb = cb;
  inA = (__popc(__ballot_sync(0xffffffffu, pa)) & 1) != 0;
  inB = (__popc(__ballot_sync(0xffffffffu, pb)) & 1) != 0;
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
template <bool F>
__device__ __forceinline__ bool inside_from_c(const EList& L, int cnt, double cx, double cy, bool in_c, double x, double y) {
  bool in = in_c;
  const double sx0 = fmin(cx, x), sx1 = fmax(cx, x), sy0 = fmin(cy, y), sy1 = fmax(cy, y);
  auto step = [&](int k) {
    const double ex0 = L.x0[k], ey0 = L.y0[k], ex1 = L.x1[k], ey1 = L.y1[k];
    if (F ? out_cmp(ex0, ey0, ex1, ey1, sx0, sy0, sx1, sy1)
          : (fmax(ex0, ex1) < sx0 || fmin(ex0, ex1) > sx1 || fmax(ey0, ey1) < sy0 || fmin(ey0, ey1) > sy1)) return false;
    bool sc = left_of(ex0, ey0, ex1, ey1, cx, cy), sx = left_of(ex0, ey0, ex1, ey1, x, y);
    if (sc == sx) return false;
    bool su = orient(cx, cy, x, y, ex0, ey0) > 0, sv = orient(cx, cy, x, y, ex1, ey1) > 0;
    if (su != sv) in = !in;
    return false;
  };
  for (int k = 0; k < cnt; k++) step(k);
  return in;
}

// The same parity for one query point shared by the whole warp: lanes split the edges, a ballot counts crossings
// (the parity does not depend on the order of the edges).
static __device__ bool inside_from_c_warp(const EList& L, int cnt, double cx, double cy, bool in_c, double x, double y, int lane) {
  const double sx0 = fmin(cx, x), sx1 = fmax(cx, x), sy0 = fmin(cy, y), sy1 = fmax(cy, y);
  bool par = false;
  for (int k = lane; k < cnt; k += 32) {
    const double ex0 = L.x0[k], ey0 = L.y0[k], ex1 = L.x1[k], ey1 = L.y1[k];
    if (out_cmp(ex0, ey0, ex1, ey1, sx0, sy0, sx1, sy1)) continue;
    bool sc = left_of(ex0, ey0, ex1, ey1, cx, cy), sx = left_of(ex0, ey0, ex1, ey1, x, y);
    if (sc == sx) continue;
    bool su = orient(cx, cy, x, y, ex0, ey0) > 0, sv = orient(cx, cy, x, y, ex1, ey1) > 0;
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
