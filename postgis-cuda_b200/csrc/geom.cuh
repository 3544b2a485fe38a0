// Device-side layer views and exact FP64 predicates of the join engine.
//
// Arithmetic contract (shared with the CPU oracle so decisions are bit-identical): the library is compiled
// with --fmad=false (no implicit multiply-add contraction) and fma() appears exactly where the reference's
// compensated orientation uses it (engine/engine.cuh:283-289 of landstats-us/postgis-cuda). Coordinates are
// stored relative to each geometry's bbox minimum (exact, Sterbenz), so a vertex shared by two parcels has the
// same doubles in every pair frame (engine.cuh:14-18).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gsj {

// Resident polygon (or point) layer, structure of arrays in HBM.
struct DLayer {
  uint32_t n = 0, nr = 0;
  uint64_t nv = 0;
  const double2* origin = nullptr;   // bbox min per geometry (FP64)
  const double2* ext = nullptr;      // bbox extent per geometry
  const float4* bb = nullptr;        // outward-rounded float bbox (world), the LBVH's leaf boxes
  const uint32_t* gro = nullptr;     // [n+1] geometry -> first ring
  const uint64_t* rvo = nullptr;     // [nr+1] ring -> first vertex (rings closed)
  const double2* xy = nullptr;       // [nv] vertex - origin (points layer: world coordinates)
  const uint32_t* synb = nullptr;    // bit per vertex: edge v -> v+1 made by subdivision (nullable)
  const uint32_t* parent = nullptr;  // piece -> parent geometry (nullable)
  const double* blen = nullptr;      // real boundary length per parent (relate)
  __device__ __forceinline__ int syn(uint64_t i) const { return synb ? (int)((synb[i >> 5] >> (i & 31)) & 1u) : 0; }
  __device__ __forceinline__ uint32_t pid(uint32_t g) const { return parent ? parent[g] : g; }
};

// LBVH node: both children's boxes in the parent (one 48-byte record per internal node). Child >= 0 is an
// internal node, ~child is a leaf's geometry id.
struct __align__(16) BNode {
  float4 lb, rb;
  int l, r, pad0, pad1;
};
struct DBvh {
  const BNode* nodes = nullptr;
  uint32_t n = 0;
  const uint32_t* order = nullptr;   // leaves in Morton order (geometry ids)
};

// ---- exact predicates (restating engine.cuh:283-316) -----------------------------------------------------
__device__ __forceinline__ double orient(double ax, double ay, double bx, double by, double cx, double cy) {
  double a = bx - ax, b = cy - ay, c = by - ay, d = cx - ax;
  double w = c * d;
  double e = fma(-c, d, w);
  double f = fma(a, b, -w);
  return f + e;
}
__device__ __forceinline__ bool onseg(double ax, double ay, double bx, double by, double px, double py) {
  return px >= fmin(ax, bx) && px <= fmax(ax, bx) && py >= fmin(ay, by) && py <= fmax(ay, by);
}
// side of p w.r.t. directed a->b with simulation of simplicity for points on the line (engine.cuh:298-304)
__device__ __forceinline__ bool left_of(double ax, double ay, double bx, double by, double px, double py) {
  double o = orient(ax, ay, bx, by, px, py);
  if (o != 0) return o > 0;
  double dy = by - ay;
  if (dy != 0) return dy < 0;
  return bx > ax;
}
// closed segments intersect (touching counts) (engine.cuh:307-316)
__device__ __forceinline__ bool seg_isect(double p0x, double p0y, double p1x, double p1y, double q0x, double q0y, double q1x, double q1y) {
  double d1 = orient(q0x, q0y, q1x, q1y, p0x, p0y), d2 = orient(q0x, q0y, q1x, q1y, p1x, p1y);
  double d3 = orient(p0x, p0y, p1x, p1y, q0x, q0y), d4 = orient(p0x, p0y, p1x, p1y, q1x, q1y);
  if (((d1 > 0 && d2 < 0) || (d1 < 0 && d2 > 0)) && ((d3 > 0 && d4 < 0) || (d3 < 0 && d4 > 0))) return true;
  if (d1 == 0 && onseg(q0x, q0y, q1x, q1y, p0x, p0y)) return true;
  if (d2 == 0 && onseg(q0x, q0y, q1x, q1y, p1x, p1y)) return true;
  if (d3 == 0 && onseg(p0x, p0y, p1x, p1y, q0x, q0y)) return true;
  if (d4 == 0 && onseg(p0x, p0y, p1x, p1y, q1x, q1y)) return true;
  return false;
}

// ---- FP32 sign filters with certified bounds (the filtered variant's optional first stage) -----------------------
// Sign of orient(a, b, c) exactly as the FP64 routine above computes it. The FP64 differences are rounded to float
// (relative error <= u = 2^-24 each) and det = fa*fb - fc*fd is formed in FP32; |det - (ab - cd)| <= 4.0000005 u
// (|p| + |q|) for the float products p, q (normal floats: |p|, |q| >= 1e-30 with differences below 720 degrees), so
// |det| > 6 u (|p| + |q|) fixes the sign of ab - cd, far outside the FP64 routine's own error (<= 2^-52 (|ab| + |cd|)),
// hence the sign the FP64 routine returns. Otherwise (near-degenerate or exact zeros) the FP64 routine decides.
__device__ __forceinline__ int orient_sign32(double ax, double ay, double bx, double by, double cx, double cy) {
  const double a = bx - ax, b = cy - ay, c = by - ay, d = cx - ax;
  const float p = __double2float_rn(a) * __double2float_rn(b), q = __double2float_rn(c) * __double2float_rn(d);
  const float ap = fabsf(p), aq = fabsf(q);
  if (ap >= 1e-30f && aq >= 1e-30f) {
    const float det = p - q, bound = 3.6e-7f * (ap + aq);
    if (det > bound) return 1;
    if (det < -bound) return -1;
  }
  const double o = orient(ax, ay, bx, by, cx, cy);
  return o > 0 ? 1 : (o < 0 ? -1 : 0);
}
// left_of and seg_isect on the filtered signs: the same booleans as the FP64 forms
__device__ __forceinline__ bool left_of32(double ax, double ay, double bx, double by, double px, double py) {
  const int o = orient_sign32(ax, ay, bx, by, px, py);
  if (o != 0) return o > 0;
  double dy = by - ay;
  if (dy != 0) return dy < 0;
  return bx > ax;
}
__device__ __forceinline__ bool seg_isect32(double p0x, double p0y, double p1x, double p1y, double q0x, double q0y, double q1x, double q1y) {
  const int d1 = orient_sign32(q0x, q0y, q1x, q1y, p0x, p0y), d2 = orient_sign32(q0x, q0y, q1x, q1y, p1x, p1y);
  const int d3 = orient_sign32(p0x, p0y, p1x, p1y, q0x, q0y), d4 = orient_sign32(p0x, p0y, p1x, p1y, q1x, q1y);
  if (d1 * d2 < 0 && d3 * d4 < 0) return true;
  if (d1 == 0 && onseg(q0x, q0y, q1x, q1y, p0x, p0y)) return true;
  if (d2 == 0 && onseg(q0x, q0y, q1x, q1y, p1x, p1y)) return true;
  if (d3 == 0 && onseg(p0x, p0y, p1x, p1y, q0x, q0y)) return true;
  if (d4 == 0 && onseg(p0x, p0y, p1x, p1y, q1x, q1y)) return true;
  return false;
}

// A geometry seen in a pair frame: world = shx + stored x.
struct Frame {
  const DLayer* L; uint32_t r0, r1; double shx, shy;
  __device__ __forceinline__ void v(uint64_t i, double& x, double& y) const {
    double2 q = L->xy[i];
    x = shx + q.x; y = shy + q.y;
  }
};
__device__ __forceinline__ Frame frame_of(const DLayer& S, uint32_t g, double rx, double ry) {
  Frame f; f.L = &S; f.r0 = S.gro[g]; f.r1 = S.gro[g + 1];
  double2 o = S.origin[g];
  f.shx = o.x - rx; f.shy = o.y - ry;
  return f;
}

constexpr uint32_t REL_COIN_SAME = 1;   // real boundaries coincide, interiors on the same side
constexpr uint32_t REL_COIN_OPP = 2;    // real boundaries coincide, interiors on opposite sides
constexpr uint32_t REL_TOUCH = 4;       // real boundaries meet
constexpr int MAXS = 24;                // split points per edge (engine.cuh:339)
constexpr int MAXO = 8;                 // collinear overlap intervals per edge (engine.cuh:340)

// Overlap box of the pair in the frame of A's origin.
struct Box { double x0, y0, x1, y1; };

// Local edge list (SoA; in shared memory for the fast bins, in global scratch for oversized pairs).
// fl: bit 0 = synthetic (cut) edge, bit 1 / bit 2 = start / end vertex is a cut point.
struct EList {
  double* x0; double* y0; double* x1; double* y1; uint32_t* fl;
};

}  // namespace gsj
