// Distance and negative-buffer joins in meters on lon/lat layers, FP64 (the reference's engine/buffer.cuh of
// landstats-us/postgis-cuda):
//   ST_DWithin(a::geography, b::geography, d)                         polygon x polygon, point x polygon
//   ST_Intersects(ST_Buffer(a::geography, -ra), ST_Buffer(b::geography, -rb))  (erosion, no buffers built)
// Distances are measured in a local metric frame per pair; boundary pairs within the frame's error band of d are
// re-decided from the closest points of the great-circle edges and the WGS84 geodesic (Vincenty), as PostGIS does.
// Trigonometric functions are CUDA's (sin, cos, tan, atan, atan2; sqrt is exact).
#include <algorithm>
#include <cub/cub.cuh>
#include "engine.h"
#include "pairkit.cuh"

namespace gsj {

constexpr double WGS84_A = 6378137.0, WGS84_F = 1.0 / 298.257223563, WGS84_E2 = WGS84_F * (2.0 - WGS84_F);
constexpr double DEG = 3.14159265358979323846 / 180.0;

// ---- geodesy (restating buffer.cuh:29-180) --------------------------------------------------------------------
__device__ __forceinline__ void m_per_deg(double lat, double& kx, double& ky) {   // meters per degree of lon / lat
  const double s = sin(lat * DEG), c = cos(lat * DEG);
  const double w2 = 1.0 - WGS84_E2 * s * s, w = sqrt(w2);
  kx = WGS84_A / w * c * DEG;
  ky = WGS84_A * (1.0 - WGS84_E2) / (w2 * w) * DEG;
}
// degrees covering d meters over latitudes [y0, y1], larger (expand) or smaller (shrink)
__device__ void deg_cover(double y0, double y1, double d, bool larger, double& dx, double& dy) {
  if (d <= 0) { dx = dy = 0; return; }
  const double pad = larger ? d / 110000.0 + 1e-9 : 0.0;
  double lo = (y0 - pad <= 0 && y1 + pad >= 0) ? 0.0 : fmin(fabs(y0), fabs(y1)) - pad;
  const double hi = fmin(fmax(fabs(y0), fabs(y1)) + pad, 89.9);
  lo = fmax(lo, 0.0);
  double kxa, kya, kxb, kyb;
  m_per_deg(hi, kxa, kya);
  m_per_deg(lo, kxb, kyb);
  if (larger) { dx = d / kxa * (1 + 1e-6); dy = d / kyb * (1 + 1e-6); }
  else { dx = d / kxb * (1 - 1e-6); dy = d / kya * (1 - 1e-6); }
}
// point scale factor of the UTM zone chosen for a geometry centred at (glon, glat), at (lon, lat)
__device__ double utm_k(double glon, double glat, double lon, double lat) {
  if (glat > 70.0 || glat < -70.0) return 1.0;
  int zone = (int)floor((glon + 180.0) / 6.0);
  if (zone > 59) zone = 59;
  const double lon0 = zone * 6.0 - 177.0;
  const double phi = lat * DEG, c = cos(phi), t = tan(phi), T = t * t;
  const double ep2 = WGS84_E2 / (1.0 - WGS84_E2), C = ep2 * c * c, A = (lon - lon0) * DEG * c, A2 = A * A;
  return 0.9996 * (1.0 + (1.0 + C) * A2 / 2.0 + (5.0 - 4.0 * T + 42.0 * C + 13.0 * C * C - 28.0 * ep2) * A2 * A2 / 24.0 +
                   (61.0 - 148.0 * T + 16.0 * T * T) * A2 * A2 * A2 / 720.0);
}
// geodesic distance on WGS84 by Vincenty's inverse formula, meters
__device__ __noinline__ double vincenty_m(double lon1, double lat1, double lon2, double lat2) {
  const double a = WGS84_A, f = WGS84_F, b = a * (1.0 - f);
  const double L = (lon2 - lon1) * DEG;
  const double U1 = atan((1.0 - f) * tan(lat1 * DEG)), U2 = atan((1.0 - f) * tan(lat2 * DEG));
  const double sU1 = sin(U1), cU1 = cos(U1), sU2 = sin(U2), cU2 = cos(U2);
  double lam = L, sinS = 0, cosS = 1, sig = 0, cos2A = 1, cos2Sm = 0;
  for (int it = 0; it < 64; it++) {
    const double sl = sin(lam), cl = cos(lam);
    const double t1 = cU2 * sl, t2 = cU1 * sU2 - sU1 * cU2 * cl;
    sinS = sqrt(t1 * t1 + t2 * t2);
    if (sinS == 0) return 0.0;
    cosS = sU1 * sU2 + cU1 * cU2 * cl;
    sig = atan2(sinS, cosS);
    const double sinA = cU1 * cU2 * sl / sinS;
    cos2A = 1.0 - sinA * sinA;
    cos2Sm = cos2A != 0 ? cosS - 2.0 * sU1 * sU2 / cos2A : 0.0;
    const double C = f / 16.0 * cos2A * (4.0 + f * (4.0 - 3.0 * cos2A));
    const double prev = lam;
    lam = L + (1.0 - C) * f * sinA * (sig + C * sinS * (cos2Sm + C * cosS * (-1.0 + 2.0 * cos2Sm * cos2Sm)));
    if (fabs(lam - prev) < 1e-14) break;
  }
  const double u2 = cos2A * (a * a - b * b) / (b * b);
  const double A = 1.0 + u2 / 16384.0 * (4096.0 + u2 * (-768.0 + u2 * (320.0 - 175.0 * u2)));
  const double B = u2 / 1024.0 * (256.0 + u2 * (-128.0 + u2 * (74.0 - 47.0 * u2)));
  const double dS = B * sinS * (cos2Sm + B / 4.0 * (cosS * (-1.0 + 2.0 * cos2Sm * cos2Sm) -
                                                    B / 6.0 * cos2Sm * (-3.0 + 4.0 * sinS * sinS) * (-3.0 + 4.0 * cos2Sm * cos2Sm)));
  return b * A * (sig - dS);
}
__device__ __forceinline__ double pt_seg_d2(double px, double py, double ax, double ay, double bx, double by) {
  const double dx = bx - ax, dy = by - ay, l2 = dx * dx + dy * dy;
  double t = l2 > 0 ? ((px - ax) * dx + (py - ay) * dy) / l2 : 0.0;
  t = fmin(1.0, fmax(0.0, t));
  const double qx = ax + t * dx, qy = ay + t * dy;
  return (px - qx) * (px - qx) + (py - qy) * (py - qy);
}
__device__ double seg_seg_d2(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y) {
  double best = pt_seg_d2(a0x, a0y, b0x, b0y, b1x, b1y);
  double d = pt_seg_d2(a1x, a1y, b0x, b0y, b1x, b1y);
  if (d < best) best = d;
  d = pt_seg_d2(b0x, b0y, a0x, a0y, a1x, a1y);
  if (d < best) best = d;
  d = pt_seg_d2(b1x, b1y, a0x, a0y, a1x, a1y);
  if (d < best) best = d;
  return best;
}
struct V3 { double x, y, z; };
__device__ __forceinline__ V3 v3_ll(double lon, double lat) { const double cl = cos(lat); return V3{cl * cos(lon), cl * sin(lon), sin(lat)}; }
__device__ __forceinline__ double v3_dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 v3_norm(V3 a) { const double l = sqrt(v3_dot(a, a)); return l > 0 ? V3{a.x / l, a.y / l, a.z / l} : a; }
__device__ __forceinline__ double v3_ang(V3 a, V3 b) {
  const V3 c{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return atan2(sqrt(v3_dot(c, c)), v3_dot(a, b));
}
// cross product of two nearby points on the sphere without cancellation (PostGIS robust_cross_product)
__device__ __forceinline__ V3 robust_cross(double plon, double plat, double qlon, double qlat) {
  const double lon_qpp = (qlon + plon) / -2.0, lon_qmp = (qlon - plon) / 2.0;
  const double smq = sin(plat - qlat), spq = sin(plat + qlat);
  const double s1 = sin(lon_qpp), s2 = sin(lon_qmp), c1 = cos(lon_qpp), c2 = cos(lon_qmp);
  return V3{smq * s1 * c2 - spq * c1 * s2, smq * c1 * c2 + spq * s1 * s2, cos(plat) * cos(qlat) * sin(qlon - plon)};
}
// angle from p to the great-circle edge s-e (radians) and the closest point
__device__ double arc_pt(double slon, double slat, double elon, double elat, double plon, double plat, double& clon, double& clat) {
  const V3 vs = v3_ll(slon, slat), ve = v3_ll(elon, elat), vp = v3_ll(plon, plat);
  double best = 1e9;
  if (!(slon == elon && slat == elat)) {
    const V3 n = v3_norm(robust_cross(slon, slat, elon, elat));
    const double t = v3_dot(vp, n);
    const V3 k = v3_norm(V3{vp.x - t * n.x, vp.y - t * n.y, vp.z - t * n.z});
    const V3 vc = v3_norm(V3{vs.x + ve.x, vs.y + ve.y, vs.z + ve.z});
    const double ds = v3_dot(vs, vc), dk = v3_dot(k, vc);
    if (dk > ds || fabs(dk - ds) < 2e-16) {
      best = v3_ang(vp, k);
      clat = atan2(k.z, sqrt(k.x * k.x + k.y * k.y)); clon = atan2(k.y, k.x);
    }
  }
  const double d2 = v3_ang(vp, vs), d3 = v3_ang(vp, ve);
  if (d2 < best) { best = d2; clon = slon; clat = slat; }
  if (d3 < best) { best = d3; clon = elon; clat = elat; }
  return best;
}
// geography distance (meters) of edge a from edge b (or from point b0 when b_is_point); degrees in
__device__ __forceinline__ double geog_dist_inl(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y, bool b_is_point) {
  const double R = DEG;
  double p1x, p1y, p2x, p2y, cx = 0, cy = 0;
  double best = arc_pt(a0x * R, a0y * R, a1x * R, a1y * R, b0x * R, b0y * R, cx, cy);
  p1x = cx; p1y = cy; p2x = b0x * R; p2y = b0y * R;
  if (!b_is_point) {
    double d = arc_pt(a0x * R, a0y * R, a1x * R, a1y * R, b1x * R, b1y * R, cx, cy);
    if (d < best) { best = d; p1x = cx; p1y = cy; p2x = b1x * R; p2y = b1y * R; }
    d = arc_pt(b0x * R, b0y * R, b1x * R, b1y * R, a0x * R, a0y * R, cx, cy);
    if (d < best) { best = d; p1x = a0x * R; p1y = a0y * R; p2x = cx; p2y = cy; }
    d = arc_pt(b0x * R, b0y * R, b1x * R, b1y * R, a1x * R, a1y * R, cx, cy);
    if (d < best) { best = d; p1x = a1x * R; p1y = a1y * R; p2x = cx; p2y = cy; }
  }
  return vincenty_m(p1x / R, p1y / R, p2x / R, p2y / R);
}
// Out of line for the kernels that call it rarely; kernels bounded to fewer registers inline geog_dist_inl instead
// (a call would need the callee's 254 registers), and spill in this rare near-threshold path only.
__device__ __noinline__ double geog_dist(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y, bool b_is_point) {
  return geog_dist_inl(a0x, a0y, a1x, a1y, b0x, b0y, b1x, b1y, b_is_point);
}
// half-width of the band around d where the straight-edge frame distance may disagree with geography
__device__ __forceinline__ double geog_band(double d, double rel_frame, double La2, double Lb2, double tl) {
  return d * (rel_frame + 5e-5) + (La2 + Lb2) * tl / (8.0 * 6.3e6) + 1e-9;
}

// box widened by d meters, rounded outward to float (k_expand_bb / k_expand_pts, buffer.cuh:703-715, 1004-1016)
__device__ __forceinline__ float4 expand_box(double x0, double y0, double x1, double y1, double d) {
  double dx, dy; deg_cover(y0, y1, d, true, dx, dy);
  return make_float4(__double2float_rd(x0 - dx), __double2float_rd(y0 - dy), __double2float_ru(x1 + dx), __double2float_ru(y1 + dy));
}
__global__ void k_expand_polys(DLayer P, double d, float4* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P.n) return;
  const double2 o = P.origin[i], e = P.ext[i];
  out[i] = expand_box(o.x, o.y, o.x + e.x, o.y + e.y, d);
}
__global__ void k_expand_points(const double2* __restrict__ pts, uint32_t n, double d, float4* out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 p = pts[i];
  out[i] = expand_box(p.x, p.y, p.x, p.y, d);
}

// ---- ST_DWithin, polygon x polygon: warp per piece pair (dw_pair, buffer.cuh:185-236) ------------------------
// 1 / 0, or -1 when a local list exceeded cap (*need = edges required).
// Q (filtered mode): the edge pairs that pass the box test are found by scanning the na x nb grid 32 cells a wave
// and are tested 32 at a time, one per lane, from a per-warp queue Q (64 entries), so that the warp runs the
// distance tests side by side; the same pairs pass the same box test and "within" is an any-of, so the answer is
// the one of the lane-per-A-edge sweep (Q = false, the reference's scheme).
constexpr int DW_QCAP = 64;
template <bool QUEUED>
__device__ int dw_pair(const DLayer& P, const DLayer& R, uint32_t a, uint32_t b, double d, EList LA, EList LB, int cap, int lane, int* need,
                       uint2* Q) {
  const double2 oa = P.origin[a], ob = R.origin[b], ea = P.ext[a], eb = R.ext[b];
  const double sx = ob.x - oa.x, sy = ob.y - oa.y;
  double gx, gy;
  deg_cover(fmin(oa.y, ob.y), fmax(oa.y + ea.y, ob.y + eb.y), d, true, gx, gy);
  const Box ov{fmax(-gx, sx - gx), fmax(-gy, sy - gy), fmin(ea.x + gx, sx + eb.x + gx), fmin(ea.y + gy, sy + eb.y + gy)};
  if (ov.x0 > ov.x1 || ov.y0 > ov.y1) return 0;
  const Frame A = frame_of(P, a, oa.x, oa.y), B = frame_of(R, b, oa.x, oa.y);
  const int na = collect<false>(A, ov, LA, cap, lane), nb = collect<false>(B, ov, LB, cap, lane);
  if (na > cap || nb > cap) { if (need) *need = max(na, nb); return -1; }
  __syncwarp();
  const double phi0 = oa.y + 0.5 * (ov.y0 + ov.y1);
  double kx, ky; m_per_deg(phi0, kx, ky);
  const double tl = fabs(tan(phi0 * DEG)) + 0.01;
  const double delta = 2.0 * 0.5 * (ov.y1 - ov.y0) * DEG * (tl + 0.04) + 1e-9;
  bool hit = false;
  if constexpr (QUEUED) {
    auto within = [&](uint2 e) {
      const int i = (int)e.x, j = (int)e.y;
      const double ex0 = LA.x0[i], ey0 = LA.y0[i], ex1 = LA.x1[i], ey1 = LA.y1[i];
      const double fx0 = LB.x0[j], fy0 = LB.y0[j], fx1 = LB.x1[j], fy1 = LB.y1[j];
      if (seg_isect(ex0, ey0, ex1, ey1, fx0, fy0, fx1, fy1)) return true;
      const double exm = (ex1 - ex0) * kx, eym = (ey1 - ey0) * ky, La2 = exm * exm + eym * eym;
      const double d2 = seg_seg_d2(ex0 * kx, ey0 * ky, ex1 * kx, ey1 * ky, fx0 * kx, fy0 * ky, fx1 * kx, fy1 * ky);
      const double fxm = (fx1 - fx0) * kx, fym = (fy1 - fy0) * ky;
      const double band = geog_band(d, delta, La2, fxm * fxm + fym * fym, tl);
      const double dlo = d - band, dhi = d + band;
      if (d2 <= dlo * dlo) return true;
      return d2 <= dhi * dhi &&
             geog_dist_inl(oa.x + ex0, oa.y + ey0, oa.x + ex1, oa.y + ey1, oa.x + fx0, oa.y + fy0, oa.x + fx1, oa.y + fy1, false) <= d;
    };
    if (na && nb) {
      const unsigned lt = (1u << lane) - 1;
      const uint64_t tot = (uint64_t)na * (uint64_t)nb;
      const int di = 32 / nb, dj = 32 % nb;
      int i = lane / nb, j = lane % nb, qn = 0;
      for (uint64_t base = 0; base < tot; base += 32) {
        bool c = false;
        if (i < na && !(LA.fl[i] & 1u) && !(LB.fl[j] & 1u)) {
          const double ex0 = LA.x0[i], ey0 = LA.y0[i], ex1 = LA.x1[i], ey1 = LA.y1[i];
          const double bx0 = fmin(ex0, ex1) - gx, bx1 = fmax(ex0, ex1) + gx, by0 = fmin(ey0, ey1) - gy, by1 = fmax(ey0, ey1) + gy;
          c = !out_cmp(LB.x0[j], LB.y0[j], LB.x1[j], LB.y1[j], bx0, by0, bx1, by1);
        }
        const unsigned m = __ballot_sync(0xffffffffu, c);
        if (c) Q[qn + __popc(m & lt)] = make_uint2((unsigned)i, (unsigned)j);
        qn += __popc(m);
        i += di; j += dj;
        if (j >= nb) { j -= nb; i++; }
        if (qn >= 32) {
          __syncwarp();
          if (__any_sync(0xffffffffu, within(Q[lane]))) return 1;
          const int rest = qn - 32;
          const uint2 t = lane < rest ? Q[32 + lane] : make_uint2(0, 0);
          __syncwarp();
          if (lane < rest) Q[lane] = t;
          __syncwarp();
          qn = rest;
        }
      }
      __syncwarp();
      if (__any_sync(0xffffffffu, lane < qn && within(Q[lane]))) return 1;
      __syncwarp();
    }
  } else
  for (int i = lane; i < na && !hit; i += 32) {
    if (LA.fl[i] & 1u) continue;
    const double ex0 = LA.x0[i], ey0 = LA.y0[i], ex1 = LA.x1[i], ey1 = LA.y1[i];
    const double bx0 = fmin(ex0, ex1) - gx, bx1 = fmax(ex0, ex1) + gx, by0 = fmin(ey0, ey1) - gy, by1 = fmax(ey0, ey1) + gy;
    const double exm = (ex1 - ex0) * kx, eym = (ey1 - ey0) * ky, La2 = exm * exm + eym * eym;
    for (int j = 0; j < nb; j++) {
      const double fx0 = LB.x0[j], fy0 = LB.y0[j], fx1 = LB.x1[j], fy1 = LB.y1[j];
      if ((LB.fl[j] & 1u) || out_cmp(fx0, fy0, fx1, fy1, bx0, by0, bx1, by1)) continue;
      if (seg_isect(ex0, ey0, ex1, ey1, fx0, fy0, fx1, fy1)) { hit = true; break; }
      const double d2 = seg_seg_d2(ex0 * kx, ey0 * ky, ex1 * kx, ey1 * ky, fx0 * kx, fy0 * ky, fx1 * kx, fy1 * ky);
      const double fxm = (fx1 - fx0) * kx, fym = (fy1 - fy0) * ky;
      const double band = geog_band(d, delta, La2, fxm * fxm + fym * fym, tl);
      const double dlo = d - band, dhi = d + band;
      if (d2 <= dlo * dlo) { hit = true; break; }
      if (d2 <= dhi * dhi && geog_dist_inl(oa.x + ex0, oa.y + ey0, oa.x + ex1, oa.y + ey1, oa.x + fx0, oa.y + fy0, oa.x + fx1, oa.y + fy1, false) <= d) {
        hit = true; break;
      }
    }
  }
  if (__any_sync(0xffffffffu, hit)) return 1;
  // no boundary within d: within d iff one contains the other (a real vertex of one inside the other piece)
  const double cx = ov.x0 + 0.381966 * (ov.x1 - ov.x0), cy = ov.y0 + 0.414213 * (ov.y1 - ov.y0);
  const bool inB_c = pip_full_warp(B, cx, cy, lane), inA_c = pip_full_warp(A, cx, cy, lane);
  bool h = false;
  for (uint32_t r = A.r0 + lane; r < A.r1 && !h; r += 32) {
    double x, y;
    if (probe_vertex(A, r, x, y) && x >= ov.x0 && x <= ov.x1 && y >= ov.y0 && y <= ov.y1 && inside_from_c<false>(LB, nb, cx, cy, inB_c, x, y)) h = true;
  }
  for (uint32_t r = B.r0 + lane; r < B.r1 && !h; r += 32) {
    double x, y;
    if (probe_vertex(B, r, x, y) && x >= ov.x0 && x <= ov.x1 && y >= ov.y0 && y <= ov.y1 && inside_from_c<false>(LA, na, cx, cy, inA_c, x, y)) h = true;
  }
  return __any_sync(0xffffffffu, h) ? 1 : 0;
}

constexpr int DW_CAP = 128, DW_WARPS = 4;
constexpr size_t DW_EDGE = 4 * sizeof(double) + sizeof(uint32_t);
__host__ __device__ constexpr size_t dw_warp_bytes(size_t cap) { return 2 * cap * DW_EDGE + DW_QCAP * sizeof(uint2); }   // lists, queue
constexpr size_t DW_SMEM = (size_t)DW_WARPS * dw_warp_bytes(DW_CAP);

template <bool QUEUED>
__global__ void __launch_bounds__(DW_WARPS * 32, 4) k_dwithin(DLayer P, DLayer R, const uint2* __restrict__ pairs, uint64_t np, double d, int same,
                                                           uint8_t* flag, uint32_t* heavy, unsigned long long* nheavy) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned char* wbase = smem + (size_t)wib * dw_warp_bytes(DW_CAP);
  EList LA = carve(wbase, DW_CAP), LB = carve(wbase + (size_t)DW_CAP * DW_EDGE, DW_CAP);
  uint2* Q = reinterpret_cast<uint2*>(wbase + 2 * (size_t)DW_CAP * DW_EDGE);
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw) {
    const uint2 pr = pairs[p];
    if (same && P.pid(pr.x) == R.pid(pr.y)) { if (lane == 0) flag[p] = 1; continue; }   // pieces of one geometry (buffer.cuh:247-250)
    const int r = dw_pair<QUEUED>(P, R, pr.x, pr.y, d, LA, LB, DW_CAP, lane, nullptr, Q);
    if (lane == 0) {
      if (r < 0) { heavy[atomicAdd(nheavy, 1ull)] = (uint32_t)p; flag[p] = 0; }
      else flag[p] = (uint8_t)r;
    }
    __syncwarp();
  }
}
template <bool QUEUED>
__global__ void __launch_bounds__(128) k_dwithin_scratch(DLayer P, DLayer R, const uint2* __restrict__ pairs, const uint32_t* __restrict__ heavy, uint64_t nh,
                                                        double d, uint8_t* flag, unsigned char* scratch, int cap, int* err) {
  const int lane = threadIdx.x & 31;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned char* base = scratch + w * dw_warp_bytes((size_t)cap);
  EList LA = carve(base, cap), LB = carve(base + (size_t)cap * DW_EDGE, cap);
  uint2* Q = reinterpret_cast<uint2*>(base + 2 * (size_t)cap * DW_EDGE);
  for (uint64_t h = w; h < nh; h += nw) {
    const uint32_t p = heavy[h];
    const int r = dw_pair<QUEUED>(P, R, pairs[p].x, pairs[p].y, d, LA, LB, cap, lane, nullptr, Q);
    if (lane == 0) { if (r < 0) *err = 1; else flag[p] = (uint8_t)r; }
    __syncwarp();
  }
}

// ---- points: thread per (point, piece) (k_pt_dwithin, buffer.cuh:1019-1055) -------------------------------------
__global__ void k_pt_dwithin(const double2* __restrict__ pts, DLayer R, const uint2* __restrict__ pairs, uint64_t np, double d, uint8_t* hit) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const uint2 pr = pairs[i];
  const double2 pt = pts[pr.x], o = R.origin[pr.y];
  const Frame B = frame_of(R, pr.y, o.x, o.y);
  const double px = pt.x - o.x, py = pt.y - o.y;
  double kx, ky; m_per_deg(pt.y, kx, ky);
  const double gy = d / ky;
  const double tl = fabs(tan(pt.y * DEG)) + 0.01;
  const double delta = 2.0 * gy * DEG * (tl + 0.04) + 1e-9;
  const double ox = B.shx - 1.0;
  bool par = false, h = false;
  for (uint32_t r = B.r0; r < B.r1 && !h; r++) {
    const uint64_t s0 = R.rvo[r], e = R.rvo[r + 1];
    double x0, y0; B.v(s0, x0, y0);
    for (uint64_t j = s0 + 1; j < e && !h; j++) {
      double x1, y1; B.v(j, x1, y1);
      if (!R.syn(j - 1)) {
        const double d2 = pt_seg_d2(px * kx, py * ky, x0 * kx, y0 * ky, x1 * kx, y1 * ky);
        const double ex = (x1 - x0) * kx, ey = (y1 - y0) * ky;
        const double band = geog_band(d, delta, ex * ex + ey * ey, 0.0, tl), dlo = d - band, dhi = d + band;
        if (d2 <= dlo * dlo || (d2 <= dhi * dhi && geog_dist(o.x + x0, o.y + y0, o.x + x1, o.y + y1, pt.x, pt.y, pt.x, pt.y, true) <= d)) h = true;
      }
      if (!((y0 > py) == (y1 > py) && y0 != py && y1 != py)) {
        const bool so = left_of(x0, y0, x1, y1, ox, py), sp = left_of(x0, y0, x1, y1, px, py);
        if (so != sp) {
          const bool su = orient(ox, py, px, py, x0, y0) > 0, sv = orient(ox, py, px, py, x1, y1) > 0;
          if (su != sv) par = !par;
        }
      }
      x0 = x1; y0 = y1;
    }
  }
  hit[i] = (h || par) ? 1 : 0;
}

// The same decision with a warp per (point, piece): lanes take consecutive edges of each ring (coalesced vertex
// loads), each edge evaluated by exactly the code above; "within" is an any-of and the crossing parity an XOR over
// the edges, so the ballots give the thread kernel's answer. A warp stops after the chunk in which some lane found
// an edge within d (the answer is then 1 whatever the parity). The per-point set-up (scales, band) of 32 pairs is
// computed one pair per lane and handed to the warp with shuffles, the same values bit for bit.
__device__ __forceinline__ double shfl_d(double v, int k) { return __shfl_sync(0xffffffffu, v, k); }
__global__ void __launch_bounds__(128, 4) k_pt_dwithin_warp(const double2* __restrict__ pts, DLayer R, const uint2* __restrict__ pairs, uint64_t np,
                                                          double d, uint8_t* hit) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; i0 < np; i0 += nw * 32) {
    uint2 mpr = make_uint2(0, 0);
    double mx = 0, my = 0, mkx = 0, mky = 0, mtl = 0, mdelta = 0;
    if (i0 + lane < np) {
      mpr = pairs[i0 + lane];
      const double2 pt = pts[mpr.x];
      mx = pt.x; my = pt.y;
      m_per_deg(pt.y, mkx, mky);
      const double gy = d / mky;
      mtl = fabs(tan(pt.y * DEG)) + 0.01;
      mdelta = 2.0 * gy * DEG * (mtl + 0.04) + 1e-9;
    }
    const int cnt = np - i0 < 32 ? (int)(np - i0) : 32;
    for (int k = 0; k < cnt; k++) {
      const uint32_t g = __shfl_sync(0xffffffffu, mpr.y, k);
      const double2 pt = make_double2(shfl_d(mx, k), shfl_d(my, k));
      const double kx = shfl_d(mkx, k), ky = shfl_d(mky, k), tl = shfl_d(mtl, k), delta = shfl_d(mdelta, k);
      const double2 o = R.origin[g];
      const Frame B = frame_of(R, g, o.x, o.y);
      const double px = pt.x - o.x, py = pt.y - o.y;
      const double ox = B.shx - 1.0;
      bool par = false, h = false;
      for (uint32_t r = B.r0; r < B.r1; r++) {
        const uint64_t s0 = R.rvo[r], e = R.rvo[r + 1];
        for (uint64_t base = s0 + 1; base < e; base += 32) {
          const uint64_t j = base + lane;
          if (j < e) {
            double x0, y0, x1, y1; B.v(j - 1, x0, y0); B.v(j, x1, y1);
            if (!R.syn(j - 1)) {
              const double d2 = pt_seg_d2(px * kx, py * ky, x0 * kx, y0 * ky, x1 * kx, y1 * ky);
              const double ex = (x1 - x0) * kx, ey = (y1 - y0) * ky;
              const double band = geog_band(d, delta, ex * ex + ey * ey, 0.0, tl), dlo = d - band, dhi = d + band;
              if (d2 <= dlo * dlo || (d2 <= dhi * dhi && geog_dist_inl(o.x + x0, o.y + y0, o.x + x1, o.y + y1, pt.x, pt.y, pt.x, pt.y, true) <= d)) h = true;
            }
            if (!((y0 > py) == (y1 > py) && y0 != py && y1 != py)) {
              const bool so = left_of(x0, y0, x1, y1, ox, py), sp = left_of(x0, y0, x1, y1, px, py);
              if (so != sp) {
                const bool su = orient(ox, py, px, py, x0, y0) > 0, sv = orient(ox, py, px, py, x1, y1) > 0;
                if (su != sv) par = !par;
              }
            }
          }
          if (__any_sync(0xffffffffu, h)) break;
        }
        if (__any_sync(0xffffffffu, h)) break;
      }
      const bool within = __any_sync(0xffffffffu, h);
      const bool inside = (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
      if (lane == 0) hit[i0 + k] = (within || inside) ? 1 : 0;
    }
  }
}

// ---- shared driver pieces ----------------------------------------------------------------------------------------
__global__ void k_flag_keep(const uint8_t* __restrict__ f, uint64_t n, uint8_t want, uint32_t* keep) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep[i] = f[i] == want;
}
__global__ void k_keys_kept(const uint2* __restrict__ pairs, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off, uint64_t n,
                            const uint32_t* parA, const uint32_t* parB, unsigned long long* keys) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  const uint2 p = pairs[i];
  keys[off[i]] = ((unsigned long long)(parA ? parA[p.x] : p.x) << 32) | (parB ? parB[p.y] : p.y);
}
__global__ void k_unique_heads(const unsigned long long* __restrict__ k, uint64_t n, uint32_t* head) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}
__global__ void k_unique_scatter(const unsigned long long* __restrict__ k, const uint32_t* __restrict__ head, const uint32_t* __restrict__ off, uint64_t n,
                                 uint2* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && head[i]) out[off[i]] = make_uint2((uint32_t)(k[i] >> 32), (uint32_t)k[i]);
}

static uint64_t scan_count(gsj_ctx* c, const uint32_t* flags, uint32_t* off, uint64_t n) {
  size_t tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flags, off, (int64_t)n, c->stream));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(c->tmp.get(tb), tb, flags, off, (int64_t)n, c->stream));
  uint32_t* h = c->h_counters.as<uint32_t>(4);
  GSJ_CK(cudaMemcpyAsync(h, off + n - 1, 4, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaMemcpyAsync(h + 1, flags + n - 1, 4, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  return (uint64_t)h[0] + h[1];
}

// (a, b) pairs with flag == want -> unique (parent a, parent b) pairs, sorted; returns count, rows in c->opairs
static uint64_t fold_unique(gsj_ctx* c, const uint2* pairs, const uint8_t* flag, uint64_t np, uint8_t want, const uint32_t* parA, const uint32_t* parB,
                            uint2** out) {
  cudaStream_t s = c->stream;
  uint32_t* keep = c->keep.as<uint32_t>(np);
  uint32_t* off = c->idx.as<uint32_t>(np);
  k_flag_keep<<<grid_for(np, 256), 256, 0, s>>>(flag, np, want, keep); c->launches++;
  const uint64_t nk = scan_count(c, keep, off, np);
  *out = c->opairs.as<uint2>(nk);
  if (!nk) return 0;
  unsigned long long* k1 = c->keys.as<unsigned long long>(nk);
  unsigned long long* k2 = c->keys2.as<unsigned long long>(nk);
  k_keys_kept<<<grid_for(np, 256), 256, 0, s>>>(pairs, keep, off, np, parA, parB, k1); c->launches++;
  size_t tb = 0;
  GSJ_CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, k1, k2, (int64_t)nk, 0, 64, s));
  GSJ_CK(cub::DeviceRadixSort::SortKeys(c->tmp.get(tb), tb, k1, k2, (int64_t)nk, 0, 64, s));
  uint32_t* head = c->misc1.as<uint32_t>(nk);
  uint32_t* hoff = c->misc2.as<uint32_t>(nk);
  k_unique_heads<<<grid_for(nk, 256), 256, 0, s>>>(k2, nk, head); c->launches++;
  const uint64_t nu = scan_count(c, head, hoff, nk);
  k_unique_scatter<<<grid_for(nk, 256), 256, 0, s>>>(k2, head, hoff, nk, *out); c->launches++;
  GSJ_CK(cudaGetLastError());
  return nu;
}

struct PairsOut {
  gsj_ctx* c; gsj_pairs_sink sink; void* user; gsj_join_stats* st;
  void operator()(const uint2* dp, uint64_t n) {
    if (!n) return;
    Timer tm(c->stream);
    tm.start();
    uint32_t* hp = c->h_pairs.as<uint32_t>(2 * n);
    GSJ_CK(cudaMemcpyAsync(hp, dp, n * 8, cudaMemcpyDeviceToHost, c->stream));
    st->copy_ms += tm.stop();
    st->hits += n;
    if (sink && sink(user, hp, n)) throw Error(GSJ_ERR_SINK, "sink stopped the join");
  }
};


void dwithin_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double d, int same, const gsj_join_opts* op, gsj_pairs_sink sink, void* user,
                  gsj_join_stats* stp) {
  if (P->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "gsj_dwithin joins two polygon layers (points: gsj_points_dwithin)");
  if (same && P != R) throw Error(GSJ_ERR_ARG, "same = 1 needs P == R");
  const gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches;
  cudaStream_t s = c->stream;
  Timer tm(s);
  const float4* qbb = P->d.bb;
  if (d > 0) {
    float4* e = c->qbb.as<float4>(P->d.n);
    k_expand_polys<<<grid_for(P->d.n, 256), 256, 0, s>>>(P->d, d, e); c->launches++;
    GSJ_CK(cudaGetLastError());
    qbb = e;
  }
  if (!c->dw_attr) {
    GSJ_CK(cudaFuncSetAttribute(k_dwithin<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DW_SMEM));
    GSJ_CK(cudaFuncSetAttribute(k_dwithin<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DW_SMEM));
    c->dw_attr = 1;
  }
  const bool queued = o.refine_mode != GSJ_REFINE_PLAIN;
  PairsOut emit{c, sink, user, &st};
  const uint32_t n = P->d.n;
  const bool whole = !o.batch_q || o.batch_q >= n;
  const bool morton = whole || P->h_parent.empty();   // batches of a layer without parents: runs of Morton positions
  for (uint32_t q0 = 0, qn; q0 < n; q0 = qn) {
    qn = whole ? n : std::min<uint32_t>(q0 + o.batch_q, n);
    if (!whole && !P->h_parent.empty()) while (qn < n && P->h_parent[qn] == P->h_parent[qn - 1]) qn++;
    if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
    tm.start();
    uint2* pairs = nullptr;
    const uint64_t np = candidates_for(c, qbb, morton ? P->bvh.order : nullptr, q0, qn - q0, R->bvh, o.upper, &pairs);
    st.traverse_ms += tm.stop(); st.candidates += np; st.batches++;
    if (!np) continue;
    tm.start();
    uint8_t* flag = c->flag.as<uint8_t>(np);
    uint32_t* heavy = c->heavy.as<uint32_t>(np);
    unsigned long long* ctr = c->counters.as<unsigned long long>(8);
    int* err = reinterpret_cast<int*>(ctr + 1);
    GSJ_CK(cudaMemsetAsync(ctr, 0, 16, s));
    const int blocks = (int)std::min<uint64_t>((np + DW_WARPS - 1) / DW_WARPS, (uint64_t)c->sm_count * 8);
    if (queued) k_dwithin<true><<<blocks, DW_WARPS * 32, DW_SMEM, s>>>(P->d, R->d, pairs, np, d, same, flag, heavy, ctr);
    else k_dwithin<false><<<blocks, DW_WARPS * 32, DW_SMEM, s>>>(P->d, R->d, pairs, np, d, same, flag, heavy, ctr);
    c->launches++;
    GSJ_CK(cudaGetLastError());
    unsigned long long* h = c->h_counters.as<unsigned long long>(2);
    GSJ_CK(cudaMemcpyAsync(h, ctr, 16, cudaMemcpyDeviceToHost, s));
    GSJ_CK(cudaStreamSynchronize(s));
    const uint64_t nh = h[0];
    if (nh) {
      const int cap = (int)((std::max<uint32_t>(std::max(P->max_geom_edges, R->max_geom_edges), 1u) + 7u) & ~7u);
      const size_t per = dw_warp_bytes((size_t)cap);
      uint64_t nwarps = std::min<uint64_t>(std::min<uint64_t>(nh, std::max<uint64_t>(1, (1ull << 30) / per)), (uint64_t)c->sm_count * 32);
      nwarps = (nwarps + 3) / 4 * 4;
      unsigned char* scr = c->scratch.as<unsigned char>(per * nwarps);
      if (queued) k_dwithin_scratch<true><<<(int)(nwarps / 4), 128, 0, s>>>(P->d, R->d, pairs, heavy, nh, d, flag, scr, cap, err);
      else k_dwithin_scratch<false><<<(int)(nwarps / 4), 128, 0, s>>>(P->d, R->d, pairs, heavy, nh, d, flag, scr, cap, err);
      c->launches++;
      GSJ_CK(cudaGetLastError());
      GSJ_CK(cudaMemcpyAsync(h, ctr, 16, cudaMemcpyDeviceToHost, s));
      GSJ_CK(cudaStreamSynchronize(s));
      if (reinterpret_cast<int*>(h + 1)[0]) throw Error(GSJ_ERR_CUDA, "oversized dwithin pair exceeded the scratch edge capacity");
    }
    st.heavy += nh;
    st.refine_ms += tm.stop();
    tm.start();
    uint2* out = nullptr;
    const uint64_t nu = fold_unique(c, pairs, flag, np, 1, P->d.parent, R->d.parent, &out);
    st.compact_ms += tm.stop();
    emit(out, nu);
  }
  st.launches = c->launches - l0;
  if (stp) *stp = st;
}

// ---- negative-buffer intersects: warp per parent pair (buffer.cuh:275-889) ------------------------------------------
// An element list per side: the eroded boundary lies on the edges offset inward by r and the GEOS-style chord fillets
// at reflex vertices; X_A and X_B meet iff elements cross outside both exclusion zones, or a vertex of one eroded
// boundary lies inside the other eroded polygon. Tested in W = shrink(bbox A, ra) x shrink(bbox B, rb).
struct BEd { double x0, y0, x1, y1, ux, uy, L, ci, si; int succ, vt; };   // real edge in frame meters + end-vertex region
struct BEl { double x0, y0, x1, y1; };                                  // element of the raw offset curve
constexpr double FILLET_QUANTUM = 3.14159265358979323846 / 16.0;       // 8 segments per quarter circle (GEOS default)
constexpr int ER_WARPS = 2, ER_CAPE = 64, ER_CAPL = 128, ER_MAX_DEPTH = 12;
constexpr int ER_QCAP = 64;                                                // crossing candidates queued per warp
constexpr int ER_RUN = 4, ER_RUNS = 64, ER_MINB = 4;   // k_erode_main: pairs per fetch, fetches per warp, blocks per SM
constexpr size_t ER_SMEM_WARP = 2 * ER_CAPE * sizeof(BEd) + 2 * ER_CAPL * sizeof(BEl) + ER_QCAP * sizeof(uint2);
constexpr size_t ER_SMEM = (size_t)ER_WARPS * ER_SMEM_WARP;
struct ErScratch { BEd* EA; BEd* EB; BEl* LA; BEl* LB; uint2* Q; int capE, capL; };
__host__ __device__ constexpr size_t er_scratch_bytes(size_t capE, size_t capL) {
  return 2 * capE * sizeof(BEd) + 2 * capL * sizeof(BEl) + ER_QCAP * sizeof(uint2);
}
struct ETile { uint32_t pair, depth; double4 box; };
struct ErCtr { unsigned int ntile, nslab; int needE, needL; unsigned long long next; };   // next: k_erode_main's pair counter
struct EFrame { double ox, oy, kx, ky; };

__device__ bool in_excl(const BEd* E, int n, double r, double x, double y, double eps) {   // buffer.cuh:285-319
  if (r <= 0) return false;
  const double ri = r - eps;
  for (int k = 0; k < n; k++) {
    const BEd& e = E[k];
    if (x < fmin(e.x0, e.x1) - r || x > fmax(e.x0, e.x1) + r || y < fmin(e.y0, e.y1) - r || y > fmax(e.y0, e.y1) + r) continue;
    const double dx = x - e.x0, dy = y - e.y0;
    const double t = dx * e.ux + dy * e.uy, s = dy * e.ux - dx * e.uy;   // s > 0: interior side
    if (fabs(s) < ri && t > -eps && t < e.L + eps) return true;
    if (e.vt == 0) continue;
    const double vx = x - e.x1, vy = y - e.y1, d2 = vx * vx + vy * vy;
    if (d2 >= r * r) continue;
    const BEd& f = E[e.succ];
    if (e.vt == 1) {
      const double s2 = vy * f.ux - vx * f.uy;
      if (d2 < ri * ri && !(s > eps && s2 > eps)) return true;
      continue;
    }
    const double nkx = -e.uy, nky = e.ux, nsx = -f.uy, nsy = f.ux;
    if (nkx * vy - nky * vx > eps) continue;
    if (nsx * vy - nsy * vx < -eps) continue;
    const double chh = sqrt(0.5 * (1.0 + e.ci)), shh = sqrt(fmax(0.0, 0.5 * (1.0 - e.ci)));
    const double ch = r * chh - eps;
    if (d2 < ch * ch) return true;
    double mx = nkx * chh + nky * shh, my = -nkx * shh + nky * chh;
    bool in = true;
    for (int i = 0, m = e.vt - 1; i < m && in; i++) {
      if (mx * vx + my * vy >= ch) in = false;
      const double t2 = mx * e.ci + my * e.si; my = -mx * e.si + my * e.ci; mx = t2;
    }
    if (in) return true;
  }
  return false;
}
__device__ __forceinline__ bool inside_m(const BEd* E, int n, double cx, double cy, bool in_c, double x, double y) {   // buffer.cuh:322-334
  bool in = in_c;
  const double sx0 = fmin(cx, x), sx1 = fmax(cx, x), sy0 = fmin(cy, y), sy1 = fmax(cy, y);
  for (int k = 0; k < n; k++) {
    const BEd& e = E[k];
    if (fmax(e.x0, e.x1) < sx0 || fmin(e.x0, e.x1) > sx1 || fmax(e.y0, e.y1) < sy0 || fmin(e.y0, e.y1) > sy1) continue;
    const bool sc = left_of(e.x0, e.y0, e.x1, e.y1, cx, cy), sx = left_of(e.x0, e.y0, e.x1, e.y1, x, y);
    if (sc == sx) continue;
    const bool su = orient(cx, cy, x, y, e.x0, e.y0) > 0, sv = orient(cx, cy, x, y, e.x1, e.y1) > 0;
    if (su != sv) in = !in;
  }
  return in;
}
__device__ __forceinline__ void fv(const DLayer& S, double shx, double shy, uint64_t v, const EFrame& F, double& x, double& y) {
  const double2 q = S.xy[v];
  x = (shx + q.x) * F.kx; y = (shy + q.y) * F.ky;
}
// c inside the parent: the piece whose box holds c decides by crossing parity (buffer.cuh:359-381)
__device__ bool pip_parent(const DLayer& S, uint32_t g0, uint32_t g1, const EFrame& F, double cx, double cy, int lane) {
  bool in = false;
  for (uint32_t g = g0; g < g1 && !in; g++) {
    const double2 o = S.origin[g], e = S.ext[g];
    const double bx0 = (o.x - F.ox) * F.kx, by0 = (o.y - F.oy) * F.ky, bx1 = (o.x + e.x - F.ox) * F.kx, by1 = (o.y + e.y - F.oy) * F.ky;
    if (cx < bx0 - 1e-6 || cx > bx1 + 1e-6 || cy < by0 - 1e-6 || cy > by1 + 1e-6) continue;
    const double shx = o.x - F.ox, shy = o.y - F.oy, ox = bx0 - 1.0;
    bool par = false;
    for (uint32_t r = S.gro[g]; r < S.gro[g + 1]; r++) {
      const uint64_t s0 = S.rvo[r], ee = S.rvo[r + 1];
      for (uint64_t j = s0 + 1 + lane; j < ee; j += 32) {
        double x0, y0, x1, y1; fv(S, shx, shy, j - 1, F, x0, y0); fv(S, shx, shy, j, F, x1, y1);
        if ((y0 > cy) == (y1 > cy) && y0 != cy && y1 != cy) continue;
        const bool so = left_of(x0, y0, x1, y1, ox, cy), sc = left_of(x0, y0, x1, y1, cx, cy);
        if (so == sc) continue;
        const bool su = orient(ox, cy, cx, cy, x0, y0) > 0, sv = orient(ox, cy, cx, cy, x1, y1) > 0;
        if (su != sv) par = !par;
      }
    }
    in = (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
  }
  return in;
}
// the parent's real, non-degenerate edges meeting box C, in piece / ring / edge order (buffer.cuh:384-408)
__device__ int collect_side(const DLayer& S, uint32_t g0, uint32_t g1, const EFrame& F, double cx0, double cy0, double cx1, double cy1, BEd* E, int cap,
                            int lane) {
  const unsigned lt = (1u << lane) - 1;
  int cnt = 0;
  for (uint32_t g = g0; g < g1; g++) {
    const double2 o = S.origin[g], ex = S.ext[g];
    if ((o.x + ex.x - F.ox) * F.kx < cx0 || (o.x - F.ox) * F.kx > cx1 || (o.y + ex.y - F.oy) * F.ky < cy0 || (o.y - F.oy) * F.ky > cy1) continue;
    const double shx = o.x - F.ox, shy = o.y - F.oy;
    for (uint32_t r = S.gro[g]; r < S.gro[g + 1]; r++) {
      const uint64_t s0 = S.rvo[r], e = S.rvo[r + 1];
      for (uint64_t base = s0; base + 1 < e; base += 32) {
        const uint64_t i = base + lane;
        bool v = false; BEd ed;
        if (i + 1 < e && !S.syn(i)) {
          fv(S, shx, shy, i, F, ed.x0, ed.y0); fv(S, shx, shy, i + 1, F, ed.x1, ed.y1);
          v = !(ed.x0 == ed.x1 && ed.y0 == ed.y1) &&
              !(fmax(ed.x0, ed.x1) < cx0 || fmin(ed.x0, ed.x1) > cx1 || fmax(ed.y0, ed.y1) < cy0 || fmin(ed.y0, ed.y1) > cy1);
        }
        const unsigned m = __ballot_sync(0xffffffffu, v);
        const int pos = cnt + __popc(m & lt);
        if (v && pos < cap) E[pos] = ed;
        cnt += __popc(m);
      }
    }
  }
  return cnt;
}
// unit directions, successor edge and end-vertex region (convex disk / reflex fillet) (buffer.cuh:411-439)
__device__ void prepare_side(BEd* E, int n, double r, int lane) {
  for (int k = lane; k < n; k += 32) {
    const double dx = E[k].x1 - E[k].x0, dy = E[k].y1 - E[k].y0, L = sqrt(dx * dx + dy * dy);
    E[k].ux = dx / L; E[k].uy = dy / L; E[k].L = L;
  }
  __syncwarp();
  for (int k = lane; k < n; k += 32) {
    const double ex1 = E[k].x1, ey1 = E[k].y1, eux = E[k].ux, euy = E[k].uy;
    int s = -1;
    if (k + 1 < n && E[k + 1].x0 == ex1 && E[k + 1].y0 == ey1) s = k + 1;
    else for (int j = 0; j < n; j++) if (j != k && E[j].x0 == ex1 && E[j].y0 == ey1) { s = j; break; }
    int vt = 0; double ci = 1, si = 0;
    if (s >= 0 && r > 0) {
      const double fux = E[s].ux, fuy = E[s].uy;
      const double cr = eux * fuy - euy * fux, dt = eux * fux + euy * fuy;
      if (cr > 0) vt = 1;
      else if (cr < 0 || dt < 0) {   // right turn or reversal: fillet
        double th = atan2(-cr, dt);
        if (cr == 0) th = 3.14159265358979323846;
        int m = (int)(th / FILLET_QUANTUM + 0.5);
        if (m < 1) m = 1;
        const double inc = th / m; ci = cos(inc); si = sin(inc);
        vt = m + 1;
      }
    }
    E[k].succ = s; E[k].vt = vt; E[k].ci = ci; E[k].si = si;
  }
  __syncwarp();
}
// raw offset curve elements meeting W +- eps (buffer.cuh:442-472)
__device__ int build_elements(const BEd* E, int n, double r, double wx0, double wy0, double wx1, double wy1, double eps, BEl* L, int cap, int lane) {
  const unsigned lt = (1u << lane) - 1;
  int cnt = 0;
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    const bool valid = k < n;
    BEd e; if (valid) e = E[k];
    const int ne = valid ? 1 + (e.vt >= 2 ? e.vt - 1 : 0) : 0;
    const int mx = __reduce_max_sync(0xffffffffu, ne);
    double nkx = 0, nky = 0, wxr = 0, wyr = 0, px = 0, py = 0, nsx = 0, nsy = 0;
    if (valid) {
      nkx = -e.uy; nky = e.ux; wxr = nkx; wyr = nky; px = e.x1 + r * nkx; py = e.y1 + r * nky;
      if (e.vt >= 2) { nsx = -E[e.succ].uy; nsy = E[e.succ].ux; }
    }
    for (int it = 0; it < mx; it++) {
      bool has = it < ne; BEl el;
      if (has) {
        if (it == 0) { el.x0 = e.x0 + r * nkx; el.y0 = e.y0 + r * nky; el.x1 = e.x1 + r * nkx; el.y1 = e.y1 + r * nky; }
        else {
          const double t2 = wxr * e.ci + wyr * e.si; wyr = -wxr * e.si + wyr * e.ci; wxr = t2;
          double qx, qy;
          if (it == ne - 1) { qx = e.x1 + r * nsx; qy = e.y1 + r * nsy; } else { qx = e.x1 + r * wxr; qy = e.y1 + r * wyr; }
          el.x0 = px; el.y0 = py; el.x1 = qx; el.y1 = qy; px = qx; py = qy;
        }
        has = !(fmax(el.x0, el.x1) < wx0 - eps || fmin(el.x0, el.x1) > wx1 + eps || fmax(el.y0, el.y1) < wy0 - eps || fmin(el.y0, el.y1) > wy1 + eps);
      }
      const unsigned m = __ballot_sync(0xffffffffu, has);
      const int pos = cnt + __popc(m & lt);
      if (has && pos < cap) L[pos] = el;
      cnt += __popc(m);
    }
  }
  return cnt;
}
__device__ int seg_points(const BEl& p, const BEl& q, double* xs, double* ys) {   // buffer.cuh:475-493
  const double rx = p.x1 - p.x0, ry = p.y1 - p.y0, sx = q.x1 - q.x0, sy = q.y1 - q.y0;
  const double den = rx * sy - ry * sx;
  if (den != 0) {
    double t = ((q.x0 - p.x0) * sy - (q.y0 - p.y0) * sx) / den;
    t = fmin(1.0, fmax(0.0, t));
    xs[0] = p.x0 + t * rx; ys[0] = p.y0 + t * ry;
    return 1;
  }
  const double l2 = rx * rx + ry * ry;
  if (l2 == 0) { xs[0] = p.x0; ys[0] = p.y0; return 1; }
  const double t0 = ((q.x0 - p.x0) * rx + (q.y0 - p.y0) * ry) / l2, t1 = ((q.x1 - p.x0) * rx + (q.y1 - p.y0) * ry) / l2;
  double lo = fmax(0.0, fmin(t0, t1)), hi = fmin(1.0, fmax(t0, t1));
  if (lo > hi) { const double m = 0.5 * (lo + hi); lo = hi = fmin(1.0, fmax(0.0, m)); }
  xs[0] = p.x0 + lo * rx; ys[0] = p.y0 + lo * ry;
  xs[1] = p.x0 + hi * rx; ys[1] = p.y0 + hi * ry;
  xs[2] = p.x0 + 0.5 * (lo + hi) * rx; ys[2] = p.y0 + 0.5 * (lo + hi) * ry;
  return 3;
}

// X_A meets X_B within the window (intersected with tile when given): 1 / 0, or -1 when a list overflowed
// (needE / needL = sizes required, *wout = the window tested) (buffer.cuh:499-588). mirror: B is A (same layer,
// same pieces, same radius), so B's edge and element lists, centre test and vertex pass are A's and are not
// built twice; every value they would hold is computed from the same inputs by the same code.
__device__ int er_pair(const DLayer& P, const DLayer& R, uint2 ga, uint2 gb, double ra_nom, double rb_nom, const ErScratch& sc, int lane, int* needE,
                       int* needL, const double4* tile, double4* wout, bool mirror) {
  if (ga.x >= ga.y || gb.x >= gb.y) return 0;
  double abx0 = 1e300, aby0 = 1e300, abx1 = -1e300, aby1 = -1e300, bbx0 = 1e300, bby0 = 1e300, bbx1 = -1e300, bby1 = -1e300;
  for (uint32_t g = ga.x; g < ga.y; g++) {
    const double2 o = P.origin[g], e = P.ext[g];
    abx0 = fmin(abx0, o.x); aby0 = fmin(aby0, o.y); abx1 = fmax(abx1, o.x + e.x); aby1 = fmax(aby1, o.y + e.y);
  }
  for (uint32_t g = gb.x; g < gb.y; g++) {
    const double2 o = R.origin[g], e = R.ext[g];
    bbx0 = fmin(bbx0, o.x); bby0 = fmin(bby0, o.y); bbx1 = fmax(bbx1, o.x + e.x); bby1 = fmax(bby1, o.y + e.y);
  }
  double dax, day, dbx, dby;
  deg_cover(aby0, aby1, ra_nom * 0.998, false, dax, day);   // shrink by a lower bound of the true radius
  if (mirror) { dbx = dax; dby = day; } else deg_cover(bby0, bby1, rb_nom * 0.998, false, dbx, dby);
  double wx0 = fmax(abx0 + dax, bbx0 + dbx), wx1 = fmin(abx1 - dax, bbx1 - dbx);
  double wy0 = fmax(aby0 + day, bby0 + dby), wy1 = fmin(aby1 - day, bby1 - dby);
  if (tile) { wx0 = fmax(wx0, tile->x); wy0 = fmax(wy0, tile->y); wx1 = fmin(wx1, tile->z); wy1 = fmin(wy1, tile->w); }
  if (wx0 > wx1 || wy0 > wy1) return 0;
  if (wout) *wout = make_double4(wx0, wy0, wx1, wy1);
  const double clon = 0.5 * (wx0 + wx1), clat = 0.5 * (wy0 + wy1);
  const double rA = ra_nom > 0 ? ra_nom / utm_k(0.5 * (abx0 + abx1), 0.5 * (aby0 + aby1), clon, clat) : 0.0;
  const double rB = mirror ? rA : rb_nom > 0 ? rb_nom / utm_k(0.5 * (bbx0 + bbx1), 0.5 * (bby0 + bby1), clon, clat) : 0.0;
  EFrame F; { const double2 o = P.origin[ga.x]; F.ox = o.x; F.oy = o.y; } m_per_deg(clat, F.kx, F.ky);
  const double Wx0 = (wx0 - F.ox) * F.kx, Wx1 = (wx1 - F.ox) * F.kx, Wy0 = (wy0 - F.oy) * F.ky, Wy1 = (wy1 - F.oy) * F.ky;
  const double ext = fmax(fmax(fabs(Wx0), fabs(Wx1)), fmax(fabs(Wy0), fabs(Wy1))) + fmax(rA, rB);
  const double eps = 1e-9 + 1e-12 * ext;
  const double fe = 1.0 + 2.0 * 0.5 * (wy1 - wy0) * DEG * (fabs(tan(clat * DEG)) + 0.05);
  const double ma = rA * fe + 1e-6, mb = rB * fe + 1e-6;
  const int na = collect_side(P, ga.x, ga.y, F, Wx0 - ma, Wy0 - ma, Wx1 + ma, Wy1 + ma, sc.EA, sc.capE, lane);
  BEd* const EBw = mirror ? sc.EA : sc.EB;
  const int nb = mirror ? na : collect_side(R, gb.x, gb.y, F, Wx0 - mb, Wy0 - mb, Wx1 + mb, Wy1 + mb, EBw, sc.capE, lane);
  if (na > sc.capE || nb > sc.capE) { if (needE) *needE = max(na, nb); return -1; }
  __syncwarp();
  prepare_side(sc.EA, na, rA, lane);
  if (!mirror) prepare_side(EBw, nb, rB, lane);
  const int la = build_elements(sc.EA, na, rA, Wx0, Wy0, Wx1, Wy1, eps, sc.LA, sc.capL, lane);
  const int lb = mirror ? la : build_elements(EBw, nb, rB, Wx0, Wy0, Wx1, Wy1, eps, sc.LB, sc.capL, lane);
  if (la > sc.capL || lb > sc.capL) { if (needE) *needE = max(na, nb); if (needL) *needL = max(la, lb); return -1; }
  __syncwarp();
  const BEd* EA = sc.EA; const BEd* EB = EBw; const BEl* LA = sc.LA; const BEl* LB = mirror ? sc.LA : sc.LB;
  auto inW = [&](double x, double y) { return x >= Wx0 - eps && x <= Wx1 + eps && y >= Wy0 - eps && y <= Wy1 + eps; };
  // (a) the eroded boundaries cross outside both exclusion zones. The la x lb element grid is scanned 32 cells a
  // wave; cells whose boxes overlap are queued and tested 32 at a time, one per lane, so that the warp runs the
  // exclusion tests side by side (the answer is an any-of, so the order of the tests does not change it).
  bool hit = false;
  if (la && lb) {
    const unsigned lt = (1u << lane) - 1;
    uint2* Q = sc.Q;
    auto cross = [&](uint2 e) {
      const BEl p = LA[e.x], q = LB[e.y];
      if (!seg_isect(p.x0, p.y0, p.x1, p.y1, q.x0, q.y0, q.x1, q.y1)) return false;
      double xs[3], ys[3]; const int k = seg_points(p, q, xs, ys);
      for (int t = 0; t < k; t++)
        if (inW(xs[t], ys[t]) && !in_excl(EA, na, rA, xs[t], ys[t], eps) && (mirror || !in_excl(EB, nb, rB, xs[t], ys[t], eps))) return true;
      return false;
    };
    const uint64_t tot = (uint64_t)la * (uint64_t)lb;
    const int di = 32 / lb, dj = 32 % lb;
    int i = lane / lb, j = lane % lb, qn = 0;
    for (uint64_t base = 0; base < tot; base += 32) {
      bool c = false;
      if (i < la) {
        const BEl p = LA[i], q = LB[j];
        c = !(fmax(q.x0, q.x1) < fmin(p.x0, p.x1) || fmin(q.x0, q.x1) > fmax(p.x0, p.x1) || fmax(q.y0, q.y1) < fmin(p.y0, p.y1) ||
              fmin(q.y0, q.y1) > fmax(p.y0, p.y1));
      }
      const unsigned m = __ballot_sync(0xffffffffu, c);
      if (c) Q[qn + __popc(m & lt)] = make_uint2((unsigned)i, (unsigned)j);
      qn += __popc(m);
      i += di; j += dj;
      if (j >= lb) { j -= lb; i++; }
      if (qn >= 32) {
        __syncwarp();
        if (__any_sync(0xffffffffu, cross(Q[lane]))) return 1;
        const int rest = qn - 32;
        const uint2 t = lane < rest ? Q[32 + lane] : make_uint2(0, 0);
        __syncwarp();
        if (lane < rest) Q[lane] = t;
        __syncwarp();
        qn = rest;
      }
    }
    __syncwarp();
    if (__any_sync(0xffffffffu, lane < qn && cross(Q[lane]))) return 1;
    __syncwarp();
  }
  // (b), (c) a vertex of one eroded boundary inside the other eroded polygon
  const double cx = Wx0 + 0.381966 * (Wx1 - Wx0), cy = Wy0 + 0.414213 * (Wy1 - Wy0);
  const bool inA_c = pip_parent(P, ga.x, ga.y, F, cx, cy, lane);
  const bool inB_c = mirror ? inA_c : pip_parent(R, gb.x, gb.y, F, cx, cy, lane);
  for (int side = 0; side < (mirror ? 1 : 2); side++) {
    const BEd* ES = side ? EB : EA; const BEd* EO = side ? EA : EB;
    const BEl* LS = side ? LB : LA;
    const int ns = side ? nb : na, no = side ? na : nb, ls = side ? lb : la;
    const double rs = side ? rB : rA, ro = side ? rA : rB;
    const bool inO_c = side ? inA_c : inB_c;
    auto vio = [&](double x, double y) {
      return inW(x, y) && !in_excl(ES, ns, rs, x, y, eps) && inside_m(EO, no, cx, cy, inO_c, x, y) && !in_excl(EO, no, ro, x, y, eps);
    };
    for (int i = lane; i < ls && !hit; i += 32) {
      const BEl p = LS[i];
      if (vio(p.x0, p.y0) || vio(p.x1, p.y1)) { hit = true; break; }
      const double px0 = fmin(p.x0, p.x1), px1 = fmax(p.x0, p.x1), py0 = fmin(p.y0, p.y1), py1 = fmax(p.y0, p.y1);
      for (int j = i + 1; j < ls && !hit; j++) {
        const BEl q = LS[j];
        if (fmax(q.x0, q.x1) < px0 || fmin(q.x0, q.x1) > px1 || fmax(q.y0, q.y1) < py0 || fmin(q.y0, q.y1) > py1) continue;
        if (!seg_isect(p.x0, p.y0, p.x1, p.y1, q.x0, q.y0, q.x1, q.y1)) continue;
        double xs[3], ys[3]; const int k = seg_points(p, q, xs, ys);
        for (int t = 0; t < k && !hit; t++) if (vio(xs[t], ys[t])) hit = true;
      }
    }
    if (__any_sync(0xffffffffu, hit)) return 1;
  }
  return 0;
}

__device__ __forceinline__ uint2 piece_range(const uint32_t* pf, uint32_t p) { return pf ? make_uint2(pf[p], pf[p + 1]) : make_uint2(p, p + 1); }
__device__ __forceinline__ ErScratch er_smem(unsigned char* raw, int wib) {
  unsigned char* base = raw + (size_t)wib * ER_SMEM_WARP;
  ErScratch sc;
  sc.EA = reinterpret_cast<BEd*>(base); sc.EB = sc.EA + ER_CAPE;
  sc.LA = reinterpret_cast<BEl*>(sc.EB + ER_CAPE); sc.LB = sc.LA + ER_CAPL;
  sc.Q = reinterpret_cast<uint2*>(sc.LB + ER_CAPL);
  sc.capE = ER_CAPE; sc.capL = ER_CAPL;
  return sc;
}
// pf[q] = first piece whose parent is >= q, q in [0, np] (parents non-decreasing)
__global__ void k_piece_first(const uint32_t* __restrict__ parent, uint32_t n, uint32_t np, uint32_t* pf) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = parent[i], lo = i ? parent[i - 1] + 1 : 0;
  for (uint32_t q = lo; q <= p; q++) pf[q] = i;
  if (i == n - 1) for (uint32_t q = p + 1; q <= np; q++) pf[q] = n;
}
// candidate piece pairs that cannot meet after erosion: both whole geometries with disjoint shrunk bboxes
__global__ void k_er_prefilter(DLayer P, DLayer R, const uint2* __restrict__ pairs, uint64_t n, double ra, double rb, uint32_t* keep) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint2 p = pairs[i];
  auto whole = [](const DLayer& S, uint32_t g) {
    if (!S.parent) return true;
    const uint32_t q = S.parent[g];
    return (g == 0 || S.parent[g - 1] != q) && (g + 1 >= S.n || S.parent[g + 1] != q);
  };
  bool k = true;
  if (whole(P, p.x) && whole(R, p.y)) {
    const double2 oa = P.origin[p.x], ea = P.ext[p.x], ob = R.origin[p.y], eb = R.ext[p.y];
    double dax, day, dbx, dby;
    deg_cover(oa.y, oa.y + ea.y, ra * 0.998, false, dax, day);
    deg_cover(ob.y, ob.y + eb.y, rb * 0.998, false, dbx, dby);
    const double wx0 = fmax(oa.x + dax, ob.x + dbx), wx1 = fmin(oa.x + ea.x - dax, ob.x + eb.x - dbx);
    const double wy0 = fmax(oa.y + day, ob.y + dby), wy1 = fmin(oa.y + ea.y - day, ob.y + eb.y - dby);
    k = wx0 <= wx1 && wy0 <= wy1;
  }
  keep[i] = k;
}
__global__ void k_compact_pairs(const uint2* __restrict__ in, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off, uint64_t n, uint2* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && keep[i]) out[off[i]] = in[i];
}
// erosion input: intersecting parent pairs whose overlap area can hold a disk of radius rmin (buffer.cuh:720-738)
__global__ void k_er_filter(const uint2* __restrict__ pr, const double* __restrict__ area, uint64_t n, DLayer P, const uint32_t* pfP, double rmin,
                            int same, const uint8_t* need_self, uint32_t* keep) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint2 p = pr[i];
  bool k = true;
  if (same && p.x == p.y && need_self) k = need_self[p.x] != 0;
  if (k && rmin >= 0) {
    const uint32_t g = pfP ? pfP[p.x] : p.x;
    const double y0 = P.origin[g].y, y1 = y0 + P.ext[g].y;
    const double lat = (y0 <= 0 && y1 >= 0) ? 0.0 : (fabs(y0) < fabs(y1) ? y0 : y1);
    double kx, ky; m_per_deg(lat, kx, ky);
    const double a_m2 = area[i] * kx * ky * 1.001;
    const double r = 0.98 * rmin;
    k = rmin > 0 ? a_m2 >= 3.14159265358979323846 * r * r : area[i] > 0;
  }
  keep[i] = k;
}
__global__ void __launch_bounds__(ER_WARPS * 32) k_erode_main(DLayer P, DLayer R, const uint32_t* pfP, const uint32_t* pfR, const uint2* __restrict__ pairs,
                                                              uint64_t np, double ra, double rb, bool self_layer, uint8_t* flag, uint32_t* heavy,
                                                              unsigned int* nheavy, unsigned long long* next) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const ErScratch sc = er_smem(smem, threadIdx.x >> 5);
  // warps take runs of ER_RUN consecutive pairs from a counter (pair costs vary widely: a fixed stride left most of
  // the GPU idle behind the slowest warps), at most ER_RUNS runs each so that blocks retire
  for (int k = 0; k < ER_RUNS; k++) {
    unsigned long long p0 = 0;
    if (lane == 0) p0 = atomicAdd(next, (unsigned long long)ER_RUN);
    p0 = __shfl_sync(0xffffffffu, p0, 0);
    if (p0 >= np) break;
    const uint64_t p1 = p0 + ER_RUN < np ? p0 + ER_RUN : np;
    for (uint64_t p = p0; p < p1; p++) {
      const uint2 pr = pairs[p];
      const int r = er_pair(P, R, piece_range(pfP, pr.x), piece_range(pfR, pr.y), ra, rb, sc, lane, nullptr, nullptr, nullptr, nullptr,
                            self_layer && pr.x == pr.y);
      if (lane == 0) { flag[p] = r > 0 ? 1 : 0; if (r < 0) heavy[atomicAdd(nheavy, 1u)] = (uint32_t)p; }
      __syncwarp();
    }
  }
}
__global__ void k_tiles_init(const uint32_t* __restrict__ heavy, uint64_t n, ETile* items) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) items[i] = ETile{heavy[i], 0, make_double4(-INFINITY, -INFINITY, INFINITY, INFINITY)};
}
// split an overflowing tile into quadrants while it is larger than the radius, else send it to the slab pass
__device__ void er_overflow(uint32_t p, uint32_t depth, double4 w, double rmax, int ne, int nl, ETile* next, ETile* slab, ErCtr* c) {
  double kx, ky; m_per_deg(0.5 * (w.y + w.w), kx, ky);
  const double ext = fmax((w.z - w.x) * kx, (w.w - w.y) * ky);
  if (depth < ER_MAX_DEPTH && ext > rmax) {
    const double xm = 0.5 * (w.x + w.z), ym = 0.5 * (w.y + w.w);
    const unsigned k = atomicAdd(&c->ntile, 4u);
    next[k] = ETile{p, depth + 1, make_double4(w.x, w.y, xm, ym)};
    next[k + 1] = ETile{p, depth + 1, make_double4(xm, w.y, w.z, ym)};
    next[k + 2] = ETile{p, depth + 1, make_double4(w.x, ym, xm, w.w)};
    next[k + 3] = ETile{p, depth + 1, make_double4(xm, ym, w.z, w.w)};
  } else {
    slab[atomicAdd(&c->nslab, 1u)] = ETile{p, depth, w};
    atomicMax(&c->needE, ne); atomicMax(&c->needL, nl);
  }
}
__global__ void __launch_bounds__(ER_WARPS * 32) k_erode_tiles(DLayer P, DLayer R, const uint32_t* pfP, const uint32_t* pfR, const uint2* __restrict__ pairs,
                                                               const ETile* items, uint64_t ni, double ra, double rb, bool self_layer, uint8_t* flag,
                                                               ETile* next, ETile* slab, ErCtr* c) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31;
  const ErScratch sc = er_smem(smem, threadIdx.x >> 5);
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < ni; i += nw) {
    ETile t = items[i];
    if (flag[t.pair]) continue;   // another tile already found an intersection
    int ne = 0, nl = 0; double4 win = t.box;
    const uint2 pr = pairs[t.pair];
    const int r = er_pair(P, R, piece_range(pfP, pr.x), piece_range(pfR, pr.y), ra, rb, sc, lane, &ne, &nl, &t.box, &win, self_layer && pr.x == pr.y);
    if (lane == 0) {
      if (r > 0) flag[t.pair] = 1;
      else if (r < 0) er_overflow(t.pair, t.depth, win, fmax(ra, rb), ne, nl, next, slab, c);
    }
    __syncwarp();
  }
}
// tiles that cannot usefully be split: per-warp lists in global scratch sized by the reported need
__global__ void k_erode_slab(DLayer P, DLayer R, const uint32_t* pfP, const uint32_t* pfR, const uint2* __restrict__ pairs, const ETile* items, uint64_t ni,
                             double ra, double rb, bool self_layer, uint8_t* flag, unsigned char* scratch, int capE, int capL, ETile* again, ErCtr* c) {
  const int lane = threadIdx.x & 31;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned char* base = scratch + w * er_scratch_bytes(capE, capL);
  ErScratch sc;
  sc.EA = reinterpret_cast<BEd*>(base); sc.EB = sc.EA + capE;
  sc.LA = reinterpret_cast<BEl*>(sc.EB + capE); sc.LB = sc.LA + capL;
  sc.Q = reinterpret_cast<uint2*>(sc.LB + capL);
  sc.capE = capE; sc.capL = capL;
  for (uint64_t i = w; i < ni; i += nw) {
    ETile t = items[i];
    if (flag[t.pair]) continue;
    int ne = 0, nl = 0;
    const uint2 pr = pairs[t.pair];
    const int r = er_pair(P, R, piece_range(pfP, pr.x), piece_range(pfR, pr.y), ra, rb, sc, lane, &ne, &nl, &t.box, nullptr, self_layer && pr.x == pr.y);
    if (lane == 0) {
      if (r > 0) flag[t.pair] = 1;
      else if (r < 0) { again[atomicAdd(&c->nslab, 1u)] = t; atomicMax(&c->needE, ne); atomicMax(&c->needL, nl); }
    }
    __syncwarp();
  }
}

static const uint32_t* piece_first_dev(gsj_ctx* c, const gsj_layer* S, DevBuf& buf) {
  if (!S->d.parent) return nullptr;
  uint32_t* pf = buf.as<uint32_t>((size_t)S->nparent + 1);
  k_piece_first<<<grid_for(S->d.n, 256), 256, 0, c->stream>>>(S->d.parent, S->d.n, S->nparent, pf); c->launches++;
  GSJ_CK(cudaGetLastError());
  return pf;
}

void erode_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double ra, double rb, int same, const uint8_t* need_self_h, const gsj_join_opts* op,
                gsj_pairs_sink sink, void* user, gsj_join_stats* stp) {
  if (P->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "gsj_erode joins two polygon layers (points: gsj_points_erode)");
  if (same && P != R) throw Error(GSJ_ERR_ARG, "same = 1 needs P == R");
  gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches;
  cudaStream_t s = c->stream;
  DevBuf pfPb, pfRb, nsb;
  const uint32_t* pfP = piece_first_dev(c, P, pfPb);
  const uint32_t* pfR = piece_first_dev(c, R, pfRb);
  const uint8_t* need_self = nullptr;
  if (same && need_self_h) {
    uint8_t* d = nsb.as<uint8_t>(P->nparent);
    GSJ_CK(cudaMemcpyAsync(d, need_self_h, P->nparent, cudaMemcpyHostToDevice, s));
    need_self = d;
  }
  if (!c->er_attr) {
    GSJ_CK(cudaFuncSetAttribute(k_erode_main, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ER_SMEM));
    GSJ_CK(cudaFuncSetAttribute(k_erode_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ER_SMEM));
    c->er_attr = 1;
  }
  const double rmin = (ra > 0 && rb > 0) ? std::min(ra, rb) : (ra > 0 || rb > 0 ? 0.0 : -1.0);
  const bool self_layer = P == R && ra == rb;   // a pair (g, g) then erodes one geometry against itself
  RefineArgs rp{1e-12, 1e-7, 1e-11, 1, 0, 0};
  PairsOut emit{c, sink, user, &st};
  PrefilterFn pre;
  if (ra > 0 || rb > 0)
    pre = [&](uint2* pairs, uint64_t n) -> uint64_t {
      uint32_t* keep = c->er_keep.as<uint32_t>(n);
      uint32_t* off = c->er_off.as<uint32_t>(n);
      k_er_prefilter<<<grid_for(n, 256), 256, 0, s>>>(P->d, R->d, pairs, n, ra, rb, keep); c->launches++;
      const uint64_t k = scan_count(c, keep, off, n);
      uint2* tmp = c->er_tmp.as<uint2>(k);
      k_compact_pairs<<<grid_for(n, 256), 256, 0, s>>>(pairs, keep, off, n, tmp); c->launches++;
      GSJ_CK(cudaMemcpyAsync(pairs, tmp, k * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
      GSJ_CK(cudaGetLastError());
      return k;
    };
  Timer tm(s);
  DeviceBatchFn pass2 = [&](const uint2* dp, const double* da, uint64_t n) {
    tm.start();
    uint32_t* keep = c->er_keep.as<uint32_t>(n);
    uint32_t* off = c->er_off.as<uint32_t>(n);
    k_er_filter<<<grid_for(n, 256), 256, 0, s>>>(dp, da, n, P->d, pfP, rmin, same, need_self, keep); c->launches++;
    const uint64_t ne = scan_count(c, keep, off, n);
    if (!ne) { st.compact_ms += tm.stop(); return; }
    uint2* ep = c->er_pairs.as<uint2>(ne);
    k_compact_pairs<<<grid_for(n, 256), 256, 0, s>>>(dp, keep, off, n, ep); c->launches++;
    uint8_t* flag = c->er_flag.as<uint8_t>(ne);
    uint32_t* heavy = c->er_heavy.as<uint32_t>(ne);
    ErCtr* ctr = c->er_ctr.as<ErCtr>(2);
    GSJ_CK(cudaMemsetAsync(ctr, 0, sizeof(ErCtr), s));
    // enough warps to cover every pair with ER_RUNS fetches each, spread over all SMs, whole waves beyond one
    const uint64_t per_block = (uint64_t)ER_WARPS * ER_RUNS * ER_RUN, wave = (uint64_t)c->sm_count * ER_MINB;
    uint64_t cover = (ne + per_block - 1) / per_block;
    if (cover > wave) cover = (cover + wave - 1) / wave * wave;
    const uint64_t spread = std::min<uint64_t>((ne + ER_WARPS * ER_RUN - 1) / (ER_WARPS * ER_RUN), wave);
    const int G = (int)std::min<uint64_t>(std::max(cover, spread), 1u << 30);
    k_erode_main<<<G, ER_WARPS * 32, ER_SMEM, s>>>(P->d, R->d, pfP, pfR, ep, ne, ra, rb, self_layer, flag, heavy, &ctr->ntile, &ctr->next);
    c->launches++;
    GSJ_CK(cudaGetLastError());
    ErCtr h{};
    GSJ_CK(cudaMemcpyAsync(&h, ctr, sizeof(ErCtr), cudaMemcpyDeviceToHost, s));
    GSJ_CK(cudaStreamSynchronize(s));
    const uint64_t nh = h.ntile;
    st.heavy += nh;
    if (nh) {   // overflowing pairs: quadrant tiles of their windows until the lists fit, then slabs
      uint64_t ni = nh;
      ETile* items = c->er_tiles.as<ETile>(ni);
      k_tiles_init<<<grid_for(ni, 256), 256, 0, s>>>(heavy, ni, items); c->launches++;
      for (int round = 0; ni; round++) {
        if (round > 4 * ER_MAX_DEPTH) throw Error(GSJ_ERR_CUDA, "erosion tiling did not converge");
        ETile* next = c->er_tiles2.as<ETile>(ni * 4);
        ETile* slab = c->er_slab.as<ETile>(ni);
        GSJ_CK(cudaMemsetAsync(ctr, 0, sizeof(ErCtr), s));
        const int GT = (int)std::min<uint64_t>((ni * 32 + 63) / 64, (uint64_t)c->sm_count * 32);
        k_erode_tiles<<<GT, ER_WARPS * 32, ER_SMEM, s>>>(P->d, R->d, pfP, pfR, ep, items, ni, ra, rb, self_layer, flag, next, slab, ctr); c->launches++;
        GSJ_CK(cudaGetLastError());
        ErCtr hc{};
        GSJ_CK(cudaMemcpyAsync(&hc, ctr, sizeof(ErCtr), cudaMemcpyDeviceToHost, s));
        GSJ_CK(cudaStreamSynchronize(s));
        uint64_t ns = hc.nslab;
        for (int sround = 0; ns; sround++) {
          if (sround >= 4) throw Error(GSJ_ERR_CUDA, "erosion slab tiles still overflow after 4 rounds");
          const int capE = std::max<int>(hc.needE, ER_CAPE), capL = std::max<int>(std::max<int>(hc.needL, 17 * capE / 4), ER_CAPL);
          const size_t per = er_scratch_bytes(capE, capL);
          uint64_t nwarps = std::max<uint64_t>(1, std::min<uint64_t>(ns, (1ull << 30) / per));
          nwarps = (nwarps + 3) / 4 * 4;
          unsigned char* scr = c->er_scr.as<unsigned char>(per * nwarps);
          // ping-pong between er_again and er_tiles (this round's tiles are consumed by now)
          ETile* again = (sround % 2 ? c->er_tiles : c->er_again).as<ETile>(ns);
          GSJ_CK(cudaMemsetAsync(ctr, 0, sizeof(ErCtr), s));
          k_erode_slab<<<(int)(nwarps / 4), 128, 0, s>>>(P->d, R->d, pfP, pfR, ep, slab, ns, ra, rb, self_layer, flag, scr, capE, capL, again, ctr); c->launches++;
          GSJ_CK(cudaGetLastError());
          ErCtr h2{};
          GSJ_CK(cudaMemcpyAsync(&h2, ctr, sizeof(ErCtr), cudaMemcpyDeviceToHost, s));
          GSJ_CK(cudaStreamSynchronize(s));
          slab = again; ns = h2.nslab; hc.needE = h2.needE; hc.needL = h2.needL;
        }
        std::swap(c->er_tiles.p, c->er_tiles2.p); std::swap(c->er_tiles.cap, c->er_tiles2.cap);
        items = reinterpret_cast<ETile*>(c->er_tiles.p);
        ni = hc.ntile;
      }
    }
    st.refine_ms += tm.stop();
    tm.start();
    uint2* out = nullptr;
    const uint64_t nu = fold_unique(c, ep, flag, ne, 1, nullptr, nullptr, &out);
    st.compact_ms += tm.stop();
    emit(out, nu);
  };
  join_device(c, P, R, rp, o, st, pre, pass2);
  st.launches = c->launches - l0;
  if (stp) *stp = st;
}

// ---- points in eroded polygons: thread per (point, piece) (k_pt_erode, buffer.cuh:1059-1132) ------------------------
__device__ bool vertex_excl(double ex, double ey, double fx, double fy, double r, double wx, double wy, double eps) {
  const double d2 = wx * wx + wy * wy;
  if (d2 >= r * r) return false;
  const double cr = ex * fy - ey * fx, dt = ex * fx + ey * fy;
  if (cr > 0) {
    const double ri = r - eps, s1 = wy * ex - wx * ey, s2 = wy * fx - wx * fy;
    return d2 < ri * ri && !(s1 > eps && s2 > eps);
  }
  if (cr == 0 && dt >= 0) return false;
  const double th = cr == 0 ? 3.14159265358979323846 : atan2(-cr, dt);
  int m = (int)(th / FILLET_QUANTUM + 0.5);
  if (m < 1) m = 1;
  const double inc = th / m, ci = cos(inc), si = sin(inc);
  const double nkx = -ey, nky = ex, nsx = -fy, nsy = fx;
  if (nkx * wy - nky * wx > eps || nsx * wy - nsy * wx < -eps) return false;
  const double chh = sqrt(0.5 * (1.0 + ci)), shh = sqrt(fmax(0.0, 0.5 * (1.0 - ci)));
  const double ch = r * chh - eps;
  if (d2 < ch * ch) return true;
  double mx = nkx * chh + nky * shh, my = -nkx * shh + nky * chh;
  for (int i = 0; i < m; i++) {
    if (mx * wx + my * wy >= ch) return false;
    const double t2 = mx * ci + my * si; my = -mx * si + my * ci; mx = t2;
  }
  return true;
}
// bit 1 = inside the piece, bit 2 = within r of its real boundary (OR-ed per (point, parent); kept iff == 1)
__global__ void k_pt_erode(const double2* __restrict__ pts, DLayer R, const uint2* __restrict__ pairs, uint64_t np, double r_nom, uint8_t* bits) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const uint2 pr = pairs[i];
  const uint32_t g = pr.y;
  const double2 pt = pts[pr.x], o = R.origin[g], ext = R.ext[g];
  const double r = r_nom / utm_k(o.x + 0.5 * ext.x, o.y + 0.5 * ext.y, pt.x, pt.y);
  double kx, ky; m_per_deg(pt.y, kx, ky);
  const double eps = 1e-9;
  const double shx = o.x - pt.x, shy = o.y - pt.y, ox = shx * kx - 1.0;   // frame: meters relative to the point
  auto vx = [&](uint64_t j, double& x, double& y) { const double2 q = R.xy[j]; x = (shx + q.x) * kx; y = (shy + q.y) * ky; };
  bool par = false, ex = false;
  for (uint32_t rr = R.gro[g]; rr < R.gro[g + 1] && !ex; rr++) {
    const uint64_t s0 = R.rvo[rr], e = R.rvo[rr + 1];
    if (e - s0 < 2) continue;
    bool pv = false; double pux = 0, puy = 0;   // previous real edge direction (the ring closes)
    {
      const uint64_t j = e - 2;
      if (!R.syn(j)) {
        double a, b, c2, dd; vx(j, a, b); vx(j + 1, c2, dd);
        const double L = hypot(c2 - a, dd - b);
        if (L > 0) { pv = true; pux = (c2 - a) / L; puy = (dd - b) / L; }
      }
    }
    double x0, y0; vx(s0, x0, y0);
    for (uint64_t j = s0; j + 1 < e && !ex; j++) {
      double x1, y1; vx(j + 1, x1, y1);
      if (!((y0 > 0) == (y1 > 0) && y0 != 0 && y1 != 0)) {
        const bool so = left_of(x0, y0, x1, y1, ox, 0.0), sp = left_of(x0, y0, x1, y1, 0.0, 0.0);
        if (so != sp) {
          const bool su = orient(ox, 0.0, 0.0, 0.0, x0, y0) > 0, sv = orient(ox, 0.0, 0.0, 0.0, x1, y1) > 0;
          if (su != sv) par = !par;
        }
      }
      const double L = hypot(x1 - x0, y1 - y0);
      if (R.syn(j) || L == 0) { if (R.syn(j)) pv = false; x0 = x1; y0 = y1; continue; }
      const double ux = (x1 - x0) / L, uy = (y1 - y0) / L;
      if (r > 0) {
        const double t = -x0 * ux - y0 * uy, s = -y0 * ux + x0 * uy;
        if (fabs(s) < r - eps && t > -eps && t < L + eps) ex = true;
        else if (pv && vertex_excl(pux, puy, ux, uy, r, -x0, -y0, eps)) ex = true;
      }
      pv = true; pux = ux; puy = uy;
      x0 = x1; y0 = y1;
    }
  }
  bits[i] = ex ? 2 : (par ? 1 : 0);
}
// The same decision with a warp per (point, piece): lanes take consecutive edges of each ring. The exclusion test
// of an edge reads the direction of the last earlier real edge of the ring with non-zero length (cut edges clear
// it, zero-length edges leave it, the ring starts from its closing edge's): a lane finds the nearest earlier lane
// whose edge is a cut or a real one with a ballot, takes that lane's state by shuffle, or the state carried from the
// previous chunk, so every edge sees the state the sequential walk gives it. "Excluded" is an any-of (it decides 2
// whatever the parity), the crossing parity an XOR. The set-up of 32 pairs is computed one pair per lane.
__global__ void __launch_bounds__(128) k_pt_erode_warp(const double2* __restrict__ pts, DLayer R, const uint2* __restrict__ pairs, uint64_t np,
                                                        double r_nom, uint8_t* bits) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i0 = (((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; i0 < np; i0 += nw * 32) {
    uint32_t mg = 0;
    double mx = 0, my = 0, mr = 0, mkx = 0, mky = 0;
    if (i0 + lane < np) {
      const uint2 pr = pairs[i0 + lane];
      const double2 pt = pts[pr.x], o = R.origin[pr.y], ext = R.ext[pr.y];
      mg = pr.y; mx = pt.x; my = pt.y;
      mr = r_nom / utm_k(o.x + 0.5 * ext.x, o.y + 0.5 * ext.y, pt.x, pt.y);
      m_per_deg(pt.y, mkx, mky);
    }
    const int cnt = np - i0 < 32 ? (int)(np - i0) : 32;
    for (int k = 0; k < cnt; k++) {
      const uint32_t g = __shfl_sync(0xffffffffu, mg, k);
      const double ptx = __shfl_sync(0xffffffffu, mx, k), pty = __shfl_sync(0xffffffffu, my, k);
      const double r = __shfl_sync(0xffffffffu, mr, k), kx = __shfl_sync(0xffffffffu, mkx, k), ky = __shfl_sync(0xffffffffu, mky, k);
      const double2 o = R.origin[g];
      const double eps = 1e-9;
      const double shx = o.x - ptx, shy = o.y - pty, ox = shx * kx - 1.0;   // frame: meters relative to the point
      auto vx = [&](uint64_t j, double& x, double& y) { const double2 q = R.xy[j]; x = (shx + q.x) * kx; y = (shy + q.y) * ky; };
      bool par = false, ex = false;
      for (uint32_t rr = R.gro[g]; rr < R.gro[g + 1]; rr++) {
        const uint64_t s0 = R.rvo[rr], e = R.rvo[rr + 1];
        if (e - s0 < 2) continue;
        bool cpv = false; double cux = 0, cuy = 0;   // state carried into the chunk: the ring's closing edge first
        {
          const uint64_t j = e - 2;
          if (!R.syn(j)) {
            double a, b, c2, dd; vx(j, a, b); vx(j + 1, c2, dd);
            const double L = hypot(c2 - a, dd - b);
            if (L > 0) { cpv = true; cux = (c2 - a) / L; cuy = (dd - b) / L; }
          }
        }
        for (uint64_t base = s0; base + 1 < e; base += 32) {
          const uint64_t j = base + lane;
          const bool valid = j + 1 < e;
          double x0 = 0, y0 = 0, x1 = 0, y1 = 0, L = 0, ux = 0, uy = 0;
          bool syn = false;
          if (valid) {
            vx(j, x0, y0); vx(j + 1, x1, y1);
            if (!((y0 > 0) == (y1 > 0) && y0 != 0 && y1 != 0)) {
              const bool so = left_of(x0, y0, x1, y1, ox, 0.0), sp = left_of(x0, y0, x1, y1, 0.0, 0.0);
              if (so != sp) {
                const bool su = orient(ox, 0.0, 0.0, 0.0, x0, y0) > 0, sv = orient(ox, 0.0, 0.0, 0.0, x1, y1) > 0;
                if (su != sv) par = !par;
              }
            }
            L = hypot(x1 - x0, y1 - y0);
            syn = R.syn(j);
            if (!syn && L != 0) { ux = (x1 - x0) / L; uy = (y1 - y0) / L; }
          }
          const bool real = valid && !syn && L != 0, marker = valid && (syn || L != 0);
          const unsigned mk = __ballot_sync(0xffffffffu, marker);
          // the state before this lane's edge: the nearest earlier marker lane, else the carried state
          const unsigned before = mk & lt;
          const int src = before ? 31 - __clz(before) : lane;
          const bool spv = __shfl_sync(0xffffffffu, (int)real, src) != 0;
          const double sux = __shfl_sync(0xffffffffu, ux, src), suy = __shfl_sync(0xffffffffu, uy, src);
          const bool pv = before ? spv : cpv;
          const double pux = before ? sux : cux, puy = before ? suy : cuy;
          if (real && r > 0) {
            const double t = -x0 * ux - y0 * uy, sd = -y0 * ux + x0 * uy;
            if (fabs(sd) < r - eps && t > -eps && t < L + eps) ex = true;
            else if (pv && vertex_excl(pux, puy, ux, uy, r, -x0, -y0, eps)) ex = true;
          }
          if (mk) {   // carry the last marker's state into the next chunk
            const int last = 31 - __clz(mk);
            cpv = __shfl_sync(0xffffffffu, (int)real, last) != 0;
            cux = __shfl_sync(0xffffffffu, ux, last);
            cuy = __shfl_sync(0xffffffffu, uy, last);
          }
          if (__any_sync(0xffffffffu, ex)) break;
        }
        if (__any_sync(0xffffffffu, ex)) break;
      }
      const bool excl = __any_sync(0xffffffffu, ex);
      const bool inside = (__popc(__ballot_sync(0xffffffffu, par)) & 1) != 0;
      if (lane == 0) bits[i0 + k] = excl ? 2 : (inside ? 1 : 0);
    }
  }
}
// (point, parent) keys of every candidate with its bits
__global__ void k_pt_keys(const uint2* __restrict__ pairs, uint64_t n, const uint32_t* parR, unsigned long long* keys) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = ((unsigned long long)pairs[i].x << 32) | (parR ? parR[pairs[i].y] : pairs[i].y);
}
__global__ void k_or_fold(const unsigned long long* __restrict__ k, const uint8_t* __restrict__ v, const uint32_t* __restrict__ head,
                          const uint32_t* __restrict__ hoff, uint64_t n, uint32_t* keep_seg, uint2* seg_pair) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !head[i]) return;
  uint8_t o = 0;
  for (uint64_t j = i; j < n && (j == i || !head[j]); j++) o |= v[j];
  const uint32_t s = hoff[i];
  keep_seg[s] = o == 1;
  seg_pair[s] = make_uint2((uint32_t)(k[i] >> 32), (uint32_t)k[i]);
}

void points_buffer_host(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, double d, int erode, const gsj_join_opts* op, gsj_pairs_sink sink,
                        void* user, gsj_join_stats* stp) {
  if (!pts->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "a point layer and a polygon layer are needed");
  const gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches;
  cudaStream_t s = c->stream;
  Timer tm(s);
  const uint32_t n = pts->d.n;
  const float4* qbb = pts->d.bb;
  const double grow = erode ? d * 1.002 : d;   // erode: every piece whose boundary may be within r of the point
  if (grow > 0) {
    float4* e = c->qbb.as<float4>(n);
    k_expand_points<<<grid_for(n, 256), 256, 0, s>>>(pts->pts, n, grow, e); c->launches++;
    GSJ_CK(cudaGetLastError());
    qbb = e;
  }
  PairsOut emit{c, sink, user, &st};
  const uint32_t bq = (o.batch_q && o.batch_q < n) ? o.batch_q : n;
  for (uint32_t q0 = 0; q0 < n; q0 += bq) {
    if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
    const uint32_t nq = std::min(bq, n - q0);
    tm.start();
    uint2* pairs = nullptr;
    const uint64_t np = candidates_for(c, qbb, pts->bvh.order, q0, nq, R->bvh, 0, &pairs);   // runs of Morton positions
    st.traverse_ms += tm.stop(); st.candidates += np; st.batches++;
    if (!np) continue;
    tm.start();
    uint8_t* hit = c->flag.as<uint8_t>(np);
    if (erode && o.refine_mode == GSJ_REFINE_PLAIN) { k_pt_erode<<<grid_for(np, 128), 128, 0, s>>>(pts->pts, R->d, pairs, np, d, hit); c->launches++; }
    else if (erode) {
      const int G = (int)std::min<uint64_t>((np + 127) / 128, (uint64_t)c->sm_count * 16);   // a warp per 32 pairs
      k_pt_erode_warp<<<G, 128, 0, s>>>(pts->pts, R->d, pairs, np, d, hit); c->launches++;
    }
    else if (o.refine_mode == GSJ_REFINE_PLAIN) { k_pt_dwithin<<<grid_for(np, 128), 128, 0, s>>>(pts->pts, R->d, pairs, np, d, hit); c->launches++; }
    else {
      const int G = (int)std::min<uint64_t>((np + 127) / 128, (uint64_t)c->sm_count * 16);   // a warp per 32 pairs
      k_pt_dwithin_warp<<<G, 128, 0, s>>>(pts->pts, R->d, pairs, np, d, hit); c->launches++;
    }
    GSJ_CK(cudaGetLastError());
    st.refine_ms += tm.stop();
    tm.start();
    uint2* out = nullptr;
    uint64_t nu = 0;
    if (!erode) nu = fold_unique(c, pairs, hit, np, 1, nullptr, R->d.parent, &out);
    else {   // OR the bits per (point, parent): inside some piece and near no real boundary (== 1)
      unsigned long long* k1 = c->keys.as<unsigned long long>(np);
      unsigned long long* k2 = c->keys2.as<unsigned long long>(np);
      uint8_t* v2 = reinterpret_cast<uint8_t*>(c->misc3.as<uint32_t>(np / 4 + 1));
      k_pt_keys<<<grid_for(np, 256), 256, 0, s>>>(pairs, np, R->d.parent, k1); c->launches++;
      size_t tb = 0;
      GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, hit, v2, (int64_t)np, 0, 64, s));
      GSJ_CK(cub::DeviceRadixSort::SortPairs(c->tmp.get(tb), tb, k1, k2, hit, v2, (int64_t)np, 0, 64, s));
      uint32_t* head = c->misc1.as<uint32_t>(np);
      uint32_t* hoff = c->misc2.as<uint32_t>(np);
      k_unique_heads<<<grid_for(np, 256), 256, 0, s>>>(k2, np, head); c->launches++;
      const uint64_t nseg = scan_count(c, head, hoff, np);
      uint32_t* keep = c->keep.as<uint32_t>(nseg);
      uint2* segp = c->agg_flag.as<uint2>(nseg);
      k_or_fold<<<grid_for(np, 256), 256, 0, s>>>(k2, v2, head, hoff, np, keep, segp); c->launches++;
      uint32_t* off = c->idx.as<uint32_t>(nseg);
      nu = scan_count(c, keep, off, nseg);
      out = c->opairs.as<uint2>(nu);
      k_compact_pairs<<<grid_for(nseg, 256), 256, 0, s>>>(segp, keep, off, nseg, out); c->launches++;
      GSJ_CK(cudaGetLastError());
    }
    st.compact_ms += tm.stop();
    emit(out, nu);
  }
  st.launches = c->launches - l0;
  if (stp) *stp = st;
}

}  // namespace gsj
