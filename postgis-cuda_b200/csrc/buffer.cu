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
__device__ __noinline__ double geog_dist(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y, bool b_is_point) {
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
// 1 / 0, or -1 when a local list exceeded cap (*need = edges required)
__device__ int dw_pair(const DLayer& P, const DLayer& R, uint32_t a, uint32_t b, double d, EList LA, EList LB, int cap, int lane, int* need) {
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
      if (d2 <= dhi * dhi && geog_dist(oa.x + ex0, oa.y + ey0, oa.x + ex1, oa.y + ey1, oa.x + fx0, oa.y + fy0, oa.x + fx1, oa.y + fy1, false) <= d) {
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
constexpr size_t DW_SMEM = (size_t)DW_WARPS * 2 * DW_CAP * DW_EDGE;

__global__ void __launch_bounds__(DW_WARPS * 32) k_dwithin(DLayer P, DLayer R, const uint2* __restrict__ pairs, uint64_t np, double d, int same,
                                                           uint8_t* flag, uint32_t* heavy, unsigned long long* nheavy) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  EList LA = carve(smem + (size_t)wib * 2 * DW_CAP * DW_EDGE, DW_CAP), LB = carve(smem + ((size_t)wib * 2 + 1) * DW_CAP * DW_EDGE, DW_CAP);
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw) {
    const uint2 pr = pairs[p];
    if (same && P.pid(pr.x) == R.pid(pr.y)) { if (lane == 0) flag[p] = 1; continue; }   // pieces of one geometry (buffer.cuh:247-250)
    const int r = dw_pair(P, R, pr.x, pr.y, d, LA, LB, DW_CAP, lane, nullptr);
    if (lane == 0) {
      if (r < 0) { heavy[atomicAdd(nheavy, 1ull)] = (uint32_t)p; flag[p] = 0; }
      else flag[p] = (uint8_t)r;
    }
    __syncwarp();
  }
}
__global__ void __launch_bounds__(128) k_dwithin_scratch(DLayer P, DLayer R, const uint2* __restrict__ pairs, const uint32_t* __restrict__ heavy, uint64_t nh,
                                                        double d, uint8_t* flag, unsigned char* scratch, int cap, int* err) {
  const int lane = threadIdx.x & 31;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned char* base = scratch + w * 2 * (size_t)cap * DW_EDGE;
  EList LA = carve(base, cap), LB = carve(base + (size_t)cap * DW_EDGE, cap);
  for (uint64_t h = w; h < nh; h += nw) {
    const uint32_t p = heavy[h];
    const int r = dw_pair(P, R, pairs[p].x, pairs[p].y, d, LA, LB, cap, lane, nullptr);
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

gsj_join_opts opts_or_default(const gsj_join_opts* o);
uint64_t candidates_for(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper, uint2** out);

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
  if (!c->dw_attr) { GSJ_CK(cudaFuncSetAttribute(k_dwithin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DW_SMEM)); c->dw_attr = 1; }
  PairsOut emit{c, sink, user, &st};
  const uint32_t n = P->d.n;
  const bool whole = !o.batch_q || o.batch_q >= n;
  for (uint32_t q0 = 0, qn; q0 < n; q0 = qn) {
    qn = whole ? n : std::min<uint32_t>(q0 + o.batch_q, n);
    if (!whole && !P->h_parent.empty()) while (qn < n && P->h_parent[qn] == P->h_parent[qn - 1]) qn++;
    if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
    tm.start();
    uint2* pairs = nullptr;
    const uint64_t np = candidates_for(c, qbb, whole ? P->bvh.order : nullptr, q0, qn - q0, R->bvh, o.upper, &pairs);
    st.traverse_ms += tm.stop(); st.candidates += np; st.batches++;
    if (!np) continue;
    tm.start();
    uint8_t* flag = c->flag.as<uint8_t>(np);
    uint32_t* heavy = c->heavy.as<uint32_t>(np);
    unsigned long long* ctr = c->counters.as<unsigned long long>(8);
    int* err = reinterpret_cast<int*>(ctr + 1);
    GSJ_CK(cudaMemsetAsync(ctr, 0, 16, s));
    const int blocks = (int)std::min<uint64_t>((np + DW_WARPS - 1) / DW_WARPS, (uint64_t)c->sm_count * 8);
    k_dwithin<<<blocks, DW_WARPS * 32, DW_SMEM, s>>>(P->d, R->d, pairs, np, d, same, flag, heavy, ctr); c->launches++;
    GSJ_CK(cudaGetLastError());
    unsigned long long* h = c->h_counters.as<unsigned long long>(2);
    GSJ_CK(cudaMemcpyAsync(h, ctr, 16, cudaMemcpyDeviceToHost, s));
    GSJ_CK(cudaStreamSynchronize(s));
    const uint64_t nh = h[0];
    if (nh) {
      const int cap = (int)((std::max<uint32_t>(std::max(P->max_geom_edges, R->max_geom_edges), 1u) + 7u) & ~7u);
      const size_t per = 2 * (size_t)cap * DW_EDGE;
      uint64_t nwarps = std::min<uint64_t>(std::min<uint64_t>(nh, std::max<uint64_t>(1, (1ull << 30) / per)), (uint64_t)c->sm_count * 32);
      nwarps = (nwarps + 3) / 4 * 4;
      unsigned char* scr = c->scratch.as<unsigned char>(per * nwarps);
      k_dwithin_scratch<<<(int)(nwarps / 4), 128, 0, s>>>(P->d, R->d, pairs, heavy, nh, d, flag, scr, cap, err); c->launches++;
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

void erode_host(gsj_ctx*, const gsj_layer*, const gsj_layer*, double, double, int, const uint8_t*, const gsj_join_opts*, gsj_pairs_sink, void*,
                gsj_join_stats*) {
  throw Error(GSJ_ERR_ARG, "erode: not built yet");
}

void points_buffer_host(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, double d, int erode, const gsj_join_opts* op, gsj_pairs_sink sink,
                        void* user, gsj_join_stats* stp) {
  if (!pts->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "a point layer and a polygon layer are needed");
  if (erode) throw Error(GSJ_ERR_ARG, "points erode: not built yet");
  const gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches;
  cudaStream_t s = c->stream;
  Timer tm(s);
  const uint32_t n = pts->d.n;
  const float4* qbb = pts->d.bb;
  if (d > 0) {
    float4* e = c->qbb.as<float4>(n);
    k_expand_points<<<grid_for(n, 256), 256, 0, s>>>(pts->pts, n, d, e); c->launches++;
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
    const uint64_t np = candidates_for(c, qbb, bq == n ? pts->bvh.order : nullptr, q0, nq, R->bvh, 0, &pairs);
    st.traverse_ms += tm.stop(); st.candidates += np; st.batches++;
    if (!np) continue;
    tm.start();
    uint8_t* hit = c->flag.as<uint8_t>(np);
    k_pt_dwithin<<<grid_for(np, 128), 128, 0, s>>>(pts->pts, R->d, pairs, np, d, hit); c->launches++;
    GSJ_CK(cudaGetLastError());
    st.refine_ms += tm.stop();
    tm.start();
    uint2* out = nullptr;
    const uint64_t nu = fold_unique(c, pairs, hit, np, 1, nullptr, R->d.parent, &out);
    st.compact_ms += tm.stop();
    emit(out, nu);
  }
  st.launches = c->launches - l0;
  if (stp) *stp = st;
}

}  // namespace gsj
