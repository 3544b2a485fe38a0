/* CPU FP64 oracle, distance and erosion joins - TEST INFRASTRUCTURE ONLY (see oracle.h).
 * Restates engine/buffer.cuh of landstats-us/postgis-cuda (line numbers cited per function). The trigonometric
 * functions are glibc's; the CUDA engine calls CUDA's, so geodesic values can differ in the last bits and a
 * decision within that distance of its threshold can flip (the tests count such flips). */
#include "oracle.h"
#include "oracle_internal.h"

using namespace orc;

namespace {

constexpr double WGS84_A = 6378137.0, WGS84_F = 1.0 / 298.257223563, WGS84_E2 = WGS84_F * (2.0 - WGS84_F);   // buffer.cuh:29
constexpr double DEG = M_PI / 180.0;

// meters per degree of longitude / latitude at latitude lat (buffer.cuh:33-38)
inline void m_per_deg(double lat, double& kx, double& ky) {
  double s = std::sin(lat * DEG), c = std::cos(lat * DEG);
  double w2 = 1.0 - WGS84_E2 * s * s, w = std::sqrt(w2);
  kx = WGS84_A / w * c * DEG;
  ky = WGS84_A * (1.0 - WGS84_E2) / (w2 * w) * DEG;
}
// degrees covering d meters over latitudes [y0, y1] (buffer.cuh:41-52)
inline void deg_cover(double y0, double y1, double d, bool larger, double& dx, double& dy) {
  if (d <= 0) { dx = dy = 0; return; }
  double pad = larger ? d / 110000.0 + 1e-9 : 0.0;
  double lo = (y0 - pad <= 0 && y1 + pad >= 0) ? 0.0 : std::fmin(std::fabs(y0), std::fabs(y1)) - pad;
  double hi = std::fmin(std::fmax(std::fabs(y0), std::fabs(y1)) + pad, 89.9);
  lo = std::fmax(lo, 0.0);
  double kxa, kya, kxb, kyb;
  m_per_deg(hi, kxa, kya);
  m_per_deg(lo, kxb, kyb);
  if (larger) { dx = d / kxa * (1 + 1e-6); dy = d / kyb * (1 + 1e-6); }
  else { dx = d / kxb * (1 - 1e-6); dy = d / kya * (1 - 1e-6); }
}
// UTM point scale factor of the zone _ST_BestSRID picks (buffer.cuh:56-65)
inline double utm_k(double glon, double glat, double lon, double lat) {
  if (glat > 70.0 || glat < -70.0) return 1.0;
  int zone = (int)std::floor((glon + 180.0) / 6.0);
  if (zone > 59) zone = 59;
  double lon0 = zone * 6.0 - 177.0;
  double phi = lat * DEG, c = std::cos(phi), t = std::tan(phi), T = t * t;
  double ep2 = WGS84_E2 / (1.0 - WGS84_E2), C = ep2 * c * c, A = (lon - lon0) * DEG * c, A2 = A * A;
  return 0.9996 * (1.0 + (1.0 + C) * A2 / 2.0 + (5.0 - 4.0 * T + 42.0 * C + 13.0 * C * C - 28.0 * ep2) * A2 * A2 / 24.0 +
                   (61.0 - 148.0 * T + 16.0 * T * T) * A2 * A2 * A2 / 720.0);
}
// Vincenty inverse on WGS84, meters (buffer.cuh:68-95)
inline double vincenty_m(double lon1, double lat1, double lon2, double lat2) {
  const double a = WGS84_A, f = WGS84_F, b = a * (1.0 - f);
  double L = (lon2 - lon1) * DEG;
  double U1 = std::atan((1.0 - f) * std::tan(lat1 * DEG)), U2 = std::atan((1.0 - f) * std::tan(lat2 * DEG));
  double sU1 = std::sin(U1), cU1 = std::cos(U1), sU2 = std::sin(U2), cU2 = std::cos(U2);
  double lam = L, sinS = 0, cosS = 1, sig = 0, cos2A = 1, cos2Sm = 0;
  for (int it = 0; it < 64; it++) {
    double sl = std::sin(lam), cl = std::cos(lam);
    double t1 = cU2 * sl, t2 = cU1 * sU2 - sU1 * cU2 * cl;
    sinS = std::sqrt(t1 * t1 + t2 * t2);
    if (sinS == 0) return 0.0;
    cosS = sU1 * sU2 + cU1 * cU2 * cl;
    sig = std::atan2(sinS, cosS);
    double sinA = cU1 * cU2 * sl / sinS;
    cos2A = 1.0 - sinA * sinA;
    cos2Sm = cos2A != 0 ? cosS - 2.0 * sU1 * sU2 / cos2A : 0.0;
    double C = f / 16.0 * cos2A * (4.0 + f * (4.0 - 3.0 * cos2A));
    double prev = lam;
    lam = L + (1.0 - C) * f * sinA * (sig + C * sinS * (cos2Sm + C * cosS * (-1.0 + 2.0 * cos2Sm * cos2Sm)));
    if (std::fabs(lam - prev) < 1e-14) break;
  }
  double u2 = cos2A * (a * a - b * b) / (b * b);
  double A = 1.0 + u2 / 16384.0 * (4096.0 + u2 * (-768.0 + u2 * (320.0 - 175.0 * u2)));
  double B = u2 / 1024.0 * (256.0 + u2 * (-128.0 + u2 * (74.0 - 47.0 * u2)));
  double dS = B * sinS * (cos2Sm + B / 4.0 * (cosS * (-1.0 + 2.0 * cos2Sm * cos2Sm) -
                                              B / 6.0 * cos2Sm * (-3.0 + 4.0 * sinS * sinS) * (-3.0 + 4.0 * cos2Sm * cos2Sm)));
  return b * A * (sig - dS);
}
// squared distance point - segment, closest point (buffer.cuh:97-103)
inline double pt_seg_d2(double px, double py, double ax, double ay, double bx, double by, double& qx, double& qy) {
  double dx = bx - ax, dy = by - ay, l2 = dx * dx + dy * dy;
  double t = l2 > 0 ? ((px - ax) * dx + (py - ay) * dy) / l2 : 0.0;
  t = std::fmin(1.0, std::fmax(0.0, t));
  qx = ax + t * dx; qy = ay + t * dy;
  return (px - qx) * (px - qx) + (py - qy) * (py - qy);
}
// squared distance of two non-crossing segments (buffer.cuh:106-117)
inline double seg_seg_d2(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y) {
  double qx, qy, tx, ty;
  double best = pt_seg_d2(a0x, a0y, b0x, b0y, b1x, b1y, qx, qy);
  double d = pt_seg_d2(a1x, a1y, b0x, b0y, b1x, b1y, tx, ty);
  if (d < best) best = d;
  d = pt_seg_d2(b0x, b0y, a0x, a0y, a1x, a1y, tx, ty);
  if (d < best) best = d;
  d = pt_seg_d2(b1x, b1y, a0x, a0y, a1x, a1y, tx, ty);
  if (d < best) best = d;
  return best;
}
// great-circle closest points (buffer.cuh:123-175)
struct V3 { double x, y, z; };
inline V3 v3_ll(double lon, double lat) { double cl = std::cos(lat); return V3{cl * std::cos(lon), cl * std::sin(lon), std::sin(lat)}; }
inline double v3_dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 v3_norm(V3 a) { double l = std::sqrt(v3_dot(a, a)); return l > 0 ? V3{a.x / l, a.y / l, a.z / l} : a; }
inline double v3_ang(V3 a, V3 b) {
  V3 c{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return std::atan2(std::sqrt(v3_dot(c, c)), v3_dot(a, b));
}
inline V3 robust_cross(double plon, double plat, double qlon, double qlat) {
  double lon_qpp = (qlon + plon) / -2.0, lon_qmp = (qlon - plon) / 2.0;
  double smq = std::sin(plat - qlat), spq = std::sin(plat + qlat);
  double s1 = std::sin(lon_qpp), s2 = std::sin(lon_qmp), c1 = std::cos(lon_qpp), c2 = std::cos(lon_qmp);
  return V3{smq * s1 * c2 - spq * c1 * s2, smq * c1 * c2 + spq * s1 * s2, std::cos(plat) * std::cos(qlat) * std::sin(qlon - plon)};
}
inline double arc_pt(double slon, double slat, double elon, double elat, double plon, double plat, double& clon, double& clat) {
  V3 vs = v3_ll(slon, slat), ve = v3_ll(elon, elat), vp = v3_ll(plon, plat);
  double best = 1e9;
  if (!(slon == elon && slat == elat)) {
    V3 n = v3_norm(robust_cross(slon, slat, elon, elat));
    double t = v3_dot(vp, n);
    V3 k = v3_norm(V3{vp.x - t * n.x, vp.y - t * n.y, vp.z - t * n.z});
    V3 vc = v3_norm(V3{vs.x + ve.x, vs.y + ve.y, vs.z + ve.z});
    double ds = v3_dot(vs, vc), dk = v3_dot(k, vc);
    if (dk > ds || std::fabs(dk - ds) < 2e-16) {
      best = v3_ang(vp, k);
      clat = std::atan2(k.z, std::sqrt(k.x * k.x + k.y * k.y)); clon = std::atan2(k.y, k.x);
    }
  }
  double d2 = v3_ang(vp, vs), d3 = v3_ang(vp, ve);
  if (d2 < best) { best = d2; clon = slon; clat = slat; }
  if (d3 < best) { best = d3; clon = elon; clat = elat; }
  return best;
}
inline double geog_dist(double a0x, double a0y, double a1x, double a1y, double b0x, double b0y, double b1x, double b1y, bool b_is_point) {
  const double R = DEG;
  double p1x, p1y, p2x, p2y, cx = 0, cy = 0, best;
  best = arc_pt(a0x * R, a0y * R, a1x * R, a1y * R, b0x * R, b0y * R, cx, cy); p1x = cx; p1y = cy; p2x = b0x * R; p2y = b0y * R;
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
inline double geog_band(double d, double rel_frame, double La2, double Lb2, double tl) {   // buffer.cuh:178-180
  return d * (rel_frame + 5e-5) + (La2 + Lb2) * tl / (8.0 * 6.3e6) + 1e-9;
}

// dw_pair (buffer.cuh:185-236): 1 when pieces a, b are within d meters
int dw_pair(const Set& P, const Set& R, uint32_t a, uint32_t b, double d, std::vector<Ed>& LA, std::vector<Ed>& LB) {
  double oax = P.ox[a], oay = P.oy[a], obx = R.ox[b], oby = R.oy[b], eax = P.ex[a], eay = P.ey[a], ebx = R.ex[b], eby = R.ey[b];
  double sx = obx - oax, sy = oby - oay;
  double gx, gy;
  deg_cover(std::fmin(oay, oby), std::fmax(oay + eay, oby + eby), d, true, gx, gy);
  Ov ov{std::fmax(-gx, sx - gx), std::fmax(-gy, sy - gy), std::fmin(eax + gx, sx + ebx + gx), std::fmin(eay + gy, sy + eby + gy)};
  if (ov.x0 > ov.x1 || ov.y0 > ov.y1) return 0;
  PV A = make_pv(P, a, oax, oay), B = make_pv(R, b, oax, oay);
  collect(A, ov, LA); collect(B, ov, LB);
  const int na = (int)LA.size(), nb = (int)LB.size();
  double phi0 = oay + 0.5 * (ov.y0 + ov.y1);
  double kx, ky; m_per_deg(phi0, kx, ky);
  const double tl = std::fabs(std::tan(phi0 * DEG)) + 0.01;
  double delta = 2.0 * 0.5 * (ov.y1 - ov.y0) * DEG * (tl + 0.04) + 1e-9;
  for (int i = 0; i < na; i++) {
    const Ed& e = LA[i];
    if (e.syn) continue;
    double bx0 = std::fmin(e.x0, e.x1) - gx, bx1 = std::fmax(e.x0, e.x1) + gx, by0 = std::fmin(e.y0, e.y1) - gy, by1 = std::fmax(e.y0, e.y1) + gy;
    const double ex = (e.x1 - e.x0) * kx, ey = (e.y1 - e.y0) * ky, La2 = ex * ex + ey * ey;
    for (int j = 0; j < nb; j++) {
      const Ed& f = LB[j];
      if (f.syn || std::fmax(f.x0, f.x1) < bx0 || std::fmin(f.x0, f.x1) > bx1 || std::fmax(f.y0, f.y1) < by0 || std::fmin(f.y0, f.y1) > by1) continue;
      if (seg_isect(e.x0, e.y0, e.x1, e.y1, f.x0, f.y0, f.x1, f.y1)) return 1;
      double d2 = seg_seg_d2(e.x0 * kx, e.y0 * ky, e.x1 * kx, e.y1 * ky, f.x0 * kx, f.y0 * ky, f.x1 * kx, f.y1 * ky);
      double fx = (f.x1 - f.x0) * kx, fy = (f.y1 - f.y0) * ky;
      double band = geog_band(d, delta, La2, fx * fx + fy * fy, tl);
      double dlo = d - band, dhi = d + band;
      if (d2 <= dlo * dlo) return 1;
      if (d2 <= dhi * dhi && geog_dist(oax + e.x0, oay + e.y0, oax + e.x1, oay + e.y1, oax + f.x0, oay + f.y0, oax + f.x1, oay + f.y1, false) <= d)
        return 1;
    }
  }
  double cx = ov.x0 + 0.381966 * (ov.x1 - ov.x0), cy = ov.y0 + 0.414213 * (ov.y1 - ov.y0);
  bool inB_c = pip_full(B, cx, cy), inA_c = pip_full(A, cx, cy);
  for (uint64_t r = A.r0; r < A.r1; r++) {
    double x, y;
    if (probe_vertex(A, r, x, y) && x >= ov.x0 && x <= ov.x1 && y >= ov.y0 && y <= ov.y1 && inside_from_c(LB.data(), nb, cx, cy, inB_c, x, y)) return 1;
  }
  for (uint64_t r = B.r0; r < B.r1; r++) {
    double x, y;
    if (probe_vertex(B, r, x, y) && x >= ov.x0 && x <= ov.x1 && y >= ov.y0 && y <= ov.y1 && inside_from_c(LA.data(), na, cx, cy, inA_c, x, y)) return 1;
  }
  return 0;
}

// k_expand_bb / k_expand_pts (buffer.cuh:703-715, 1004-1016): box widened by d meters, rounded outward to float
inline void expand_box(double x0, double y0, double x1, double y1, double d, float* out) {
  double dx, dy; deg_cover(y0, y1, d, true, dx, dy);
  double a = x0 - dx, b = y0 - dy, c = x1 + dx, e = y1 + dy;
  out[0] = f_down(a); out[1] = f_down(b); out[2] = f_up(c); out[3] = f_up(e);
}

std::vector<std::pair<uint32_t, uint32_t>> unique_parents(const uint32_t* cand, const std::vector<uint8_t>& keep, int64_t nc, const Set* Pp,
                                                          const Set& R) {
  std::vector<uint64_t> k;
  for (int64_t i = 0; i < nc; i++)
    if (keep[i]) k.push_back(((uint64_t)(Pp ? Pp->pid(cand[2 * i]) : cand[2 * i]) << 32) | R.pid(cand[2 * i + 1]));
  std::sort(k.begin(), k.end());
  k.erase(std::unique(k.begin(), k.end()), k.end());
  std::vector<std::pair<uint32_t, uint32_t>> out;
  for (uint64_t v : k) out.push_back({(uint32_t)(v >> 32), (uint32_t)v});
  return out;
}

int64_t emit(const std::vector<std::pair<uint32_t, uint32_t>>& v, uint32_t** out) {
  int64_t n = (int64_t)v.size();
  uint32_t* o = (uint32_t*)malloc(8 * (n ? n : 1));
  for (int64_t i = 0; i < n; i++) { o[2 * i] = v[i].first; o[2 * i + 1] = v[i].second; }
  *out = o;
  return n;
}

}  // namespace

extern "C" {

// dwithin_join_stream (buffer.cuh:892-991): expanded probe boxes, piece pairs (same-parent shortcut), parents
int64_t orc_dwithin(const orc_set* Po, const orc_set* Ro, double d, int same, int nthreads, uint32_t** out_pairs, int64_t* n_candidates) {
  const Set& P = Po->s; const Set& R = Ro->s;
  int nth = nthreads_or_default(nthreads);
  std::vector<float> qbb(4 * P.n);
  for (uint64_t i = 0; i < P.n; i++) {
    if (d > 0) expand_box(P.ox[i], P.oy[i], P.ox[i] + P.ex[i], P.oy[i] + P.ey[i], d, &qbb[4 * i]);
    else memcpy(&qbb[4 * i], &P.bb[4 * i], 16);
  }
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(qbb.data(), P.n, R, same, nth, &cand);
  if (n_candidates) *n_candidates = nc;
  std::vector<uint8_t> flag(nc);
#pragma omp parallel num_threads(nth)
  {
    std::vector<Ed> LA, LB;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < nc; i++) {
      uint32_t a = cand[2 * i], b = cand[2 * i + 1];
      if (same && P.pid(a) == R.pid(b)) { flag[i] = 1; continue; }   // buffer.cuh:247-250
      flag[i] = (uint8_t)dw_pair(P, R, a, b, d, LA, LB);
    }
  }
  auto v = unique_parents(cand, flag, nc, &P, R);
  free(cand);
  return emit(v, out_pairs);
}

// k_pt_dwithin (buffer.cuh:1019-1055) + points_buffer_join_stream folding (:1209-1219)
int64_t orc_pt_dwithin(const double* pts, uint64_t npts, const orc_set* Ro, double d, int nthreads, uint32_t** out_pairs) {
  const Set& R = Ro->s;
  int nth = nthreads_or_default(nthreads);
  std::vector<float> qbb(4 * npts);
  for (uint64_t i = 0; i < npts; i++) {
    if (d > 0) expand_box(pts[2 * i], pts[2 * i + 1], pts[2 * i], pts[2 * i + 1], d, &qbb[4 * i]);
    else { qbb[4 * i] = f_down(pts[2 * i]); qbb[4 * i + 1] = f_down(pts[2 * i + 1]); qbb[4 * i + 2] = f_up(pts[2 * i]); qbb[4 * i + 3] = f_up(pts[2 * i + 1]); }
  }
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(qbb.data(), npts, R, 0, nth, &cand);
  std::vector<uint8_t> hit(nc);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1024)
  for (int64_t i = 0; i < nc; i++) {
    uint32_t p = cand[2 * i], g = cand[2 * i + 1];
    double ptx = pts[2 * p], pty = pts[2 * p + 1], ox = R.ox[g], oy = R.oy[g];
    PV B = make_pv(R, g, ox, oy);
    double px = ptx - ox, py = pty - oy;
    double kx, ky; m_per_deg(pty, kx, ky);
    double gy = d / ky;
    const double tl = std::fabs(std::tan(pty * DEG)) + 0.01;
    double delta = 2.0 * gy * DEG * (tl + 0.04) + 1e-9;
    double lx = B.shx - 1.0;
    bool par = false, h = false;
    for (uint64_t r = B.r0; r < B.r1 && !h; r++) {
      uint64_t s0 = R.rvo[r], e = R.rvo[r + 1];
      double x0, y0; B.v(s0, x0, y0);
      for (uint64_t j = s0 + 1; j < e && !h; j++) {
        double x1, y1; B.v(j, x1, y1);
        if (!B.syn(j - 1)) {
          double qx, qy;
          double d2 = pt_seg_d2(px * kx, py * ky, x0 * kx, y0 * ky, x1 * kx, y1 * ky, qx, qy);
          double ex = (x1 - x0) * kx, ey = (y1 - y0) * ky;
          double band = geog_band(d, delta, ex * ex + ey * ey, 0.0, tl), dlo = d - band, dhi = d + band;
          if (d2 <= dlo * dlo || (d2 <= dhi * dhi && geog_dist(ox + x0, oy + y0, ox + x1, oy + y1, ptx, pty, ptx, pty, true) <= d)) h = true;
        }
        if (!((y0 > py) == (y1 > py) && y0 != py && y1 != py)) {
          bool so = left_of(x0, y0, x1, y1, lx, py), sp = left_of(x0, y0, x1, y1, px, py);
          if (so != sp) {
            bool su = orient(lx, py, px, py, x0, y0) > 0, sv = orient(lx, py, px, py, x1, y1) > 0;
            if (su != sv) par = !par;
          }
        }
        x0 = x1; y0 = y1;
      }
    }
    hit[i] = (h || par) ? 1 : 0;
  }
  auto v = unique_parents(cand, hit, nc, nullptr, R);
  free(cand);
  return emit(v, out_pairs);
}

}  // extern "C"

// ===== negative-buffer (erosion) intersects (buffer.cuh:275-889) ==============================================
namespace {

struct BEd { double x0, y0, x1, y1, ux, uy, L, ci, si; int succ, vt; };   // buffer.cuh:280
struct BEl { double x0, y0, x1, y1; };
constexpr double FILLET_QUANTUM = M_PI / 16.0;
constexpr int ER_CAPE = 64, ER_CAPL = 128, ER_MAX_DEPTH = 12;              // buffer.cuh:590, 593

// strictly inside the region within r of the boundary (buffer.cuh:285-319)
bool in_excl(const std::vector<BEd>& E, double r, double x, double y, double eps) {
  if (r <= 0) return false;
  const double ri = r - eps;
  for (size_t k = 0; k < E.size(); k++) {
    const BEd& e = E[k];
    if (x < std::fmin(e.x0, e.x1) - r || x > std::fmax(e.x0, e.x1) + r || y < std::fmin(e.y0, e.y1) - r || y > std::fmax(e.y0, e.y1) + r) continue;
    double dx = x - e.x0, dy = y - e.y0;
    double t = dx * e.ux + dy * e.uy, s = dy * e.ux - dx * e.uy;
    if (std::fabs(s) < ri && t > -eps && t < e.L + eps) return true;
    if (e.vt == 0) continue;
    double vx = x - e.x1, vy = y - e.y1, d2 = vx * vx + vy * vy;
    if (d2 >= r * r) continue;
    const BEd& f = E[e.succ];
    if (e.vt == 1) {
      double s2 = vy * f.ux - vx * f.uy;
      if (d2 < ri * ri && !(s > eps && s2 > eps)) return true;
      continue;
    }
    double nkx = -e.uy, nky = e.ux, nsx = -f.uy, nsy = f.ux;
    if (nkx * vy - nky * vx > eps) continue;
    if (nsx * vy - nsy * vx < -eps) continue;
    double chh = std::sqrt(0.5 * (1.0 + e.ci)), shh = std::sqrt(std::fmax(0.0, 0.5 * (1.0 - e.ci)));
    double ch = r * chh - eps;
    if (d2 < ch * ch) return true;
    double mx = nkx * chh + nky * shh, my = -nkx * shh + nky * chh;
    bool in = true;
    for (int i = 0, m = e.vt - 1; i < m && in; i++) {
      if (mx * vx + my * vy >= ch) in = false;
      double t2 = mx * e.ci + my * e.si; my = -mx * e.si + my * e.ci; mx = t2;
    }
    if (in) return true;
  }
  return false;
}
// parity from c (buffer.cuh:322-334)
bool inside_m(const std::vector<BEd>& E, double cx, double cy, bool in_c, double x, double y) {
  bool in = in_c;
  double sx0 = std::fmin(cx, x), sx1 = std::fmax(cx, x), sy0 = std::fmin(cy, y), sy1 = std::fmax(cy, y);
  for (const BEd& e : E) {
    if (std::fmax(e.x0, e.x1) < sx0 || std::fmin(e.x0, e.x1) > sx1 || std::fmax(e.y0, e.y1) < sy0 || std::fmin(e.y0, e.y1) > sy1) continue;
    bool sc = left_of(e.x0, e.y0, e.x1, e.y1, cx, cy), sx = left_of(e.x0, e.y0, e.x1, e.y1, x, y);
    if (sc == sx) continue;
    bool su = orient(cx, cy, x, y, e.x0, e.y0) > 0, sv = orient(cx, cy, x, y, e.x1, e.y1) > 0;
    if (su != sv) in = !in;
  }
  return in;
}
struct ESide { uint32_t g0, g1; double r; double bminx, bminy, bmaxx, bmaxy; };
struct EFrame { double ox, oy, kx, ky; };
inline void fv(const Set& S, double shx, double shy, uint64_t v, const EFrame& F, double& x, double& y) {   // buffer.cuh:352-355
  x = (shx + S.q[2 * v]) * F.kx;
  y = (shy + S.q[2 * v + 1]) * F.ky;
}
// c inside the parent (buffer.cuh:359-381)
bool pip_parent(const Set& S, const ESide& s, const EFrame& F, double cx, double cy) {
  bool in = false;
  for (uint32_t g = s.g0; g < s.g1 && !in; g++) {
    double bx0 = (S.ox[g] - F.ox) * F.kx, by0 = (S.oy[g] - F.oy) * F.ky, bx1 = (S.ox[g] + S.ex[g] - F.ox) * F.kx, by1 = (S.oy[g] + S.ey[g] - F.oy) * F.ky;
    if (cx < bx0 - 1e-6 || cx > bx1 + 1e-6 || cy < by0 - 1e-6 || cy > by1 + 1e-6) continue;
    double shx = S.ox[g] - F.ox, shy = S.oy[g] - F.oy, ox = bx0 - 1.0;
    bool par = false;
    for (uint64_t r = S.gro[g]; r < S.gro[g + 1]; r++)
      for (uint64_t j = S.rvo[r] + 1; j < S.rvo[r + 1]; j++) {
        double x0, y0, x1, y1; fv(S, shx, shy, j - 1, F, x0, y0); fv(S, shx, shy, j, F, x1, y1);
        if ((y0 > cy) == (y1 > cy) && y0 != cy && y1 != cy) continue;
        bool so = left_of(x0, y0, x1, y1, ox, cy), sc = left_of(x0, y0, x1, y1, cx, cy);
        if (so == sc) continue;
        bool su = orient(ox, cy, cx, cy, x0, y0) > 0, sv = orient(ox, cy, cx, cy, x1, y1) > 0;
        if (su != sv) par = !par;
      }
    in = par;
  }
  return in;
}
// the parent's real edges meeting box C (buffer.cuh:384-408); returns the count (all kept: no cap here)
void collect_side(const Set& S, const ESide& s, const EFrame& F, double cx0, double cy0, double cx1, double cy1, std::vector<BEd>& E) {
  E.clear();
  for (uint32_t g = s.g0; g < s.g1; g++) {
    if ((S.ox[g] + S.ex[g] - F.ox) * F.kx < cx0 || (S.ox[g] - F.ox) * F.kx > cx1 || (S.oy[g] + S.ey[g] - F.oy) * F.ky < cy0 || (S.oy[g] - F.oy) * F.ky > cy1) continue;
    double shx = S.ox[g] - F.ox, shy = S.oy[g] - F.oy;
    for (uint64_t r = S.gro[g]; r < S.gro[g + 1]; r++)
      for (uint64_t i = S.rvo[r]; i + 1 < S.rvo[r + 1]; i++) {
        if (S.synv(i)) continue;
        BEd ed{};
        fv(S, shx, shy, i, F, ed.x0, ed.y0); fv(S, shx, shy, i + 1, F, ed.x1, ed.y1);
        bool v = !(ed.x0 == ed.x1 && ed.y0 == ed.y1) &&
                 !(std::fmax(ed.x0, ed.x1) < cx0 || std::fmin(ed.x0, ed.x1) > cx1 || std::fmax(ed.y0, ed.y1) < cy0 || std::fmin(ed.y0, ed.y1) > cy1);
        if (v) E.push_back(ed);
      }
  }
}
// directions, successors, end-vertex regions (buffer.cuh:411-439)
void prepare_side(std::vector<BEd>& E, double r) {
  const int n = (int)E.size();
  for (int k = 0; k < n; k++) {
    double dx = E[k].x1 - E[k].x0, dy = E[k].y1 - E[k].y0, L = std::sqrt(dx * dx + dy * dy);
    E[k].ux = dx / L; E[k].uy = dy / L; E[k].L = L;
  }
  for (int k = 0; k < n; k++) {
    const BEd e = E[k];
    int s = -1;
    if (k + 1 < n && E[k + 1].x0 == e.x1 && E[k + 1].y0 == e.y1) s = k + 1;
    else for (int j = 0; j < n; j++) if (j != k && E[j].x0 == e.x1 && E[j].y0 == e.y1) { s = j; break; }
    int vt = 0; double ci = 1, si = 0;
    if (s >= 0 && r > 0) {
      const BEd& f = E[s];
      double cr = e.ux * f.uy - e.uy * f.ux, dt = e.ux * f.ux + e.uy * f.uy;
      if (cr > 0) vt = 1;
      else if (cr < 0 || dt < 0) {
        double th = std::atan2(-cr, dt);
        if (cr == 0) th = M_PI;
        int m = (int)(th / FILLET_QUANTUM + 0.5);
        if (m < 1) m = 1;
        double inc = th / m; ci = std::cos(inc); si = std::sin(inc);
        vt = m + 1;
      }
    }
    E[k].succ = s; E[k].vt = vt; E[k].ci = ci; E[k].si = si;
  }
}
// raw offset curve elements meeting W +- eps, in the warp's order: per 32-edge chunk, element index, edge (buffer.cuh:442-472)
void build_elements(const std::vector<BEd>& E, double r, double wx0, double wy0, double wx1, double wy1, double eps, std::vector<BEl>& L) {
  L.clear();
  const int n = (int)E.size();
  for (int base = 0; base < n; base += 32) {
    int mx = 0;
    for (int k = base; k < std::min(n, base + 32); k++) mx = std::max(mx, 1 + (E[k].vt >= 2 ? E[k].vt - 1 : 0));
    struct St { double wxr, wyr, px, py; };
    std::vector<St> st(32);
    for (int l = 0; l < 32 && base + l < n; l++) {
      const BEd& e = E[base + l];
      double nkx = -e.uy, nky = e.ux;
      st[l] = St{nkx, nky, e.x1 + r * nkx, e.y1 + r * nky};
    }
    for (int it = 0; it < mx; it++)
      for (int l = 0; l < 32 && base + l < n; l++) {
        const BEd& e = E[base + l];
        int ne = 1 + (e.vt >= 2 ? e.vt - 1 : 0);
        if (it >= ne) continue;
        double nkx = -e.uy, nky = e.ux, nsx = 0, nsy = 0;
        if (e.vt >= 2) { nsx = -E[e.succ].uy; nsy = E[e.succ].ux; }
        BEl el;
        if (it == 0) { el.x0 = e.x0 + r * nkx; el.y0 = e.y0 + r * nky; el.x1 = e.x1 + r * nkx; el.y1 = e.y1 + r * nky; }
        else {
          St& s = st[l];
          double t2 = s.wxr * e.ci + s.wyr * e.si; s.wyr = -s.wxr * e.si + s.wyr * e.ci; s.wxr = t2;
          double qx, qy;
          if (it == ne - 1) { qx = e.x1 + r * nsx; qy = e.y1 + r * nsy; } else { qx = e.x1 + r * s.wxr; qy = e.y1 + r * s.wyr; }
          el.x0 = s.px; el.y0 = s.py; el.x1 = qx; el.y1 = qy; s.px = qx; s.py = qy;
        }
        if (!(std::fmax(el.x0, el.x1) < wx0 - eps || std::fmin(el.x0, el.x1) > wx1 + eps || std::fmax(el.y0, el.y1) < wy0 - eps || std::fmin(el.y0, el.y1) > wy1 + eps))
          L.push_back(el);
      }
  }
}
// intersection points of two intersecting segments (buffer.cuh:475-493)
int seg_points(const BEl& p, const BEl& q, double* xs, double* ys) {
  double rx = p.x1 - p.x0, ry = p.y1 - p.y0, sx = q.x1 - q.x0, sy = q.y1 - q.y0;
  double den = rx * sy - ry * sx;
  if (den != 0) {
    double t = ((q.x0 - p.x0) * sy - (q.y0 - p.y0) * sx) / den;
    t = std::fmin(1.0, std::fmax(0.0, t));
    xs[0] = p.x0 + t * rx; ys[0] = p.y0 + t * ry;
    return 1;
  }
  double l2 = rx * rx + ry * ry;
  if (l2 == 0) { xs[0] = p.x0; ys[0] = p.y0; return 1; }
  double t0 = ((q.x0 - p.x0) * rx + (q.y0 - p.y0) * ry) / l2, t1 = ((q.x1 - p.x0) * rx + (q.y1 - p.y0) * ry) / l2;
  double lo = std::fmax(0.0, std::fmin(t0, t1)), hi = std::fmin(1.0, std::fmax(t0, t1));
  if (lo > hi) { double m = 0.5 * (lo + hi); lo = hi = std::fmin(1.0, std::fmax(0.0, m)); }
  xs[0] = p.x0 + lo * rx; ys[0] = p.y0 + lo * ry;
  xs[1] = p.x0 + hi * rx; ys[1] = p.y0 + hi * ry;
  xs[2] = p.x0 + 0.5 * (lo + hi) * rx; ys[2] = p.y0 + 0.5 * (lo + hi) * ry;
  return 3;
}

struct Win { double x0, y0, x1, y1; };

// er_pair (buffer.cuh:499-588): 1 / 0, or -1 when a list exceeded the caps (capE / capL < 0: unlimited)
int er_pair(const Set& P, const Set& R, uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, double ra_nom, double rb_nom, int capE, int capL,
            const Win* tile, Win* wout) {
  ESide A{a0, a1, 0, 1e300, 1e300, -1e300, -1e300}, B{b0, b1, 0, 1e300, 1e300, -1e300, -1e300};
  if (A.g0 >= A.g1 || B.g0 >= B.g1) return 0;
  auto bbox = [](const Set& S, ESide& s) {
    for (uint32_t g = s.g0; g < s.g1; g++) {
      s.bminx = std::fmin(s.bminx, S.ox[g]); s.bminy = std::fmin(s.bminy, S.oy[g]);
      s.bmaxx = std::fmax(s.bmaxx, S.ox[g] + S.ex[g]); s.bmaxy = std::fmax(s.bmaxy, S.oy[g] + S.ey[g]);
    }
  };
  bbox(P, A); bbox(R, B);
  double dax, day, dbx, dby;
  deg_cover(A.bminy, A.bmaxy, ra_nom * 0.998, false, dax, day);
  deg_cover(B.bminy, B.bmaxy, rb_nom * 0.998, false, dbx, dby);
  double wx0 = std::fmax(A.bminx + dax, B.bminx + dbx), wx1 = std::fmin(A.bmaxx - dax, B.bmaxx - dbx);
  double wy0 = std::fmax(A.bminy + day, B.bminy + dby), wy1 = std::fmin(A.bmaxy - day, B.bmaxy - dby);
  if (tile) { wx0 = std::fmax(wx0, tile->x0); wy0 = std::fmax(wy0, tile->y0); wx1 = std::fmin(wx1, tile->x1); wy1 = std::fmin(wy1, tile->y1); }
  if (wx0 > wx1 || wy0 > wy1) return 0;
  if (wout) *wout = Win{wx0, wy0, wx1, wy1};
  double clon = 0.5 * (wx0 + wx1), clat = 0.5 * (wy0 + wy1);
  A.r = ra_nom > 0 ? ra_nom / utm_k(0.5 * (A.bminx + A.bmaxx), 0.5 * (A.bminy + A.bmaxy), clon, clat) : 0.0;
  B.r = rb_nom > 0 ? rb_nom / utm_k(0.5 * (B.bminx + B.bmaxx), 0.5 * (B.bminy + B.bmaxy), clon, clat) : 0.0;
  EFrame F; F.ox = P.ox[A.g0]; F.oy = P.oy[A.g0]; m_per_deg(clat, F.kx, F.ky);
  double Wx0 = (wx0 - F.ox) * F.kx, Wx1 = (wx1 - F.ox) * F.kx, Wy0 = (wy0 - F.oy) * F.ky, Wy1 = (wy1 - F.oy) * F.ky;
  double ext = std::fmax(std::fmax(std::fabs(Wx0), std::fabs(Wx1)), std::fmax(std::fabs(Wy0), std::fabs(Wy1))) + std::fmax(A.r, B.r);
  const double eps = 1e-9 + 1e-12 * ext;
  double fe = 1.0 + 2.0 * 0.5 * (wy1 - wy0) * DEG * (std::fabs(std::tan(clat * DEG)) + 0.05);
  double ma = A.r * fe + 1e-6, mb = B.r * fe + 1e-6;
  std::vector<BEd> EA, EB; std::vector<BEl> LA, LB;
  collect_side(P, A, F, Wx0 - ma, Wy0 - ma, Wx1 + ma, Wy1 + ma, EA);
  collect_side(R, B, F, Wx0 - mb, Wy0 - mb, Wx1 + mb, Wy1 + mb, EB);
  if (capE >= 0 && ((int)EA.size() > capE || (int)EB.size() > capE)) return -1;
  prepare_side(EA, A.r); prepare_side(EB, B.r);
  build_elements(EA, A.r, Wx0, Wy0, Wx1, Wy1, eps, LA);
  build_elements(EB, B.r, Wx0, Wy0, Wx1, Wy1, eps, LB);
  if (capL >= 0 && ((int)LA.size() > capL || (int)LB.size() > capL)) return -1;
  auto inW = [&](double x, double y) { return x >= Wx0 - eps && x <= Wx1 + eps && y >= Wy0 - eps && y <= Wy1 + eps; };
  for (const BEl& p : LA) {
    double px0 = std::fmin(p.x0, p.x1), px1 = std::fmax(p.x0, p.x1), py0 = std::fmin(p.y0, p.y1), py1 = std::fmax(p.y0, p.y1);
    for (const BEl& q : LB) {
      if (std::fmax(q.x0, q.x1) < px0 || std::fmin(q.x0, q.x1) > px1 || std::fmax(q.y0, q.y1) < py0 || std::fmin(q.y0, q.y1) > py1) continue;
      if (!seg_isect(p.x0, p.y0, p.x1, p.y1, q.x0, q.y0, q.x1, q.y1)) continue;
      double xs[3], ys[3]; int k = seg_points(p, q, xs, ys);
      for (int t = 0; t < k; t++)
        if (inW(xs[t], ys[t]) && !in_excl(EA, A.r, xs[t], ys[t], eps) && !in_excl(EB, B.r, xs[t], ys[t], eps)) return 1;
    }
  }
  const double cx = Wx0 + 0.381966 * (Wx1 - Wx0), cy = Wy0 + 0.414213 * (Wy1 - Wy0);
  bool inA_c = pip_parent(P, A, F, cx, cy);
  bool inB_c = pip_parent(R, B, F, cx, cy);
  for (int side = 0; side < 2; side++) {
    const std::vector<BEd>& ES = side ? EB : EA; const std::vector<BEd>& EO = side ? EA : EB;
    const std::vector<BEl>& LS = side ? LB : LA;
    double rs = side ? B.r : A.r, ro = side ? A.r : B.r;
    bool inO_c = side ? inA_c : inB_c;
    auto vio = [&](double x, double y) {
      return inW(x, y) && !in_excl(ES, rs, x, y, eps) && inside_m(EO, cx, cy, inO_c, x, y) && !in_excl(EO, ro, x, y, eps);
    };
    for (size_t i = 0; i < LS.size(); i++) {
      const BEl& p = LS[i];
      if (vio(p.x0, p.y0) || vio(p.x1, p.y1)) return 1;
      double px0 = std::fmin(p.x0, p.x1), px1 = std::fmax(p.x0, p.x1), py0 = std::fmin(p.y0, p.y1), py1 = std::fmax(p.y0, p.y1);
      for (size_t j = i + 1; j < LS.size(); j++) {
        const BEl& q = LS[j];
        if (std::fmax(q.x0, q.x1) < px0 || std::fmin(q.x0, q.x1) > px1 || std::fmax(q.y0, q.y1) < py0 || std::fmin(q.y0, q.y1) > py1) continue;
        if (!seg_isect(p.x0, p.y0, p.x1, p.y1, q.x0, q.y0, q.x1, q.y1)) continue;
        double xs[3], ys[3]; int k = seg_points(p, q, xs, ys);
        for (int t = 0; t < k; t++) if (vio(xs[t], ys[t])) return 1;
      }
    }
  }
  return 0;
}

// the reference's overflow handling: window quadrants while larger than the radius (depth <= 12), then one
// evaluation with unlimited lists (k_erode_tiles / er_overflow / k_erode_slab, buffer.cuh:608-684)
int er_eval(const Set& P, const Set& R, uint32_t a0, uint32_t a1, uint32_t b0, uint32_t b1, double ra, double rb, const Win* tile, int depth) {
  Win win;
  int r = er_pair(P, R, a0, a1, b0, b1, ra, rb, ER_CAPE, ER_CAPL, tile, &win);
  if (r >= 0) return r;
  double kx, ky; m_per_deg(0.5 * (win.y0 + win.y1), kx, ky);
  double ext = std::fmax((win.x1 - win.x0) * kx, (win.y1 - win.y0) * ky);
  if (depth < ER_MAX_DEPTH && ext > std::fmax(ra, rb)) {
    double xm = 0.5 * (win.x0 + win.x1), ym = 0.5 * (win.y0 + win.y1);
    Win q[4] = {{win.x0, win.y0, xm, ym}, {xm, win.y0, win.x1, ym}, {win.x0, ym, xm, win.y1}, {xm, ym, win.x1, win.y1}};
    for (int i = 0; i < 4; i++) if (er_eval(P, R, a0, a1, b0, b1, ra, rb, &q[i], depth + 1) == 1) return 1;
    return 0;
  }
  return er_pair(P, R, a0, a1, b0, b1, ra, rb, -1, -1, &win, nullptr) == 1 ? 1 : 0;
}

inline void piece_range(const Set& S, uint32_t p, const std::vector<uint32_t>& pf, uint32_t& g0, uint32_t& g1) {
  if (S.has_parent) { g0 = pf[p]; g1 = pf[p + 1]; } else { g0 = p; g1 = p + 1; }
}
std::vector<uint32_t> piece_first(const Set& S) {   // k_piece_first (buffer.cuh:342-348)
  std::vector<uint32_t> pf(S.nparent + 1, (uint32_t)S.n);
  for (int64_t g = (int64_t)S.n - 1; g >= 0; g--) pf[S.parent[g]] = (uint32_t)g;
  for (int64_t p = (int64_t)S.nparent - 1; p >= 0; p--) if (pf[p] == S.n && p + 1 <= (int64_t)S.nparent) pf[p] = pf[p + 1];
  return pf;
}

}  // namespace

extern "C" {

// erode_join_stream (buffer.cuh:765-889): pass 1 = intersects + area join (with the shrunk-bbox prefilter), then
// the area filter and the erosion test on the surviving parent pairs
int64_t orc_erode(const orc_set* Po, const orc_set* Ro, double ra, double rb, int same, const uint8_t* need_self, int nthreads, uint32_t** out_pairs) {
  const Set& P = Po->s; const Set& R = Ro->s;
  int nth = nthreads_or_default(nthreads);
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(P.bb.data(), P.n, R, same, nth, &cand);
  // k_er_prefilter (buffer.cuh:742-762): whole-geometry pieces whose shrunk bboxes are disjoint cannot meet
  auto whole = [](const Set& S, uint32_t g) {
    if (!S.has_parent) return true;
    uint32_t q = S.parent[g];
    return (g == 0 || S.parent[g - 1] != q) && (g + 1 >= S.n || S.parent[g + 1] != q);
  };
  std::vector<uint32_t> kept;
  for (int64_t i = 0; i < nc; i++) {
    uint32_t a = cand[2 * i], b = cand[2 * i + 1];
    bool k = true;
    if ((ra > 0 || rb > 0) && whole(P, a) && whole(R, b)) {
      double dax, day, dbx, dby;
      deg_cover(P.oy[a], P.oy[a] + P.ey[a], ra * 0.998, false, dax, day);
      deg_cover(R.oy[b], R.oy[b] + R.ey[b], rb * 0.998, false, dbx, dby);
      double wx0 = std::fmax(P.ox[a] + dax, R.ox[b] + dbx), wx1 = std::fmin(P.ox[a] + P.ex[a] - dax, R.ox[b] + R.ex[b] - dbx);
      double wy0 = std::fmax(P.oy[a] + day, R.oy[b] + dby), wy1 = std::fmin(P.oy[a] + P.ey[a] - day, R.oy[b] + R.ey[b] - dby);
      k = wx0 <= wx1 && wy0 <= wy1;
    }
    if (k) { kept.push_back(a); kept.push_back(b); }
  }
  free(cand);
  // pass 1: exact intersects + area over the kept piece pairs, folded to parents (engine.cuh:963-1042 semantics)
  int64_t nk = (int64_t)kept.size() / 2;
  orc_params rp{1e-12, 1e-7, 1e-11, 1, 0, 0};
  std::vector<uint8_t> flag(nk); std::vector<double> area(nk);
  orc_refine_pairs(Po, Ro, kept.data(), nk, &rp, flag.data(), area.data(), nullptr, nullptr, nth);
  const bool agg = P.has_parent || R.has_parent;
  std::vector<std::pair<uint64_t, double>> parents;   // (parent key, area) of parent pairs with real contact
  {
    std::vector<int64_t> idx;
    for (int64_t i = 0; i < nk; i++) if (agg ? flag[i] != 0 : flag[i] == 1) idx.push_back(i);
    auto key = [&](int64_t i) { return ((uint64_t)P.pid(kept[2 * i]) << 32) | R.pid(kept[2 * i + 1]); };
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return key(x) < key(y); });
    for (size_t k = 0; k < idx.size();) {
      size_t m = k; uint64_t kk = key(idx[k]); double a = 0; uint8_t f = 255;
      for (; m < idx.size() && key(idx[m]) == kk; m++) { a += area[idx[m]]; f = std::min(f, flag[idx[m]]); }
      if (f == 1) parents.push_back({kk, a});
      k = m;
    }
  }
  // k_er_filter (buffer.cuh:720-738)
  const double rmin = (ra > 0 && rb > 0) ? std::min(ra, rb) : (ra > 0 || rb > 0 ? 0.0 : -1.0);
  std::vector<uint32_t> pfP, pfR;
  if (P.has_parent) pfP = piece_first(P);
  if (R.has_parent) pfR = piece_first(R);
  std::vector<uint64_t> ep;
  for (auto& pa : parents) {
    uint32_t x = (uint32_t)(pa.first >> 32), y = (uint32_t)pa.first;
    bool k = true;
    if (same && x == y && need_self) k = need_self[x] != 0;
    if (k && rmin >= 0) {
      uint32_t g = P.has_parent ? pfP[x] : x;
      double y0 = P.oy[g], y1 = y0 + P.ey[g];
      double lat = (y0 <= 0 && y1 >= 0) ? 0.0 : (std::fabs(y0) < std::fabs(y1) ? y0 : y1);
      double kx, ky; m_per_deg(lat, kx, ky);
      double a_m2 = pa.second * kx * ky * 1.001;
      double r = 0.98 * rmin;
      k = rmin > 0 ? a_m2 >= M_PI * r * r : pa.second > 0;
    }
    if (k) ep.push_back(pa.first);
  }
  std::vector<uint8_t> hit(ep.size());
#pragma omp parallel for num_threads(nth) schedule(dynamic, 16)
  for (int64_t i = 0; i < (int64_t)ep.size(); i++) {
    uint32_t x = (uint32_t)(ep[i] >> 32), y = (uint32_t)ep[i], a0, a1, b0, b1;
    piece_range(P, x, pfP, a0, a1); piece_range(R, y, pfR, b0, b1);
    hit[i] = (uint8_t)er_eval(P, R, a0, a1, b0, b1, ra, rb, nullptr, 0);
  }
  std::vector<std::pair<uint32_t, uint32_t>> out;
  for (size_t i = 0; i < ep.size(); i++) if (hit[i]) out.push_back({(uint32_t)(ep[i] >> 32), (uint32_t)ep[i]});
  return emit(out, out_pairs);
}

}  // extern "C"

namespace {
// inside the exclusion region of vertex v (edges with unit directions e -> f), w relative to v (buffer.cuh:1059-1083)
bool vertex_excl(double ex, double ey, double fx, double fy, double r, double wx, double wy, double eps) {
  double d2 = wx * wx + wy * wy;
  if (d2 >= r * r) return false;
  double cr = ex * fy - ey * fx, dt = ex * fx + ey * fy;
  if (cr > 0) {
    double ri = r - eps, s1 = wy * ex - wx * ey, s2 = wy * fx - wx * fy;
    return d2 < ri * ri && !(s1 > eps && s2 > eps);
  }
  if (cr == 0 && dt >= 0) return false;
  double th = cr == 0 ? M_PI : std::atan2(-cr, dt);
  int m = (int)(th / FILLET_QUANTUM + 0.5);
  if (m < 1) m = 1;
  double inc = th / m, ci = std::cos(inc), si = std::sin(inc);
  double nkx = -ey, nky = ex, nsx = -fy, nsy = fx;
  if (nkx * wy - nky * wx > eps || nsx * wy - nsy * wx < -eps) return false;
  double chh = std::sqrt(0.5 * (1.0 + ci)), shh = std::sqrt(std::fmax(0.0, 0.5 * (1.0 - ci)));
  double ch = r * chh - eps;
  if (d2 < ch * ch) return true;
  double mx = nkx * chh + nky * shh, my = -nkx * shh + nky * chh;
  for (int i = 0; i < m; i++) {
    if (mx * wx + my * wy >= ch) return false;
    double t2 = mx * ci + my * si; my = -mx * si + my * ci; mx = t2;
  }
  return true;
}
}  // namespace

extern "C" {

// k_pt_erode (buffer.cuh:1087-1132) + the (point, parent) OR fold of points_buffer_join_stream (:1187-1208)
int64_t orc_pt_erode(const double* pts, uint64_t npts, const orc_set* Ro, double r_nom, int nthreads, uint32_t** out_pairs) {
  const Set& R = Ro->s;
  int nth = nthreads_or_default(nthreads);
  const double grow = r_nom * 1.002;
  std::vector<float> qbb(4 * npts);
  for (uint64_t i = 0; i < npts; i++) {
    if (grow > 0) expand_box(pts[2 * i], pts[2 * i + 1], pts[2 * i], pts[2 * i + 1], grow, &qbb[4 * i]);
    else { qbb[4 * i] = f_down(pts[2 * i]); qbb[4 * i + 1] = f_down(pts[2 * i + 1]); qbb[4 * i + 2] = f_up(pts[2 * i]); qbb[4 * i + 3] = f_up(pts[2 * i + 1]); }
  }
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(qbb.data(), npts, R, 0, nth, &cand);
  std::vector<uint8_t> bits(nc);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1024)
  for (int64_t i = 0; i < nc; i++) {
    uint32_t p = cand[2 * i], g = cand[2 * i + 1];
    double ptx = pts[2 * p], pty = pts[2 * p + 1];
    double r = r_nom / utm_k(R.ox[g] + 0.5 * R.ex[g], R.oy[g] + 0.5 * R.ey[g], ptx, pty);
    double kx, ky; m_per_deg(pty, kx, ky);
    const double eps = 1e-9;
    double shx = R.ox[g] - ptx, shy = R.oy[g] - pty, ox = shx * kx - 1.0;
    auto vx = [&](uint64_t j, double& x, double& y) { x = (shx + R.q[2 * j]) * kx; y = (shy + R.q[2 * j + 1]) * ky; };
    bool par = false, ex = false;
    for (uint64_t rr = R.gro[g]; rr < R.gro[g + 1] && !ex; rr++) {
      uint64_t s0 = R.rvo[rr], e = R.rvo[rr + 1];
      if (e - s0 < 2) continue;
      bool pv = false; double pux = 0, puy = 0;
      { uint64_t j = e - 2; if (!R.synv(j)) { double a, b, c, dd; vx(j, a, b); vx(j + 1, c, dd); double L = std::hypot(c - a, dd - b);
          if (L > 0) { pv = true; pux = (c - a) / L; puy = (dd - b) / L; } } }
      double x0, y0; vx(s0, x0, y0);
      for (uint64_t j = s0; j + 1 < e && !ex; j++) {
        double x1, y1; vx(j + 1, x1, y1);
        if (!((y0 > 0) == (y1 > 0) && y0 != 0 && y1 != 0)) {
          bool so = left_of(x0, y0, x1, y1, ox, 0.0), sp = left_of(x0, y0, x1, y1, 0.0, 0.0);
          if (so != sp) {
            bool su = orient(ox, 0.0, 0.0, 0.0, x0, y0) > 0, sv = orient(ox, 0.0, 0.0, 0.0, x1, y1) > 0;
            if (su != sv) par = !par;
          }
        }
        double L = std::hypot(x1 - x0, y1 - y0);
        if (R.synv(j) || L == 0) { if (R.synv(j)) pv = false; x0 = x1; y0 = y1; continue; }
        double ux = (x1 - x0) / L, uy = (y1 - y0) / L;
        if (r > 0) {
          double t = -x0 * ux - y0 * uy, s = -y0 * ux + x0 * uy;
          if (std::fabs(s) < r - eps && t > -eps && t < L + eps) ex = true;
          else if (pv && vertex_excl(pux, puy, ux, uy, r, -x0, -y0, eps)) ex = true;
        }
        pv = true; pux = ux; puy = uy;
        x0 = x1; y0 = y1;
      }
    }
    bits[i] = ex ? 2 : (par ? 1 : 0);
  }
  // OR per (point, parent), keep == 1
  std::vector<std::pair<uint64_t, uint8_t>> kv;
  for (int64_t i = 0; i < nc; i++) kv.push_back({((uint64_t)cand[2 * i] << 32) | R.pid(cand[2 * i + 1]), bits[i]});
  free(cand);
  std::sort(kv.begin(), kv.end());
  std::vector<std::pair<uint32_t, uint32_t>> out;
  for (size_t k = 0; k < kv.size();) {
    size_t m = k; uint8_t o = 0;
    for (; m < kv.size() && kv[m].first == kv[k].first; m++) o |= kv[m].second;
    if (o == 1) out.push_back({(uint32_t)(kv[k].first >> 32), (uint32_t)kv[k].first});
    k = m;
  }
  return emit(out, out_pairs);
}

}  // extern "C"
