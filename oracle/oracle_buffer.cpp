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
