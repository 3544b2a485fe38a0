// Shared internals of the CPU FP64 oracle - TEST INFRASTRUCTURE ONLY (see oracle.h).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

struct Set {
  uint64_t n = 0, nr = 0, nv = 0;
  std::vector<uint64_t> gro, rvo;
  std::vector<double> q;             // xy - origin (engine.cuh:60-63)
  std::vector<double> ox, oy, ex, ey;   // origin = bbox min, ext = bbox extent (engine.cuh:57-58)
  std::vector<float> bb;             // outward-rounded float bbox (engine.cuh:59)
  bool has_parent = false; std::vector<uint32_t> parent;
  bool has_syn = false; std::vector<uint8_t> syn;
  uint32_t nparent = 0; std::vector<double> blen;   // real boundary length per parent (engine.cuh:69-82)
  uint32_t pid(uint32_t g) const { return has_parent ? parent[g] : g; }
  int synv(uint64_t i) const { return has_syn ? (int)syn[i] : 0; }
};

inline float f_down(double v) { float f = (float)v; if ((double)f > v) f = nextafterf(f, -INFINITY); return f; }   // engine.cuh:34
inline float f_up(double v) { float f = (float)v; if ((double)f < v) f = nextafterf(f, INFINITY); return f; }      // engine.cuh:35

// ---- predicates (engine.cuh:283-316) ----
inline double orient(double ax, double ay, double bx, double by, double cx, double cy) {
  double a = bx - ax, b = cy - ay, c = by - ay, d = cx - ax;
  double w = c * d;
  double e = std::fma(-c, d, w);
  double f = std::fma(a, b, -w);
  return f + e;
}
inline bool onseg(double ax, double ay, double bx, double by, double px, double py) {
  return px >= std::fmin(ax, bx) && px <= std::fmax(ax, bx) && py >= std::fmin(ay, by) && py <= std::fmax(ay, by);
}
inline bool left_of(double ax, double ay, double bx, double by, double px, double py) {
  double o = orient(ax, ay, bx, by, px, py);
  if (o != 0) return o > 0;
  double dy = by - ay;
  if (dy != 0) return dy < 0;
  return bx > ax;
}
inline bool seg_isect(double p0x, double p0y, double p1x, double p1y, double q0x, double q0y, double q1x, double q1y) {
  double d1 = orient(q0x, q0y, q1x, q1y, p0x, p0y), d2 = orient(q0x, q0y, q1x, q1y, p1x, p1y);
  double d3 = orient(p0x, p0y, p1x, p1y, q0x, q0y), d4 = orient(p0x, p0y, p1x, p1y, q1x, q1y);
  if (((d1 > 0 && d2 < 0) || (d1 < 0 && d2 > 0)) && ((d3 > 0 && d4 < 0) || (d3 < 0 && d4 > 0))) return true;
  if (d1 == 0 && onseg(q0x, q0y, q1x, q1y, p0x, p0y)) return true;
  if (d2 == 0 && onseg(q0x, q0y, q1x, q1y, p1x, p1y)) return true;
  if (d3 == 0 && onseg(p0x, p0y, p1x, p1y, q0x, q0y)) return true;
  if (d4 == 0 && onseg(p0x, p0y, p1x, p1y, q1x, q1y)) return true;
  return false;
}

// polygon in a pair frame (engine.cuh:265-279)
struct PV {
  const Set* s; uint64_t r0, r1; double shx, shy;
  void v(uint64_t i, double& x, double& y) const { x = shx + s->q[2 * i]; y = shy + s->q[2 * i + 1]; }
  int syn(uint64_t i) const { return s->synv(i); }
};
inline PV make_pv(const Set& s, uint32_t g, double rx, double ry) {
  PV p; p.s = &s; p.r0 = s.gro[g]; p.r1 = s.gro[g + 1]; p.shx = s.ox[g] - rx; p.shy = s.oy[g] - ry; return p;
}

struct Ov { double x0, y0, x1, y1; };
struct Ed { double x0, y0, x1, y1; int syn; int cut; };

inline bool edge_outside(double px, double py, double qx, double qy, const Ov& o) {   // engine.cuh:329-331
  return std::fmax(px, qx) < o.x0 || std::fmin(px, qx) > o.x1 || std::fmax(py, qy) < o.y0 || std::fmin(py, qy) > o.y1;
}
inline bool probe_vertex(const PV& A, uint64_t r, double& x, double& y) {   // engine.cuh:322-327
  uint64_t v = A.s->rvo[r], e = A.s->rvo[r + 1];
  if (A.s->has_syn) { while (v + 1 < e && A.syn(v)) v++; if (v + 1 >= e) return false; }
  A.v(v, x, y);
  return true;
}
// all edges meeting the overlap box, in ring order (collect_edges, engine.cuh:358-377, without a cap)
inline void collect(const PV& A, const Ov& ov, std::vector<Ed>& out) {
  out.clear();
  const bool hs = A.s->has_syn;
  for (uint64_t ra = A.r0; ra < A.r1; ra++) {
    uint64_t s = A.s->rvo[ra], e = A.s->rvo[ra + 1];
    for (uint64_t i = s; i + 1 < e; i++) {
      Ed ed; A.v(i, ed.x0, ed.y0); A.v(i + 1, ed.x1, ed.y1); ed.syn = A.syn(i);
      ed.cut = hs ? ((A.syn(i > s ? i - 1 : e - 2) ? 1 : 0) | (A.syn(i + 2 < e ? i + 1 : s) ? 2 : 0)) : 0;
      if (!edge_outside(ed.x0, ed.y0, ed.x1, ed.y1, ov)) out.push_back(ed);
    }
  }
}
// crossing parity from a point left of B's bbox (pip_full_warp, engine.cuh:382-397)
inline bool pip_full(const PV& B, double mx, double my) {
  double ox = B.shx - (double)1, oy = my;
  bool par = false;
  for (uint64_t r = B.r0; r < B.r1; r++) {
    uint64_t s = B.s->rvo[r], e = B.s->rvo[r + 1];
    for (uint64_t j = s + 1; j < e; j++) {
      double x0, y0, x1, y1; B.v(j - 1, x0, y0); B.v(j, x1, y1);
      if ((y0 > my) == (y1 > my) && y0 != my && y1 != my) continue;
      bool so = left_of(x0, y0, x1, y1, ox, oy), sc = left_of(x0, y0, x1, y1, mx, my);
      if (so == sc) continue;
      bool su = orient(ox, oy, mx, my, x0, y0) > 0, sv = orient(ox, oy, mx, my, x1, y1) > 0;
      if (su != sv) par = !par;
    }
  }
  return par;
}
// engine.cuh:400-412
inline bool inside_from_c(const Ed* L, int cnt, double cx, double cy, bool in_c, double x, double y) {
  bool in = in_c;
  double sx0 = std::fmin(cx, x), sx1 = std::fmax(cx, x), sy0 = std::fmin(cy, y), sy1 = std::fmax(cy, y);
  for (int k = 0; k < cnt; k++) {
    const Ed& e = L[k];
    if (std::fmax(e.x0, e.x1) < sx0 || std::fmin(e.x0, e.x1) > sx1 || std::fmax(e.y0, e.y1) < sy0 || std::fmin(e.y0, e.y1) > sy1) continue;
    bool sc = left_of(e.x0, e.y0, e.x1, e.y1, cx, cy), sx = left_of(e.x0, e.y0, e.x1, e.y1, x, y);
    if (sc == sx) continue;
    bool su = orient(cx, cy, x, y, e.x0, e.y0) > 0, sv = orient(cx, cy, x, y, e.x1, e.y1) > 0;
    if (su != sv) in = !in;
  }
  return in;
}

constexpr uint32_t REL_COIN_SAME = 1, REL_COIN_OPP = 2, REL_TOUCH = 4;   // engine.cuh:334-336
constexpr int MAXS = 24, MAXO = 8;                                        // engine.cuh:339-340

// engine.cuh:416-515: Green's-theorem contribution of edge p->q clipped to the other polygon, product-rule
// weights on coincident pieces, and (relate) inside / on lengths plus coincidence bits.
inline double edge_contrib(double px, double py, double qx, double qy, const Ed* L, int cnt, double cx, double cy, bool in_c, const Ov& ov,
                    double tol, double eps_par, bool real, double* l_in, double* l_on, uint32_t* bits, int cut, double snap) {
  double dx = qx - px, dy = qy - py;
  double len2 = dx * dx + dy * dy;
  if (len2 == 0) return 0.0;
  double tol2len2 = tol * tol * len2, eps2 = eps_par * eps_par;
  double ts[MAXS]; int ns = 0;
  double ol0[MAXO], ol1[MAXO]; bool osame[MAXO]; int oidx[MAXO]; int no = 0;
  ts[ns++] = 0; ts[ns++] = 1;
  double bx0 = std::fmin(px, qx) - tol, bx1 = std::fmax(px, qx) + tol, by0 = std::fmin(py, qy) - tol, by1 = std::fmax(py, qy) + tol;
  for (int k = 0; k < cnt; k++) {
    const Ed& e = L[k];
    if (std::fmax(e.x0, e.x1) < bx0 || std::fmin(e.x0, e.x1) > bx1 || std::fmax(e.y0, e.y1) < by0 || std::fmin(e.y0, e.y1) > by1) continue;
    double fx = e.x1 - e.x0, fy = e.y1 - e.y0;
    double r = dx * fy - dy * fx;
    double flen2 = fx * fx + fy * fy;
    double snap2 = snap * snap;
    double c0 = orient(px, py, qx, qy, e.x0, e.y0), c1 = orient(px, py, qx, qy, e.x1, e.y1);
    bool col = (c0 * c0 <= snap2 * len2 || ((e.cut & 1) && c0 * c0 <= tol2len2)) && (c1 * c1 <= snap2 * len2 || ((e.cut & 2) && c1 * c1 <= tol2len2));
    if (!col && flen2 > 0) {
      double g0 = orient(e.x0, e.y0, e.x1, e.y1, px, py), g1 = orient(e.x0, e.y0, e.x1, e.y1, qx, qy), tf = tol * tol * flen2;
      col = (g0 * g0 <= snap2 * flen2 || ((cut & 1) && g0 * g0 <= tf)) && (g1 * g1 <= snap2 * flen2 || ((cut & 2) && g1 * g1 <= tf));
    }
    if (col) {
      double tc = ((e.x0 - px) * dx + (e.y0 - py) * dy) / len2, te = ((e.x1 - px) * dx + (e.y1 - py) * dy) / len2;
      double lo = std::fmax((double)0, std::fmin(tc, te)), hi = std::fmin((double)1, std::fmax(tc, te));
      if (hi > lo) {
        if (lo > 0 && ns < MAXS) ts[ns++] = lo;
        if (hi < 1 && ns < MAXS) ts[ns++] = hi;
        if (no < MAXO) { ol0[no] = lo; ol1[no] = hi; osame[no] = (dx * fx + dy * fy) > 0; oidx[no] = k; no++; }
      }
    } else if (r * r > eps2 * len2 * flen2) {
      double wx = e.x0 - px, wy = e.y0 - py;
      double tn = wx * fy - wy * fx;
      if (r > 0 ? (tn <= 0 || tn >= r) : (tn >= 0 || tn <= r)) continue;
      double t = tn / r, u = (wx * dy - wy * dx) / r;
      double du = tol / (flen2 > 0 ? std::sqrt(flen2) : (double)1);
      if (u >= -du && u <= 1 + du && ns < MAXS) ts[ns++] = t;
    }
  }
  for (int a = 1; a < ns; a++) { double v = ts[a]; int b = a - 1; while (b >= 0 && ts[b] > v) { ts[b + 1] = ts[b]; b--; } ts[b + 1] = v; }
  double acc = 0.0;
  for (int k = 0; k + 1 < ns; k++) {
    double t0 = ts[k], t1 = ts[k + 1];
    if (!(t1 > t0)) continue;
    double tm = (double)0.5 * (t0 + t1);
    double mx = px + dx * tm, my = py + dy * tm;
    bool in_ov = mx >= ov.x0 && mx <= ov.x1 && my >= ov.y0 && my <= ov.y1;
    int net = 0, first = -1, net_real = 0, n_real = 0;
    for (int o = 0; o < no; o++)
      if (tm > ol0[o] && tm < ol1[o]) {
        int sgn = osame[o] ? 1 : -1;
        net += sgn; if (first < 0) first = o;
        if (!L[oidx[o]].syn) { net_real += sgn; n_real++; }
      }
    int vin = -1;
    auto inside_m = [&]() { if (vin < 0) vin = (in_ov && inside_from_c(L, cnt, cx, cy, in_c, mx, my)) ? 1 : 0; return vin; };
    if (l_in && real) {
      double seg = std::sqrt(len2) * (t1 - t0);
      if (net_real != 0) { *l_on += seg; *bits |= (net_real > 0 ? REL_COIN_SAME : REL_COIN_OPP) | REL_TOUCH; }
      else if (n_real == 0 && (net == 1 || net == -1)) *l_in += 0.5 * seg;
      else if (inside_m()) *l_in += seg;
    }
    double w;
    if (first < 0) w = inside_m() ? 1.0 : 0.0;
    else if (net == 1 || net == -1) w = 0.5;
    else if (net == 0) w = inside_m() ? 1.0 : 0.0;
    else {
      const Ed& eb = L[oidx[first]];
      bool sb = left_of(eb.x0, eb.y0, eb.x1, eb.y1, mx, my);
      bool m_left = osame[first] ? sb : !sb;
      int v = inside_m();
      int other = m_left ? v - net : v + net;
      other = other < 0 ? 0 : (other > 1 ? 1 : other);
      w = 0.5 * (v + other);
    }
    if (w != 0.0) {
      double ax = px + dx * t0 - cx, ay = py + dy * t0 - cy, bx = px + dx * t1 - cx, by = py + dy * t1 - cy;
      acc += w * (double)(ax * by - ay * bx);
    }
  }
  return acc;
}

// warp reduction of the reference (__shfl_down_sync tree 16, 8, 4, 2, 1), lane 0's result
inline double warp_sum(const double* v) {
  double a[32]; memcpy(a, v, sizeof(a));
  for (int o = 16; o > 0; o >>= 1) {
    double b[32];
    for (int l = 0; l < 32; l++) b[l] = a[l] + (l + o < 32 ? a[l + o] : a[l]);
    memcpy(a, b, sizeof(a));
  }
  return a[0];
}

inline double pair_snap(double oax, double oay, double eax, double eay) {   // engine.cuh:524-527
  double m = std::fmax(std::fmax(std::fabs(oax), std::fabs(oax + eax)), std::fmax(std::fabs(oay), std::fabs(oay + eay)));
  return 0.5 * (std::nextafter(m, INFINITY) - m);
}

struct PairOut { uint8_t flag; double area; double ev[4]; uint32_t evb; };

// k_refine for one pair (engine.cuh:530-636), without the shared-memory cap (the heavy path computes the
// same decision for oversized pairs)
inline PairOut refine_pair(const Set& P, const Set& R, uint32_t a, uint32_t b, const orc_params& rp, std::vector<Ed>& LA, std::vector<Ed>& LB) {
  PairOut o; o.flag = 0; o.area = 0; o.ev[0] = o.ev[1] = o.ev[2] = o.ev[3] = 0; o.evb = 0;
  double oax = P.ox[a], oay = P.oy[a], obx = R.ox[b], oby = R.oy[b];
  double eax = P.ex[a], eay = P.ey[a], ebx = R.ex[b], eby = R.ey[b];
  double sx = obx - oax, sy = oby - oay;
  double pad = 4.0 * std::fmax(rp.tol_abs, (double)rp.tol_rel * std::fmax(std::fmax(eax, eay), std::fmax(ebx, eby)));
  Ov ov{std::fmax(0.0, sx) - pad, std::fmax(0.0, sy) - pad, std::fmin(eax, sx + ebx) + pad, std::fmin(eay, sy + eby) + pad};
  PV A = make_pv(P, a, oax, oay), B = make_pv(R, b, oax, oay);
  double tol = std::fmax(rp.tol_abs, (double)rp.tol_rel * std::fmax(ov.x1 - ov.x0, ov.y1 - ov.y0));
  const double snap = rp.snap_half_ulp ? pair_snap(oax, oay, eax, eay) : 0.0;
  collect(A, ov, LA); collect(B, ov, LB);
  const int na = (int)LA.size(), nb = (int)LB.size();
  bool hit = false, hit_any = false;
  for (int i = 0; i < na && !hit; i++) {
    const Ed& e = LA[i];
    double ax0 = std::fmin(e.x0, e.x1), ax1 = std::fmax(e.x0, e.x1), ay0 = std::fmin(e.y0, e.y1), ay1 = std::fmax(e.y0, e.y1);
    for (int j = 0; j < nb; j++) {
      const Ed& f = LB[j];
      if (std::fmax(f.x0, f.x1) < ax0 || std::fmin(f.x0, f.x1) > ax1 || std::fmax(f.y0, f.y1) < ay0 || std::fmin(f.y0, f.y1) > ay1) continue;
      if (seg_isect(e.x0, e.y0, e.x1, e.y1, f.x0, f.y0, f.x1, f.y1)) {
        hit_any = true;
        if (!(e.syn | f.syn)) { hit = true; break; }
      }
    }
  }
  hit_any = hit_any || hit;
  const bool rtouch = hit;
  double cx = (double)(ov.x0 + 0.381966 * (ov.x1 - ov.x0)), cy = (double)(ov.y0 + 0.414213 * (ov.y1 - ov.y0));
  bool inB_c = false, inA_c = false;
  if (!hit || rp.want_area || rp.want_relate) { inB_c = pip_full(B, cx, cy); inA_c = pip_full(A, cx, cy); }
  bool contain_any = false;
  if (!hit) {
    bool h = false, ha = false;
    for (int side = 0; side < 2; side++) {
      const PV& S = side ? B : A;
      const std::vector<Ed>& LO = side ? LA : LB;
      bool in_c = side ? inA_c : inB_c;
      for (uint64_t r = S.r0; r < S.r1; r++) {
        double x, y; bool real = probe_vertex(S, r, x, y);
        if (!real) S.v(S.s->rvo[r], x, y);
        if (x >= ov.x0 && x <= ov.x1 && y >= ov.y0 && y <= ov.y1 && inside_from_c(LO.data(), (int)LO.size(), cx, cy, in_c, x, y)) {
          ha = true; if (real) h = true;
        }
      }
    }
    hit = h; contain_any = ha;
  }
  double ar = 0.0; double e4[4] = {0, 0, 0, 0}; uint32_t eb4 = 0;
  if ((hit || hit_any || contain_any) && (rp.want_area || rp.want_relate)) {
    double s2[32] = {0}, ai[32] = {0}, ao[32] = {0}, bi[32] = {0}, bo[32] = {0};
    uint32_t bits = rtouch ? REL_TOUCH : 0;
    const bool rel = rp.want_relate != 0;
    for (int i = 0; i < na; i++) {
      const Ed& e = LA[i]; int l = i & 31;
      s2[l] += edge_contrib(e.x0, e.y0, e.x1, e.y1, LB.data(), nb, cx, cy, inB_c, ov, tol, (double)rp.eps_par, !e.syn, rel ? &ai[l] : nullptr,
                            &ao[l], &bits, e.cut, snap);
    }
    for (int i = 0; i < nb; i++) {
      const Ed& e = LB[i]; int l = i & 31;
      s2[l] += edge_contrib(e.x0, e.y0, e.x1, e.y1, LA.data(), na, cx, cy, inA_c, ov, tol, (double)rp.eps_par, !e.syn, rel ? &bi[l] : nullptr,
                            &bo[l], &bits, e.cut, snap);
    }
    ar = 0.5 * warp_sum(s2);
    e4[0] = warp_sum(ai); e4[1] = warp_sum(ao); e4[2] = warp_sum(bi); e4[3] = warp_sum(bo);
    eb4 = bits;
  } else if (rtouch) eb4 = REL_TOUCH;
  bool ev_any = e4[0] != 0 || e4[1] != 0 || e4[2] != 0 || e4[3] != 0;
  o.flag = hit ? 1 : ((ar != 0.0 || ev_any) ? 2 : 0);
  o.area = rp.want_area ? ar : 0.0;
  if (rp.want_relate) { for (int k = 0; k < 4; k++) o.ev[k] = e4[k]; o.evb = eb4; }
  return o;
}

inline uint32_t de9im_code(const double* e, uint32_t bits, double LA, double LB) {   // engine.cuh:848-856
  const double ta = 1e-9 * LA, tb = 1e-9 * LB;
  bool aIn = e[0] > ta, aOut = (LA - e[0] - e[1]) > ta, bIn = e[2] > tb, bOut = (LB - e[2] - e[3]) > tb;
  bool same = bits & REL_COIN_SAME, opp = bits & REL_COIN_OPP, touch = bits & REL_TOUCH;
  uint32_t II = (aIn || bIn || same) ? 3 : 0, IB = bIn ? 2 : 0, IE = (aOut || bIn || opp) ? 3 : 0;
  uint32_t BI = aIn ? 2 : 0, BB = (same || opp) ? 2 : (touch ? 1 : 0), BE = aOut ? 2 : 0;
  uint32_t EI = (bOut || aIn || opp) ? 3 : 0, EB = bOut ? 2 : 0, EE = 3;
  return II | IB << 2 | IE << 4 | BI << 6 | BB << 8 | BE << 10 | EI << 12 | EB << 14 | EE << 16;
}

inline int nthreads_or_default(int t) {
#ifdef _OPENMP
  return t > 0 ? t : omp_get_max_threads();
#else
  (void)t; return 1;
#endif
}

// bbox overlap candidates (the set k_traverse reports; engine.cuh:241, 248): uniform grid over R's boxes
inline int64_t candidates_bb(const float* qbb, uint64_t nq, const Set& R, int upper, int nth, uint32_t** out) {
  const uint64_t nr = R.n;
  if (!nq || !nr) { *out = nullptr; return 0; }
  float gx0 = INFINITY, gy0 = INFINITY, gx1 = -INFINITY, gy1 = -INFINITY;
  for (uint64_t i = 0; i < nr; i++) {
    gx0 = std::min(gx0, R.bb[4 * i]); gy0 = std::min(gy0, R.bb[4 * i + 1]); gx1 = std::max(gx1, R.bb[4 * i + 2]); gy1 = std::max(gy1, R.bb[4 * i + 3]);
  }
  int G = std::max(1, (int)std::sqrt((double)nr / 2.0));
  double wx = ((double)gx1 - gx0) / G, wy = ((double)gy1 - gy0) / G;
  if (!(wx > 0)) wx = 1; if (!(wy > 0)) wy = 1;
  auto cxr = [&](double x) { int c = (int)std::floor((x - gx0) / wx); return std::min(G - 1, std::max(0, c)); };
  auto cyr = [&](double y) { int c = (int)std::floor((y - gy0) / wy); return std::min(G - 1, std::max(0, c)); };
  std::vector<uint32_t> cnt((size_t)G * G + 1, 0);
  for (uint64_t i = 0; i < nr; i++)
    for (int y = cyr(R.bb[4 * i + 1]); y <= cyr(R.bb[4 * i + 3]); y++)
      for (int x = cxr(R.bb[4 * i]); x <= cxr(R.bb[4 * i + 2]); x++) cnt[(size_t)y * G + x + 1]++;
  for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
  std::vector<uint32_t> cell(cnt.back());
  { std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (uint64_t i = 0; i < nr; i++)
      for (int y = cyr(R.bb[4 * i + 1]); y <= cyr(R.bb[4 * i + 3]); y++)
        for (int x = cxr(R.bb[4 * i]); x <= cxr(R.bb[4 * i + 2]); x++) cell[fill[(size_t)y * G + x]++] = (uint32_t)i; }
  const int64_t CH = 4096;
  int64_t nch = ((int64_t)nq + CH - 1) / CH;
  std::vector<std::vector<uint32_t>> parts(nch);
#pragma omp parallel num_threads(nth)
  {
    std::vector<uint32_t> stamp(nr, UINT32_MAX), tmp;
#pragma omp for schedule(dynamic, 1)
    for (int64_t c = 0; c < nch; c++) {
      auto& o = parts[c];
      for (uint64_t q = (uint64_t)c * CH; q < std::min<uint64_t>(nq, (uint64_t)(c + 1) * CH); q++) {
        const float* b = qbb + 4 * q;
        if (b[0] > gx1 || b[2] < gx0 || b[1] > gy1 || b[3] < gy0) continue;
        tmp.clear();
        for (int y = cyr(b[1]); y <= cyr(b[3]); y++)
          for (int x = cxr(b[0]); x <= cxr(b[2]); x++)
            for (uint32_t k = cnt[(size_t)y * G + x]; k < cnt[(size_t)y * G + x + 1]; k++) {
              uint32_t l = cell[k];
              if (stamp[l] == (uint32_t)q) continue;
              stamp[l] = (uint32_t)q;
              const float* c4 = R.bb.data() + 4 * (size_t)l;
              if (c4[0] > b[2] || c4[2] < b[0] || c4[1] > b[3] || c4[3] < b[1]) continue;
              if (upper && l < q) continue;
              tmp.push_back(l);
            }
        std::sort(tmp.begin(), tmp.end());
        for (uint32_t l : tmp) { o.push_back((uint32_t)q); o.push_back(l); }
      }
    }
  }
  size_t tot = 0; for (auto& v : parts) tot += v.size();
  uint32_t* r = (uint32_t*)malloc(sizeof(uint32_t) * (tot ? tot : 1));
  size_t off = 0; for (auto& v : parts) { memcpy(r + off, v.data(), v.size() * 4); off += v.size(); }
  *out = r;
  return (int64_t)(tot / 2);
}


}  // namespace orc

struct orc_set { orc::Set s; };
