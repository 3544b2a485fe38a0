// CPU FP64 oracle - TEST INFRASTRUCTURE ONLY (see oracle.h). Build: oracle/Makefile (g++ -O2 -ffp-contract=off
// -fopenmp). Every function cites the reference file:line it restates; the reference is
// landstats-us/postgis-cuda, paths relative to that project.
#include "oracle.h"
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

namespace {

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
double edge_contrib(double px, double py, double qx, double qy, const Ed* L, int cnt, double cx, double cy, bool in_c, const Ov& ov,
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
PairOut refine_pair(const Set& P, const Set& R, uint32_t a, uint32_t b, const orc_params& rp, std::vector<Ed>& LA, std::vector<Ed>& LB) {
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

int nthreads_or_default(int t) {
#ifdef _OPENMP
  return t > 0 ? t : omp_get_max_threads();
#else
  (void)t; return 1;
#endif
}

// bbox overlap candidates (the set k_traverse reports; engine.cuh:241, 248): uniform grid over R's boxes
int64_t candidates_bb(const float* qbb, uint64_t nq, const Set& R, int upper, int nth, uint32_t** out) {
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

}  // namespace

struct orc_set { Set s; };

extern "C" {

orc_set* orc_set_create(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy,
                        const uint32_t* parent, const uint8_t* syn) {
  orc_set* o = new orc_set();
  Set& s = o->s;
  s.n = n; s.nr = nr; s.nv = nv;
  s.gro.assign(gro, gro + n + 1); s.rvo.assign(rvo, rvo + nr + 1);
  s.q.resize(2 * nv); s.ox.resize(n); s.oy.resize(n); s.ex.resize(n); s.ey.resize(n); s.bb.resize(4 * n);
  // upload_set (engine.cuh:49-64)
  for (uint64_t g = 0; g < n; g++) {
    uint64_t v0 = rvo[gro[g]], v1 = rvo[gro[g + 1]];
    double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
    for (uint64_t v = v0; v < v1; v++) {
      double x = xy[2 * v], y = xy[2 * v + 1];
      x0 = std::min(x0, x); x1 = std::max(x1, x); y0 = std::min(y0, y); y1 = std::max(y1, y);
    }
    s.ox[g] = x0; s.oy[g] = y0; s.ex[g] = x1 - x0; s.ey[g] = y1 - y0;
    s.bb[4 * g] = f_down(x0); s.bb[4 * g + 1] = f_down(y0); s.bb[4 * g + 2] = f_up(x1); s.bb[4 * g + 3] = f_up(y1);
    for (uint64_t v = v0; v < v1; v++) { s.q[2 * v] = xy[2 * v] - x0; s.q[2 * v + 1] = xy[2 * v + 1] - y0; }
  }
  if (parent) { s.has_parent = true; s.parent.assign(parent, parent + n); }
  if (syn) { s.has_syn = true; s.syn.assign(syn, syn + nv); }
  s.nparent = parent ? (n ? parent[n - 1] + 1 : 0) : (uint32_t)n;
  // real boundary length per parent (engine.cuh:69-82)
  s.blen.assign(s.nparent, 0.0);
  for (uint64_t g = 0; g < n; g++) {
    double L = 0;
    for (uint64_t r = gro[g]; r < gro[g + 1]; r++)
      for (uint64_t v = rvo[r]; v + 1 < rvo[r + 1]; v++)
        if (!syn || !syn[v]) L += std::hypot(xy[2 * v + 2] - xy[2 * v], xy[2 * v + 3] - xy[2 * v + 1]);
    s.blen[parent ? parent[g] : g] += L;
  }
  return o;
}

void orc_set_free(orc_set* s) { delete s; }
void orc_set_bbox(const orc_set* s, float* bb4) { memcpy(bb4, s->s.bb.data(), s->s.bb.size() * sizeof(float)); }
void orc_free(void* p) { free(p); }
double orc_blen(const orc_set* s, uint32_t p) { return s->s.blen[p]; }

int64_t orc_candidates(const orc_set* P, const orc_set* R, int upper, uint32_t** out) {
  return candidates_bb(P->s.bb.data(), P->s.n, R->s, upper, nthreads_or_default(0), out);
}
int64_t orc_candidates_bb(const float* qbb4, uint64_t nq, const orc_set* R, int upper, uint32_t** out) {
  return candidates_bb(qbb4, nq, R->s, upper, nthreads_or_default(0), out);
}

void orc_refine_pairs(const orc_set* P, const orc_set* R, const uint32_t* pairs, int64_t np, const orc_params* rp, uint8_t* flag,
                      double* area, double* ev, uint32_t* evb, int nthreads) {
  int nth = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nth)
  {
    std::vector<Ed> LA, LB;
#pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < np; i++) {
      PairOut o = refine_pair(P->s, R->s, pairs[2 * i], pairs[2 * i + 1], *rp, LA, LB);
      if (flag) flag[i] = o.flag;
      if (area) area[i] = o.area;
      if (ev) for (int k = 0; k < 4; k++) ev[4 * i + k] = o.ev[k];
      if (evb) evb[i] = o.evb;
    }
  }
}

uint32_t orc_de9im_code(const double* ev4, uint32_t bits, double la, double lb) { return de9im_code(ev4, bits, la, lb); }
uint32_t orc_de9im_transpose(uint32_t c) {   // engine.cuh:872-876
  uint32_t t = 0;
  for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) t |= ((c >> (2 * (3 * r + q))) & 3) << (2 * (3 * q + r));
  return t;
}
int orc_de9im_match(uint32_t code, const char* pat) {   // engine.cuh:878-888
  for (int k = 0; k < 9; k++) {
    char p = pat[k]; uint32_t v = (code >> (2 * k)) & 3;
    if (p == '*') continue;
    if (p == 'T' || p == 't') { if (v == 0) return 0; continue; }
    if (p == 'F' || p == 'f') { if (v != 0) return 0; continue; }
    if (p >= '0' && p <= '2') { if (v != (uint32_t)(p - '0') + 1) return 0; continue; }
    return 0;
  }
  return 1;
}

// join_stream semantics (engine.cuh:963-1042): no pieces: keep flag 1; pieces: keep flags 1|2, fold per parent
// pair (area sum, Sum4, BitOr, min flag; summed in (parent pair, piece a, piece b) order), keep min flag == 1.
int64_t orc_join(const orc_set* P, const orc_set* R, const orc_params* rp, int upper, int nthreads, uint32_t** out_pairs, double** out_area,
                 uint32_t** out_code, int64_t* n_candidates) {
  int nth = nthreads_or_default(nthreads);
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(P->s.bb.data(), P->s.n, R->s, upper, nth, &cand);
  if (n_candidates) *n_candidates = nc;
  std::vector<uint8_t> flag(nc); std::vector<double> area(nc), ev(4 * (size_t)nc); std::vector<uint32_t> evb(nc);
  orc_refine_pairs(P, R, cand, nc, rp, flag.data(), area.data(), ev.data(), evb.data(), nth);
  const bool agg = P->s.has_parent || R->s.has_parent;
  struct Row { uint32_t a, b; double area; double ev[4]; uint32_t bits; uint8_t flag; };
  std::vector<Row> rows;
  if (!agg) {
    for (int64_t i = 0; i < nc; i++) if (flag[i] == 1)
      rows.push_back(Row{cand[2 * i], cand[2 * i + 1], area[i], {ev[4 * i], ev[4 * i + 1], ev[4 * i + 2], ev[4 * i + 3]}, evb[i], 1});
  } else {
    std::vector<int64_t> idx;
    for (int64_t i = 0; i < nc; i++) if (flag[i] != 0) idx.push_back(i);
    auto key = [&](int64_t i) { return ((uint64_t)P->s.pid(cand[2 * i]) << 32) | R->s.pid(cand[2 * i + 1]); };
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return key(x) < key(y); });
    for (size_t k = 0; k < idx.size();) {
      size_t m = k; uint64_t kk = key(idx[k]);
      Row r{(uint32_t)(kk >> 32), (uint32_t)kk, 0.0, {0, 0, 0, 0}, 0, 255};
      for (; m < idx.size() && key(idx[m]) == kk; m++) {
        int64_t i = idx[m];
        r.area += area[i];
        for (int q = 0; q < 4; q++) r.ev[q] += ev[4 * i + q];
        r.bits |= evb[i]; r.flag = std::min(r.flag, flag[i]);
      }
      if (r.flag == 1) rows.push_back(r);
      k = m;
    }
  }
  free(cand);
  int64_t n = (int64_t)rows.size();
  uint32_t* op = (uint32_t*)malloc(8 * (n ? n : 1)); double* oa = (double*)malloc(8 * (n ? n : 1)); uint32_t* oc = (uint32_t*)malloc(4 * (n ? n : 1));
  for (int64_t i = 0; i < n; i++) {
    op[2 * i] = rows[i].a; op[2 * i + 1] = rows[i].b; oa[i] = rows[i].area;
    oc[i] = rp->want_relate ? de9im_code(rows[i].ev, rows[i].bits, P->s.blen[rows[i].a], R->s.blen[rows[i].b]) : 0;
  }
  *out_pairs = op; *out_area = oa; *out_code = oc;
  return n;
}

// k_pip_pairs (engine.cuh:1079-1106) + join_points_stream folding (engine.cuh:1147-1163)
int64_t orc_pip(const double* pts, uint64_t npts, const orc_set* Ro, int nthreads, uint32_t** out_pairs, uint8_t** out_where, int64_t* n_candidates) {
  const Set& R = Ro->s;
  int nth = nthreads_or_default(nthreads);
  std::vector<float> qbb(4 * npts);
  for (uint64_t i = 0; i < npts; i++) { qbb[4 * i] = f_down(pts[2 * i]); qbb[4 * i + 1] = f_down(pts[2 * i + 1]); qbb[4 * i + 2] = f_up(pts[2 * i]); qbb[4 * i + 3] = f_up(pts[2 * i + 1]); }
  uint32_t* cand = nullptr;
  int64_t nc = candidates_bb(qbb.data(), npts, R, 0, nth, &cand);
  if (n_candidates) *n_candidates = nc;
  std::vector<uint8_t> hit(nc);
#pragma omp parallel for num_threads(nth) schedule(dynamic, 1024)
  for (int64_t i = 0; i < nc; i++) {
    uint32_t p = cand[2 * i], g = cand[2 * i + 1];
    PV B = make_pv(R, g, R.ox[g], R.oy[g]);
    double px = (double)(pts[2 * p] - R.ox[g]), py = (double)(pts[2 * p + 1] - R.oy[g]);
    double ox = B.shx - (double)1;
    bool par = false, on = false;
    for (uint64_t r = B.r0; r < B.r1 && !on; r++) {
      uint64_t s0 = R.rvo[r], e = R.rvo[r + 1];
      double x0, y0; B.v(s0, x0, y0);
      for (uint64_t j = s0 + 1; j < e; j++) {
        double x1, y1; B.v(j, x1, y1);
        if (!((y0 > py) == (y1 > py) && y0 != py && y1 != py)) {
          double o_ = orient(x0, y0, x1, y1, px, py);
          if (o_ == 0 && !B.syn(j - 1) && onseg(x0, y0, x1, y1, px, py)) { on = true; break; }
          bool so = left_of(x0, y0, x1, y1, ox, py), sp = left_of(x0, y0, x1, y1, px, py);
          if (so != sp) {
            bool su = orient(ox, py, px, py, x0, y0) > 0, sv = orient(ox, py, px, py, x1, y1) > 0;
            if (su != sv) par = !par;
          }
        }
        x0 = x1; y0 = y1;
      }
    }
    hit[i] = on ? 2 : (par ? 1 : 0);
  }
  std::vector<std::pair<uint64_t, uint8_t>> kv;
  for (int64_t i = 0; i < nc; i++) if (hit[i]) kv.push_back({((uint64_t)cand[2 * i] << 32) | R.pid(cand[2 * i + 1]), hit[i]});
  free(cand);
  std::sort(kv.begin(), kv.end());
  std::vector<std::pair<uint64_t, uint8_t>> u;
  for (auto& e : kv) { if (!u.empty() && u.back().first == e.first) u.back().second = std::max(u.back().second, e.second); else u.push_back(e); }
  int64_t n = (int64_t)u.size();
  uint32_t* op = (uint32_t*)malloc(8 * (n ? n : 1)); uint8_t* ow = (uint8_t*)malloc(n ? n : 1);
  for (int64_t i = 0; i < n; i++) { op[2 * i] = (uint32_t)(u[i].first >> 32); op[2 * i + 1] = (uint32_t)u[i].first; ow[i] = u[i].second; }
  *out_pairs = op; *out_where = ow;
  return n;
}

// cluster_intersecting (engine.cuh:1216-1234): components of the intersects graph over parents
void orc_cluster(const orc_set* P, uint32_t nparent, const orc_params* rp0, int nthreads, uint32_t* root) {
  orc_params rp = *rp0; rp.want_area = 0; rp.want_relate = 0;
  uint32_t* pairs = nullptr; double* area = nullptr; uint32_t* code = nullptr;
  int64_t n = orc_join(P, P, &rp, 1, nthreads, &pairs, &area, &code, nullptr);
  std::vector<uint32_t> par(nparent);
  std::iota(par.begin(), par.end(), 0u);
  auto find = [&](uint32_t x) { while (par[x] != x) { par[x] = par[par[x]]; x = par[x]; } return x; };
  for (int64_t i = 0; i < n; i++) {
    uint32_t a = find(pairs[2 * i]), b = find(pairs[2 * i + 1]);
    if (a == b) continue;
    if (a > b) std::swap(a, b);
    par[b] = a;
  }
  for (uint32_t g = 0; g < nparent; g++) root[g] = find(g);
  free(pairs); free(area); free(code);
}

}  // extern "C"
