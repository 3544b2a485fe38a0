// CPU FP64 oracle - TEST INFRASTRUCTURE ONLY (see oracle.h). Build: oracle/Makefile (g++ -O2 -ffp-contract=off
// -fopenmp). Every function cites the reference file:line it restates; the reference is
// landstats-us/postgis-cuda, paths relative to that project.
#include "oracle.h"
#include "oracle_internal.h"

using namespace orc;
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
