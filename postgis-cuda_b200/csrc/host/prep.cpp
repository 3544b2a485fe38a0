// Host-side layer preparation: subdivision of large polygons into pieces (the reference's ST_Subdivide analogue,
// engine/subdivide.h of landstats-us/postgis-cuda) and exact deduplication of identical geometries
// (engine/dedup.h). C++17 + OpenMP, FP64; compiled without FMA contraction so the cut points are the reference's.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>
#include "../../../include/gsj.h"

namespace {

struct Ring { std::vector<double> xy; std::vector<uint8_t> syn; };   // closed; syn[i]: edge i -> i+1 is a cut

// Sutherland-Hodgman clip of a closed ring against the half-plane coord[axis] <= m (le) or >= m (subdivide.h:16-48)
void clip_ring(const Ring& r, int axis, double m, bool le, Ring& out) {
  out.xy.clear(); out.syn.clear();
  const size_t n = r.xy.size() / 2;
  auto inside = [&](size_t i) { const double v = r.xy[2 * i + axis]; return le ? v <= m : v >= m; };
  auto push = [&](double x, double y, uint8_t f) {
    const size_t k = out.xy.size();
    if (k >= 2 && out.xy[k - 2] == x && out.xy[k - 1] == y) { out.syn.back() = f; return; }   // repeated point: keep one
    out.xy.push_back(x); out.xy.push_back(y); out.syn.push_back(f);
  };
  for (size_t i = 0; i + 1 < n; i++) {
    const double px = r.xy[2 * i], py = r.xy[2 * i + 1], qx = r.xy[2 * i + 2], qy = r.xy[2 * i + 3];
    const bool pin = inside(i), qin = inside(i + 1);
    const uint8_t f = r.syn[i];
    auto cut = [&](double& ix, double& iy) {
      if (axis == 0) { ix = m; iy = py + (m - px) * (qy - py) / (qx - px); }
      else { iy = m; ix = px + (m - py) * (qx - px) / (qy - py); }
    };
    if (pin) push(px, py, f);
    if (pin && !qin) { double ix, iy; cut(ix, iy); push(ix, iy, 1); }        // leaving: the next edge runs along the cut
    else if (!pin && qin) { double ix, iy; cut(ix, iy); push(ix, iy, f); }   // entering
  }
  size_t k = out.xy.size() / 2;
  if (k < 3) { out.xy.clear(); out.syn.clear(); return; }
  if (out.xy[0] != out.xy[2 * k - 2] || out.xy[1] != out.xy[2 * k - 1]) { out.xy.push_back(out.xy[0]); out.xy.push_back(out.xy[1]); out.syn.push_back(0); }
  else out.syn.back() = 0;
  k = out.xy.size() / 2;
  double a = 0;
  for (size_t i = 0; i + 1 < k; i++) a += out.xy[2 * i] * out.xy[2 * i + 3] - out.xy[2 * i + 2] * out.xy[2 * i + 1];
  if (k < 4 || a == 0.0) { out.xy.clear(); out.syn.clear(); }   // degenerate slivers are dropped
}

size_t nverts(const std::vector<Ring>& p) { size_t n = 0; for (auto& r : p) n += r.xy.size() / 2; return n; }

// halve the bbox's longer side until a piece has at most maxv vertices (subdivide.h:52-67)
void subdivide_rec(std::vector<Ring>& rings, int maxv, int depth, std::vector<std::vector<Ring>>& out) {
  const size_t nv = nverts(rings);
  if (nv == 0) return;
  double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
  for (auto& r : rings)
    for (size_t i = 0; i < r.xy.size(); i += 2) {
      x0 = std::min(x0, r.xy[i]); x1 = std::max(x1, r.xy[i]); y0 = std::min(y0, r.xy[i + 1]); y1 = std::max(y1, r.xy[i + 1]);
    }
  if ((int)nv <= maxv || depth >= 24 || (x1 - x0 <= 0 && y1 - y0 <= 0)) { out.push_back(std::move(rings)); return; }
  const int axis = (x1 - x0) >= (y1 - y0) ? 0 : 1;
  const double m = axis == 0 ? 0.5 * (x0 + x1) : 0.5 * (y0 + y1);
  for (int side = 0; side < 2; side++) {
    std::vector<Ring> part; Ring c;
    for (auto& r : rings) { clip_ring(r, axis, m, side == 0, c); if (!c.xy.empty()) part.push_back(c); }
    if (!part.empty()) subdivide_rec(part, maxv, depth + 1, out);
  }
}

template <class T> T* dup(const std::vector<T>& v) {
  T* p = (T*)malloc(sizeof(T) * (v.empty() ? 1 : v.size()));
  if (!p) return nullptr;
  if (!v.empty()) memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

uint64_t mix_hash(const uint64_t* gro, const uint64_t* rvo, const double* xy, uint64_t g) {   // order-sensitive hash of one geometry
  uint64_t h = 0x9E3779B97F4A7C15ull ^ (gro[g + 1] - gro[g]);
  for (uint64_t r = gro[g]; r < gro[g + 1]; r++) {
    h = (h ^ (rvo[r + 1] - rvo[r])) * 0xBF58476D1CE4E5B9ull;
    const uint64_t* w = reinterpret_cast<const uint64_t*>(xy + 2 * rvo[r]);
    for (uint64_t i = 0; i < 2 * (rvo[r + 1] - rvo[r]); i++) { h ^= w[i]; h *= 0x94D049BB133111EBull; h ^= h >> 31; }
  }
  return h;
}
bool same_geom(const uint64_t* gro, const uint64_t* rvo, const double* xy, uint64_t a, uint64_t b) {
  if (gro[a + 1] - gro[a] != gro[b + 1] - gro[b]) return false;
  for (uint64_t k = 0; k < gro[a + 1] - gro[a]; k++)
    if (rvo[gro[a] + k + 1] - rvo[gro[a] + k] != rvo[gro[b] + k + 1] - rvo[gro[b] + k]) return false;
  const uint64_t va = rvo[gro[a]], vb = rvo[gro[b]], nv = rvo[gro[a + 1]] - va;
  return memcmp(xy + 2 * va, xy + 2 * vb, nv * 16) == 0;
}
uint64_t spread32(uint64_t v) {
  v &= 0xFFFFFFFFull;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull; v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full; v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull; return v;
}

}  // namespace

extern "C" {

int gsj_subdivide(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv, uint64_t* out_n,
                  uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint32_t** out_parent,
                  uint8_t** out_syn) {
  if (!gro || !rvo || !xy || maxv < 4 || !out_n || !out_nr || !out_nv || !out_gro || !out_rvo || !out_xy || !out_parent || !out_syn) return GSJ_ERR_ARG;
  if (n >= (1ull << 32) || gro[n] != nr || rvo[nr] != nv) return GSJ_ERR_ARG;
  const int64_t CH = 1 << 14;
  const int64_t nch = ((int64_t)n + CH - 1) / CH;
  struct Frag { std::vector<uint64_t> gro{0}, rvo{0}; std::vector<double> xy; std::vector<uint8_t> syn; std::vector<uint32_t> parent; };
  std::vector<Frag> frags(nch);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c = 0; c < nch; c++) {
    Frag& f = frags[c];
    std::vector<std::vector<Ring>> pieces;
    for (int64_t g = c * CH; g < std::min<int64_t>((int64_t)n, (c + 1) * CH); g++) {
      const uint64_t r0 = gro[g], r1 = gro[g + 1];
      if ((int64_t)(rvo[r1] - rvo[r0]) <= maxv) {   // small geometry: one piece, unchanged
        for (uint64_t r = r0; r < r1; r++) {
          f.xy.insert(f.xy.end(), xy + 2 * rvo[r], xy + 2 * rvo[r + 1]);
          f.syn.insert(f.syn.end(), rvo[r + 1] - rvo[r], 0);
          f.rvo.push_back(f.xy.size() / 2);
        }
        f.gro.push_back(f.rvo.size() - 1); f.parent.push_back((uint32_t)g);
        continue;
      }
      std::vector<Ring> rings;
      for (uint64_t r = r0; r < r1; r++) {
        Ring sr; sr.xy.assign(xy + 2 * rvo[r], xy + 2 * rvo[r + 1]); sr.syn.assign(rvo[r + 1] - rvo[r], 0);
        rings.push_back(std::move(sr));
      }
      pieces.clear();
      subdivide_rec(rings, maxv, 0, pieces);
      for (auto& p : pieces) {
        for (auto& r : p) { f.xy.insert(f.xy.end(), r.xy.begin(), r.xy.end()); f.syn.insert(f.syn.end(), r.syn.begin(), r.syn.end()); f.rvo.push_back(f.xy.size() / 2); }
        f.gro.push_back(f.rvo.size() - 1); f.parent.push_back((uint32_t)g);
      }
    }
  }
  std::vector<uint64_t> og{0}, orv{0}; std::vector<double> oxy; std::vector<uint8_t> osyn; std::vector<uint32_t> opar;
  for (auto& f : frags) {
    const uint64_t rb = orv.size() - 1, vb = oxy.size() / 2;
    for (size_t i = 1; i < f.gro.size(); i++) og.push_back(rb + f.gro[i]);
    for (size_t i = 1; i < f.rvo.size(); i++) orv.push_back(vb + f.rvo[i]);
    oxy.insert(oxy.end(), f.xy.begin(), f.xy.end());
    osyn.insert(osyn.end(), f.syn.begin(), f.syn.end());
    opar.insert(opar.end(), f.parent.begin(), f.parent.end());
  }
  *out_n = opar.size(); *out_nr = orv.size() - 1; *out_nv = oxy.size() / 2;
  *out_gro = dup(og); *out_rvo = dup(orv); *out_xy = dup(oxy); *out_parent = dup(opar); *out_syn = dup(osyn);
  if (!*out_gro || !*out_rvo || !*out_xy || !*out_parent || !*out_syn) return GSJ_ERR_NOMEM;
  return GSJ_OK;
}

int gsj_dedup(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton, uint64_t* out_n,
              uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint64_t** out_moff, uint32_t** out_midx) {
  if (!gro || !rvo || !xy || !out_n || !out_gro || !out_rvo || !out_xy || !out_moff || !out_midx) return GSJ_ERR_ARG;
  if (n >= (1ull << 32) || gro[n] != nr || rvo[nr] != nv) return GSJ_ERR_ARG;
  std::vector<uint64_t> h(n);
#pragma omp parallel for schedule(static)
  for (int64_t g = 0; g < (int64_t)n; g++) h[g] = mix_hash(gro, rvo, xy, (uint64_t)g);
  std::vector<uint32_t> ord(n);
  std::iota(ord.begin(), ord.end(), 0u);
  std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return h[a] != h[b] ? h[a] < h[b] : a < b; });
  std::vector<uint32_t> rep(n);   // lowest-index geometry identical to g
  for (uint64_t i = 0; i < n;) {
    uint64_t j = i;
    while (j < n && h[ord[j]] == h[ord[i]]) j++;
    for (uint64_t k = i; k < j; k++) {
      const uint32_t g = ord[k]; rep[g] = g;
      for (uint64_t q = i; q < k; q++) if (rep[ord[q]] == ord[q] && same_geom(gro, rvo, xy, ord[q], g)) { rep[g] = ord[q]; break; }
    }
    i = j;
  }
  std::vector<uint32_t> first, uid(n, UINT32_MAX);
  for (uint64_t g = 0; g < n; g++) if (rep[g] == g) { uid[g] = (uint32_t)first.size(); first.push_back((uint32_t)g); }
  const uint64_t un = first.size();
  if (morton && un > 1) {   // distinct geometries in Z-order of their bbox centres (dedup.h:81-96)
    std::vector<double> cx(un), cy(un);
    for (uint64_t i = 0; i < un; i++) {
      const uint32_t g = first[i];
      double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
      for (uint64_t v = rvo[gro[g]]; v < rvo[gro[g + 1]]; v++) { x0 = std::min(x0, xy[2 * v]); x1 = std::max(x1, xy[2 * v]); y0 = std::min(y0, xy[2 * v + 1]); y1 = std::max(y1, xy[2 * v + 1]); }
      cx[i] = 0.5 * (x0 + x1); cy[i] = 0.5 * (y0 + y1);
    }
    const double mx0 = *std::min_element(cx.begin(), cx.end()), mx1 = *std::max_element(cx.begin(), cx.end());
    const double my0 = *std::min_element(cy.begin(), cy.end()), my1 = *std::max_element(cy.begin(), cy.end());
    const double sx = mx1 > mx0 ? 4294967295.0 / (mx1 - mx0) : 0, sy = my1 > my0 ? 4294967295.0 / (my1 - my0) : 0;
    std::vector<std::pair<uint64_t, uint32_t>> key(un);
    for (uint64_t i = 0; i < un; i++) key[i] = {(spread32((uint64_t)((cx[i] - mx0) * sx)) << 1) | spread32((uint64_t)((cy[i] - my0) * sy)), first[i]};
    std::sort(key.begin(), key.end());
    for (uint64_t i = 0; i < un; i++) { first[i] = key[i].second; uid[first[i]] = (uint32_t)i; }
  }
  std::vector<uint64_t> moff(un + 1, 0);
  for (uint64_t g = 0; g < n; g++) moff[uid[rep[g]] + 1]++;
  for (uint64_t i = 0; i < un; i++) moff[i + 1] += moff[i];
  std::vector<uint32_t> midx(n);
  { std::vector<uint64_t> fill(moff.begin(), moff.end() - 1); for (uint64_t g = 0; g < n; g++) midx[fill[uid[rep[g]]]++] = (uint32_t)g; }
  std::vector<uint64_t> og(un + 1, 0), ov(un + 1, 0);
  for (uint64_t i = 0; i < un; i++) {
    const uint32_t g = first[i];
    og[i + 1] = og[i] + (gro[g + 1] - gro[g]);
    ov[i + 1] = ov[i] + (rvo[gro[g + 1]] - rvo[gro[g]]);
  }
  std::vector<uint64_t> orv(og[un] + 1); std::vector<double> oxy(2 * ov[un]);
  for (uint64_t i = 0; i < un; i++) {
    const uint32_t g = first[i];
    const uint64_t r0 = gro[g], vb = rvo[r0];
    for (uint64_t r = r0; r < gro[g + 1]; r++) orv[og[i] + (r - r0)] = ov[i] + (rvo[r] - vb);
    memcpy(oxy.data() + 2 * ov[i], xy + 2 * vb, (ov[i + 1] - ov[i]) * 16);
  }
  orv[og[un]] = ov[un];
  *out_n = un; if (out_nr) *out_nr = og[un]; if (out_nv) *out_nv = ov[un];
  *out_gro = dup(og); *out_rvo = dup(orv); *out_xy = dup(oxy); *out_moff = dup(moff); *out_midx = dup(midx);
  if (!*out_gro || !*out_rvo || !*out_xy || !*out_moff || !*out_midx) return GSJ_ERR_NOMEM;
  return GSJ_OK;
}

void gsj_host_free(void* p) { free(p); }

}  // extern "C"
