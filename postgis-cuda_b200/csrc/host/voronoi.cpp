// Synthetic Voronoi parcel layers (see gsjgen.h). Host C++17 + OpenMP; compiled with -ffp-contract=off so
// the output is a pure function of the parameters.
//
// Cell construction: the box is clipped by the bisector half-planes of nearby seeds (bucket grid, searched in
// growing rings until the cell's circumradius proves the rest cannot cut it). A cell is a cyclic list of
// constraint lines (bisector with seed j, or a box side); vertex k is the intersection of lines k-1 and k and
// is named by its sorted set of defining seeds/sides. Coordinates and the clip predicate are evaluated only
// from that canonical name, so two cells that share a vertex compute the same double values and take the same
// keep/remove decisions.
#include "gsjgen.h"
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
inline double u01(uint64_t seed, uint64_t idx, uint64_t tag) {
  uint64_t h = splitmix64(seed ^ splitmix64(idx * 0x632BE59BD9B4E019ull + tag));
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// Vertex name: sorted triple; sides are encoded as negative ids -1..-4 (0 bottom, 1 right, 2 top, 3 left).
struct Key {
  int64_t k[3];
  bool operator<(const Key& o) const { return k[0] != o.k[0] ? k[0] < o.k[0] : (k[1] != o.k[1] ? k[1] < o.k[1] : k[2] < o.k[2]); }
  bool operator==(const Key& o) const { return k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2]; }
};
inline int64_t side_id(int s) { return -1 - (int64_t)s; }

struct Gen {
  gsjgen_params p;
  std::vector<double> sx, sy;
  int nbx = 1, nby = 1; double bsx = 1, bsy = 1;
  std::vector<uint32_t> bstart, bidx;

  void seeds() {
    sx.resize(p.n); sy.resize(p.n);
    const double W = p.x1 - p.x0, H = p.y1 - p.y0;
    if (p.jitter_grid) {
      uint64_t m = (uint64_t)std::ceil(std::sqrt((double)p.n * W / H));
      if (m < 1) m = 1;
      uint64_t rows = (p.n + m - 1) / m;
      const double cw = W / (double)m, ch = H / (double)rows;
      for (uint64_t i = 0; i < p.n; i++) {
        uint64_t r = i / m, c = i % m;
        double jx = (u01(p.seed, i, 1) * 2.0 - 1.0) * p.jitter, jy = (u01(p.seed, i, 2) * 2.0 - 1.0) * p.jitter;
        sx[i] = p.x0 + ((double)c + 0.5 + jx) * cw;
        sy[i] = p.y0 + ((double)r + 0.5 + jy) * ch;
      }
    } else {
      for (uint64_t i = 0; i < p.n; i++) {
        sx[i] = p.x0 + u01(p.seed, i, 1) * W;
        sy[i] = p.y0 + u01(p.seed, i, 2) * H;
      }
    }
    // bucket grid, ~1 seed per bucket
    double per = std::sqrt(W * H / (double)p.n);
    nbx = std::max(1, (int)std::floor(W / per)); nby = std::max(1, (int)std::floor(H / per));
    bsx = W / nbx; bsy = H / nby;
    std::vector<uint32_t> cnt((size_t)nbx * nby + 1, 0);
    std::vector<uint32_t> b(p.n);
    for (uint64_t i = 0; i < p.n; i++) { b[i] = bucket_of(sx[i], sy[i]); cnt[b[i] + 1]++; }
    for (size_t k = 1; k < cnt.size(); k++) cnt[k] += cnt[k - 1];
    bstart = cnt; bidx.resize(p.n);
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (uint64_t i = 0; i < p.n; i++) bidx[fill[b[i]]++] = (uint32_t)i;   // index order within a bucket
  }
  uint32_t bucket_of(double x, double y) const {
    int bx = std::min(nbx - 1, std::max(0, (int)((x - p.x0) / bsx)));
    int by = std::min(nby - 1, std::max(0, (int)((y - p.y0) / bsy)));
    return (uint32_t)by * nbx + bx;
  }

  // canonical coordinates of a named vertex
  void vcoord(const Key& K, double& x, double& y) const {
    if (K.k[1] < 0) {   // two sides: a box corner
      int s0 = (int)(-1 - K.k[0]), s1 = (int)(-1 - K.k[1]);
      for (int s : {s0, s1}) { if (s == 0) y = p.y0; else if (s == 2) y = p.y1; else if (s == 1) x = p.x1; else x = p.x0; }
      return;
    }
    if (K.k[0] < 0) {   // a side and the bisector of seeds a < b
      int s = (int)(-1 - K.k[0]);
      uint64_t a = (uint64_t)K.k[1], b = (uint64_t)K.k[2];
      double mx = 0.5 * (sx[a] + sx[b]), my = 0.5 * (sy[a] + sy[b]);
      double dx = -(sy[b] - sy[a]), dy = sx[b] - sx[a];   // bisector direction
      if (s == 1 || s == 3) { double X = s == 1 ? p.x1 : p.x0; double t = (X - mx) / dx; x = X; y = my + t * dy; }
      else { double Y = s == 0 ? p.y0 : p.y1; double t = (Y - my) / dy; y = Y; x = mx + t * dx; }
      return;
    }
    // circumcenter of seeds a < b < c, relative to a
    uint64_t a = (uint64_t)K.k[0], b = (uint64_t)K.k[1], c = (uint64_t)K.k[2];
    double bx = sx[b] - sx[a], by = sy[b] - sy[a], cx = sx[c] - sx[a], cy = sy[c] - sy[a];
    double d = 2.0 * (bx * cy - by * cx);
    double b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
    x = sx[a] + (cy * b2 - by * c2) / d;
    y = sy[a] + (bx * c2 - cx * b2) / d;
  }
  // Is the named vertex strictly closer to seed l than to every seed that defines it? (keep/remove decision
  // of a clip by bisector(i, l); depends only on (K, l), so every cell that holds the vertex agrees)
  bool outside(const Key& K, double x, double y, uint64_t l) const {
    double dl = (x - sx[l]) * (x - sx[l]) + (y - sy[l]) * (y - sy[l]);
    double dmin = INFINITY;
    for (int t = 0; t < 3; t++) if (K.k[t] >= 0) {
      uint64_t s = (uint64_t)K.k[t];
      double d = (x - sx[s]) * (x - sx[s]) + (y - sy[s]) * (y - sy[s]);
      dmin = std::min(dmin, d);
    }
    return dl < dmin;
  }

  static Key vkey(uint64_t i, int64_t A, int64_t B) {   // vertex between lines A and B of cell i
    // line ids: >= 0 bisector with that seed, < 0 side
    int64_t v[3];
    if (A < 0 && B < 0) { v[0] = A; v[1] = B; v[2] = (int64_t)i; }
    else if (A < 0 || B < 0) { v[0] = A < 0 ? A : B; v[1] = (int64_t)i; v[2] = A < 0 ? B : A; }
    else { v[0] = (int64_t)i; v[1] = A; v[2] = B; }
    std::sort(v, v + 3);
    return Key{{v[0], v[1], v[2]}};
  }

  struct Cell { std::vector<int64_t> lines; std::vector<Key> keys; std::vector<double> vx, vy; bool bad = false; };

  void refresh(uint64_t i, Cell& c) const {
    size_t m = c.lines.size();
    c.keys.resize(m); c.vx.resize(m); c.vy.resize(m);
    for (size_t k = 0; k < m; k++) {
      c.keys[k] = vkey(i, c.lines[(k + m - 1) % m], c.lines[k]);
      vcoord(c.keys[k], c.vx[k], c.vy[k]);
    }
  }

  void clip(uint64_t i, Cell& c, uint64_t l) const {
    size_t m = c.lines.size();
    std::vector<char> out(m);
    size_t nout = 0;
    for (size_t k = 0; k < m; k++) { out[k] = outside(c.keys[k], c.vx[k], c.vy[k], l); nout += out[k]; }
    if (!nout) return;
    if (nout == m) { c.bad = true; return; }
    size_t k0 = m, starts = 0;
    for (size_t k = 0; k < m; k++) if (out[k] && !out[(k + m - 1) % m]) { if (k0 == m) k0 = k; starts++; }
    if (starts != 1) c.bad = true;
    size_t k1 = k0; while (out[(k1 + 1) % m]) k1 = (k1 + 1) % m;
    std::vector<int64_t> nl;
    // keep lines k1 .. k0-1 (cyclic), then the new line
    for (size_t k = k1; ; k = (k + 1) % m) { nl.push_back(c.lines[k]); if (k == (k0 + m - 1) % m) break; }
    nl.push_back((int64_t)l);
    c.lines.swap(nl);
    refresh(i, c);
  }

  Cell build(uint64_t i) const {
    Cell c; c.lines = {side_id(0), side_id(1), side_id(2), side_id(3)};
    refresh(i, c);
    int bx = std::min(nbx - 1, std::max(0, (int)((sx[i] - p.x0) / bsx)));
    int by = std::min(nby - 1, std::max(0, (int)((sy[i] - p.y0) / bsy)));
    int rmax = std::max(nbx, nby);
    for (int r = 0; r <= rmax; r++) {
      for (int yy = by - r; yy <= by + r; yy++) {
        if (yy < 0 || yy >= nby) continue;
        for (int xx = bx - r; xx <= bx + r; xx++) {
          if (xx < 0 || xx >= nbx) continue;
          if (std::max(std::abs(xx - bx), std::abs(yy - by)) != r) continue;
          uint32_t b = (uint32_t)yy * nbx + xx;
          for (uint32_t k = bstart[b]; k < bstart[b + 1]; k++) if (bidx[k] != i) clip(i, c, bidx[k]);
        }
      }
      double D = (double)r * std::min(bsx, bsy), rad2 = 0;
      for (size_t k = 0; k < c.vx.size(); k++)
        rad2 = std::max(rad2, (c.vx[k] - sx[i]) * (c.vx[k] - sx[i]) + (c.vy[k] - sy[i]) * (c.vy[k] - sy[i]));
      if (4.0 * rad2 < D * D) break;
    }
    return c;
  }
};

inline int target_kappa(const gsjgen_params& p, uint64_t c) {
  double u = u01(p.seed, c, 7);
  double V;
  if (p.log_uniform) V = std::exp(std::log((double)p.vmin) + u * (std::log((double)p.vmax) - std::log((double)p.vmin)));
  else V = (double)p.vmin + u * (double)(p.vmax - p.vmin);
  // a cell has ~6 edges; each edge contributes (1 + kappa) distinct vertices, plus the closing vertex
  int k = (int)std::lround((V - 1.0) / 6.0) - 1;
  return k < 0 ? 0 : k;
}

}  // namespace

extern "C" int gsjgen_voronoi(const gsjgen_params* pp, gsjgen_set* out) {
  if (!pp || !out || pp->n == 0 || !(pp->x1 > pp->x0) || !(pp->y1 > pp->y0) || pp->vmin < 4 || pp->vmax < pp->vmin) return 1;
  memset(out, 0, sizeof(*out));
  Gen G; G.p = *pp;
  G.seeds();
  const uint64_t n = pp->n;
  std::vector<Gen::Cell> cells(n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < (int64_t)n; i++) cells[i] = G.build((uint64_t)i);

  // shared-edge consistency: edge (i, j) must appear in cell j with the endpoint names swapped
  uint64_t bad = 0;
#pragma omp parallel for reduction(+ : bad) schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    const auto& c = cells[i];
    if (c.bad) { bad++; continue; }
    size_t m = c.lines.size();
    for (size_t k = 0; k < m; k++) {
      int64_t j = c.lines[k];
      if (j < 0) continue;
      const Key &a = c.keys[k], &b = c.keys[(k + 1) % m];
      const auto& d = cells[j];
      bool found = false;
      for (size_t q = 0; q < d.lines.size() && !found; q++)
        if (d.lines[q] == i && d.keys[q] == b && d.keys[(q + 1) % d.lines.size()] == a) found = true;
      if (!found) bad++;
    }
  }
  out->n_inconsistent = bad;

  // roles: 0 plain, 1 multipolygon root, 2 consumed part of a multipolygon; holes on plain cells
  std::vector<uint8_t> role(n, 0), hole(n, 0);
  std::vector<std::vector<uint32_t>> parts;
  std::vector<int64_t> mp_of(n, -1);
  auto is_nb = [&](uint64_t a, uint64_t b) {
    for (int64_t l : cells[a].lines) if (l == (int64_t)b) return true;
    return false;
  };
  if (pp->mp_frac > 0) {
    for (uint64_t c = 0; c < n; c++) {
      if (role[c] != 0 || u01(pp->seed, c, 11) >= pp->mp_frac) continue;
      int span = std::max(1, pp->mp_parts_max - pp->mp_parts_min + 1);
      int want = pp->mp_parts_min + (int)(u01(pp->seed, c, 12) * span) - 1;   // extra parts
      std::vector<uint32_t> got;
      int bx = std::min(G.nbx - 1, std::max(0, (int)((G.sx[c] - pp->x0) / G.bsx)));
      int by = std::min(G.nby - 1, std::max(0, (int)((G.sy[c] - pp->y0) / G.bsy)));
      for (int r = 2; r <= 3 && (int)got.size() < want; r++)
        for (int yy = by - r; yy <= by + r && (int)got.size() < want; yy++)
          for (int xx = bx - r; xx <= bx + r && (int)got.size() < want; xx++) {
            if (yy < 0 || yy >= G.nby || xx < 0 || xx >= G.nbx || std::max(std::abs(xx - bx), std::abs(yy - by)) != r) continue;
            uint32_t b = (uint32_t)yy * G.nbx + xx;
            for (uint32_t k = G.bstart[b]; k < G.bstart[b + 1] && (int)got.size() < want; k++) {
              uint32_t d = G.bidx[k];
              if (role[d] != 0 || cells[d].bad || is_nb(c, d)) continue;
              bool ok = true;
              for (uint32_t e : got) if (is_nb(e, d)) ok = false;
              if (ok) got.push_back(d);
            }
          }
      if (got.empty()) continue;
      std::sort(got.begin(), got.end());
      role[c] = 1; mp_of[c] = (int64_t)parts.size();
      for (uint32_t d : got) role[d] = 2;
      parts.push_back(got);
    }
  }
  for (uint64_t c = 0; c < n; c++) if (role[c] == 0 && pp->hole_frac > 0 && u01(pp->seed, c, 13) < pp->hole_frac) hole[c] = 1;
  out->n_mp = parts.size();

  std::vector<int> kappa(n);
  for (uint64_t c = 0; c < n; c++) kappa[c] = target_kappa(*pp, c);

  // subdivision points on the edge of cell c along line l: shared edges use the mean of both cells' targets
  auto edge_kappa = [&](uint64_t c, int64_t l) -> int { return l >= 0 ? (kappa[c] + kappa[l] + 1) / 2 : kappa[c]; };
  // ring vertex counts
  auto shell_nv = [&](uint64_t c) -> uint64_t {
    const auto& cl = cells[c];
    uint64_t nvv = 1;
    for (int64_t l : cl.lines) nvv += 1 + (uint64_t)edge_kappa(c, l);
    return nvv;
  };
  // geometry list: (kind, cell): kind 0 = geometry of cell c (shell [+hole] [+parts]), 1 = island in c's hole
  std::vector<std::pair<int, uint64_t>> geoms;
  geoms.reserve(n + n / 16);
  for (uint64_t c = 0; c < n; c++) {
    if (role[c] == 2) continue;
    geoms.push_back({0, c});
    if (hole[c]) geoms.push_back({1, c});
  }
  uint64_t ng = geoms.size();
  std::vector<uint64_t> gr(ng + 1, 0), gv(ng + 1, 0);
  for (uint64_t g = 0; g < ng; g++) {
    auto [kind, c] = geoms[g];
    uint64_t nr = 0, nvv = 0;
    if (kind == 1) { nr = 1; nvv = cells[c].lines.size() + 1; }
    else {
      nr = 1; nvv = shell_nv(c);
      if (hole[c]) { nr++; nvv += cells[c].lines.size() + 1; }
      if (role[c] == 1) for (uint32_t d : parts[mp_of[c]]) { nr++; nvv += shell_nv(d); }
    }
    gr[g + 1] = gr[g] + nr; gv[g + 1] = gv[g] + nvv;
  }
  out->n = ng; out->nr = gr[ng]; out->nv = gv[ng];
  out->n_holes = 0; for (uint64_t c = 0; c < n; c++) out->n_holes += hole[c];
  out->gro = (uint64_t*)malloc(sizeof(uint64_t) * (ng + 1));
  out->rvo = (uint64_t*)malloc(sizeof(uint64_t) * (out->nr + 1));
  out->xy = (double*)malloc(sizeof(double) * 2 * (out->nv ? out->nv : 1));
  if (!out->gro || !out->rvo || !out->xy) { gsjgen_free(out); return 2; }
  for (uint64_t g = 0; g <= ng; g++) out->gro[g] = gr[g];

#pragma omp parallel for schedule(dynamic, 512)
  for (int64_t g = 0; g < (int64_t)ng; g++) {
    auto [kind, c] = geoms[g];
    uint64_t r = gr[g], v = gv[g];
    double* xy = out->xy;
    auto emit_shell = [&](uint64_t cc) {
      const auto& cl = cells[cc];
      size_t m = cl.lines.size();
      out->rvo[r++] = v;
      for (size_t k = 0; k < m; k++) {
        xy[2 * v] = cl.vx[k]; xy[2 * v + 1] = cl.vy[k]; v++;
        int64_t l = cl.lines[k];
        int ke = edge_kappa(cc, l);
        if (!ke) continue;
        size_t k2 = (k + 1) % m;
        // canonical orientation: from the smaller vertex name to the larger
        bool fwd = cl.keys[k] < cl.keys[k2];
        double ax = fwd ? cl.vx[k] : cl.vx[k2], ay = fwd ? cl.vy[k] : cl.vy[k2];
        double bx = fwd ? cl.vx[k2] : cl.vx[k], by = fwd ? cl.vy[k2] : cl.vy[k];
        for (int q = 1; q <= ke; q++) {
          int mm = fwd ? q : ke + 1 - q;
          double t = (double)mm / (double)(ke + 1);
          xy[2 * v] = ax + (bx - ax) * t; xy[2 * v + 1] = ay + (by - ay) * t; v++;
        }
      }
      xy[2 * v] = cl.vx[0]; xy[2 * v + 1] = cl.vy[0]; v++;
    };
    auto hole_pts = [&](uint64_t cc, bool ccw) {
      const auto& cl = cells[cc];
      size_t m = cl.lines.size();
      out->rvo[r++] = v;
      for (size_t q = 0; q <= m; q++) {
        size_t k = ccw ? q % m : (m - q) % m;
        xy[2 * v] = G.sx[cc] + 0.35 * (cl.vx[k] - G.sx[cc]);
        xy[2 * v + 1] = G.sy[cc] + 0.35 * (cl.vy[k] - G.sy[cc]);
        v++;
      }
    };
    if (kind == 1) hole_pts(c, true);
    else {
      emit_shell(c);
      if (hole[c]) hole_pts(c, false);
      if (role[c] == 1) for (uint32_t d : parts[mp_of[c]]) emit_shell(d);
    }
  }
  out->rvo[out->nr] = out->nv;
  return 0;
}

extern "C" void gsjgen_free(gsjgen_set* s) {
  if (!s) return;
  free(s->gro); free(s->rvo); free(s->xy);
  s->gro = nullptr; s->rvo = nullptr; s->xy = nullptr; s->n = s->nr = s->nv = 0;
}

extern "C" void gsjgen_points(uint64_t n, double x0, double y0, double x1, double y1, uint64_t seed, double* xy) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    xy[2 * i] = x0 + u01(seed, (uint64_t)i, 21) * (x1 - x0);
    xy[2 * i + 1] = y0 + u01(seed, (uint64_t)i, 22) * (y1 - y0);
  }
}

extern "C" int gsjgen_write_gset(const char* path, const gsjgen_set* s) {
  FILE* f = fopen(path, "wb");
  if (!f) return 1;
  uint32_t ver = 1;
  bool ok = fwrite("GSET", 1, 4, f) == 4 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&s->n, 8, 1, f) == 1 &&
            fwrite(&s->nr, 8, 1, f) == 1 && fwrite(&s->nv, 8, 1, f) == 1 &&
            fwrite(s->gro, 8, s->n + 1, f) == s->n + 1 && fwrite(s->rvo, 8, s->nr + 1, f) == s->nr + 1 &&
            fwrite(s->xy, 8, 2 * s->nv, f) == 2 * s->nv;
  fclose(f);
  if (!ok) return 2;
  std::string ip = std::string(path) + ".ids";
  FILE* g = fopen(ip.c_str(), "w");
  if (!g) return 3;
  for (uint64_t i = 0; i < s->n; i++) fprintf(g, "%llu\n", (unsigned long long)i);
  fclose(g);
  return 0;
}

extern "C" int gsjgen_write_pset(const char* path, uint64_t n, const double* xy) {
  FILE* f = fopen(path, "wb");
  if (!f) return 1;
  uint32_t ver = 1;
  bool ok = fwrite("PSET", 1, 4, f) == 4 && fwrite(&ver, 4, 1, f) == 1 && fwrite(&n, 8, 1, f) == 1 && fwrite(xy, 8, 2 * n, f) == 2 * n;
  fclose(f);
  if (!ok) return 2;
  std::string ip = std::string(path) + ".ids";
  FILE* g = fopen(ip.c_str(), "w");
  if (!g) return 3;
  for (uint64_t i = 0; i < n; i++) fprintf(g, "%llu\n", (unsigned long long)i);
  fclose(g);
  return 0;
}

extern "C" int gsjgen_read_gset(const char* path, gsjgen_set* s) {
  memset(s, 0, sizeof(*s));
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  char magic[4]; uint32_t ver;
  if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "GSET", 4) || fread(&ver, 4, 1, f) != 1 || fread(&s->n, 8, 1, f) != 1 ||
      fread(&s->nr, 8, 1, f) != 1 || fread(&s->nv, 8, 1, f) != 1) { fclose(f); return 2; }
  s->gro = (uint64_t*)malloc(8 * (s->n + 1)); s->rvo = (uint64_t*)malloc(8 * (s->nr + 1)); s->xy = (double*)malloc(16 * (s->nv ? s->nv : 1));
  bool ok = s->gro && s->rvo && s->xy && fread(s->gro, 8, s->n + 1, f) == s->n + 1 && fread(s->rvo, 8, s->nr + 1, f) == s->nr + 1 &&
            fread(s->xy, 8, 2 * s->nv, f) == 2 * s->nv;
  fclose(f);
  if (!ok) { gsjgen_free(s); return 3; }
  return 0;
}
