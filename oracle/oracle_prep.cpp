// CPU restatement of layer preparation - TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Subdivision (ST_Subdivide analogue, landstats-us/postgis-cuda engine/subdivide.h:14-129) and exact
// deduplication (engine/dedup.h:22-124), restated as plain sequential C++ with the engine's GPU design
// (csrc/prep_gpu.cu): subdivision runs breadth-first over a work list of pieces keyed by their cut path and sorts
// the leaves by key, deduplication walks the geometries once in input order with a hash table of the distinct
// ones seen so far. The FP64 steps that decide the output bits are the reference's: the cut point
// p + (m - p_axis) * (q - p) / (q_axis - p_axis), the repeated-point rule, the closing point, the shoelace area
// that drops slivers, the bbox midpoint of the longer side, the depth limit of 24, and for the Z-ordered variant
// the bbox-centre quantisation to 32 bits per axis. Compiled with -ffp-contract=off like the rest of the oracle.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string_view>
#include <unordered_map>
#include <vector>

#include "oracle.h"

namespace {

struct Ring {
  std::vector<double> xy;      // closed: last point == first
  std::vector<uint8_t> cut;    // cut[i]: edge i -> i+1 lies on a cut line
};

// One clipped ring, built point by point. The shoelace terms are summed as the points arrive (the same terms in
// the same order as summing over the finished ring), so a ring of zero area is recognised without a second pass.
class Clipper {
 public:
  void begin() { r_.xy.clear(); r_.cut.clear(); area_ = 0.0; }
  void add(double x, double y, uint8_t f) {
    const size_t k = r_.cut.size();
    if (k && r_.xy[2 * k - 2] == x && r_.xy[2 * k - 1] == y) { r_.cut[k - 1] = f; return; }   // same point twice: one point
    if (k) area_ += r_.xy[2 * k - 2] * y - x * r_.xy[2 * k - 1];
    r_.xy.push_back(x); r_.xy.push_back(y); r_.cut.push_back(f);
  }
  // false: the ring vanished (fewer than 4 points once closed, or zero area)
  bool finish(Ring& out) {
    size_t k = r_.cut.size();
    if (k < 3) return false;
    const double fx = r_.xy[0], fy = r_.xy[1], lx = r_.xy[2 * k - 2], ly = r_.xy[2 * k - 1];
    if (fx != lx || fy != ly) { area_ += lx * fy - fx * ly; r_.xy.push_back(fx); r_.xy.push_back(fy); r_.cut.push_back(0); k++; }
    else r_.cut[k - 1] = 0;
    if (k < 4 || area_ == 0.0) return false;
    out = r_;
    return true;
  }
 private:
  Ring r_;
  double area_ = 0.0;
};

// keep the part of ring `in` on one side of the line coord[axis] = m (low: coord <= m, else coord >= m)
bool clip(const Ring& in, int axis, double m, bool low, Clipper& c, Ring& out) {
  c.begin();
  const size_t n = in.cut.size();
  for (size_t i = 0; i + 1 < n; i++) {
    const double px = in.xy[2 * i], py = in.xy[2 * i + 1], qx = in.xy[2 * i + 2], qy = in.xy[2 * i + 3];
    const double pa = axis ? py : px, qa = axis ? qy : qx;
    const bool pin = low ? pa <= m : pa >= m, qin = low ? qa <= m : qa >= m;
    if (pin) c.add(px, py, in.cut[i]);
    if (pin == qin) continue;
    double ix, iy;
    if (axis == 0) { ix = m; iy = py + (m - px) * (qy - py) / (qx - px); }
    else { iy = m; ix = px + (m - py) * (qx - px) / (qy - py); }
    c.add(ix, iy, pin ? 1 : in.cut[i]);   // leaving: the edge that follows runs along the cut line
  }
  return c.finish(out);
}

struct Piece {
  uint32_t path = 0;   // cut decisions, the first in the top bit of 24 (0 = low side)
  int depth = 0;
  std::vector<Ring> rings;
};
constexpr int MAX_DEPTH = 24;

// the leaves of one geometry in cut-path order (the reference's depth-first order)
std::vector<Piece> split_geometry(std::vector<Ring> rings, int maxv) {
  std::vector<Piece> work(1), next, leaves;
  work[0].rings = std::move(rings);
  Clipper c;
  while (!work.empty()) {
    next.clear();
    for (Piece& p : work) {
      uint64_t nv = 0;
      double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
      for (const Ring& r : p.rings) {
        nv += r.cut.size();
        for (size_t i = 0; i < r.cut.size(); i++) {
          x0 = std::fmin(x0, r.xy[2 * i]); x1 = std::fmax(x1, r.xy[2 * i]);
          y0 = std::fmin(y0, r.xy[2 * i + 1]); y1 = std::fmax(y1, r.xy[2 * i + 1]);
        }
      }
      if (nv <= (uint64_t)maxv || p.depth >= MAX_DEPTH || (x1 - x0 <= 0 && y1 - y0 <= 0)) { leaves.push_back(std::move(p)); continue; }
      const int axis = (x1 - x0) >= (y1 - y0) ? 0 : 1;
      const double m = axis == 0 ? 0.5 * (x0 + x1) : 0.5 * (y0 + y1);
      for (int side = 0; side < 2; side++) {
        Piece q;
        q.depth = p.depth + 1;
        q.path = p.path | ((uint32_t)side << (MAX_DEPTH - 1 - p.depth));
        Ring out;
        for (const Ring& r : p.rings)
          if (clip(r, axis, m, side == 0, c, out)) q.rings.push_back(out);
        if (!q.rings.empty()) next.push_back(std::move(q));
      }
    }
    work.swap(next);
  }
  std::stable_sort(leaves.begin(), leaves.end(), [](const Piece& a, const Piece& b) { return a.path < b.path; });
  return leaves;
}

template <class T> T* to_malloc(const std::vector<T>& v) {
  T* p = static_cast<T*>(malloc(sizeof(T) * (v.empty() ? 1 : v.size())));
  if (p && !v.empty()) memcpy(p, v.data(), sizeof(T) * v.size());
  return p;
}

uint64_t interleave(uint32_t v) {   // bit i of v -> bit 2i
  uint64_t r = 0;
  for (int i = 0; i < 32; i++) r |= (uint64_t)((v >> i) & 1u) << (2 * i);
  return r;
}

}  // namespace

extern "C" {

int64_t orc_subdivide(uint64_t n, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv, uint64_t** out_gro, uint64_t** out_rvo,
                      double** out_xy, uint32_t** out_parent, uint8_t** out_syn, uint64_t* out_nr, uint64_t* out_nv) {
  std::vector<std::vector<Piece>> per(n);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t g = 0; g < (int64_t)n; g++) {
    std::vector<Ring> rings;
    uint64_t nv = 0;
    for (uint64_t r = gro[g]; r < gro[g + 1]; r++) {
      Ring ring;
      ring.xy.assign(xy + 2 * rvo[r], xy + 2 * rvo[r + 1]);
      ring.cut.assign(rvo[r + 1] - rvo[r], 0);
      nv += ring.cut.size();
      rings.push_back(std::move(ring));
    }
    if (nv <= (uint64_t)maxv) { per[g].resize(1); per[g][0].rings = std::move(rings); }
    else per[g] = split_geometry(std::move(rings), maxv);
  }
  std::vector<uint64_t> og{0}, orv{0};
  std::vector<double> oxy;
  std::vector<uint8_t> osyn;
  std::vector<uint32_t> opar;
  for (uint64_t g = 0; g < n; g++)
    for (const Piece& p : per[g]) {
      for (const Ring& r : p.rings) {
        oxy.insert(oxy.end(), r.xy.begin(), r.xy.end());
        osyn.insert(osyn.end(), r.cut.begin(), r.cut.end());
        orv.push_back(oxy.size() / 2);
      }
      og.push_back(orv.size() - 1);
      opar.push_back((uint32_t)g);
    }
  *out_gro = to_malloc(og); *out_rvo = to_malloc(orv); *out_xy = to_malloc(oxy); *out_parent = to_malloc(opar); *out_syn = to_malloc(osyn);
  *out_nr = orv.size() - 1;
  *out_nv = oxy.size() / 2;
  return (int64_t)opar.size();
}

int64_t orc_dedup(uint64_t n, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton, uint64_t** out_gro, uint64_t** out_rvo,
                  double** out_xy, uint64_t** out_moff, uint32_t** out_midx, uint64_t* out_nr, uint64_t* out_nv) {
  // a geometry's bytes: ring sizes, then its vertex words
  auto key_of = [&](uint64_t g, std::vector<uint64_t>& buf) {
    buf.clear();
    for (uint64_t r = gro[g]; r < gro[g + 1]; r++) buf.push_back(rvo[r + 1] - rvo[r]);
    const uint64_t v0 = rvo[gro[g]], v1 = rvo[gro[g + 1]];
    const size_t at = buf.size();
    buf.resize(at + 2 * (v1 - v0));
    if (v1 > v0) memcpy(buf.data() + at, xy + 2 * v0, 16 * (v1 - v0));
  };
  std::vector<uint64_t> h(n);
#pragma omp parallel
  {
    std::vector<uint64_t> buf;
#pragma omp for schedule(static)
    for (int64_t g = 0; g < (int64_t)n; g++) {
      key_of((uint64_t)g, buf);
      h[g] = std::hash<std::string_view>()(std::string_view(reinterpret_cast<const char*>(buf.data()), buf.size() * 8)) ^ (gro[g + 1] - gro[g]);
    }
  }
  // one pass in input order: a geometry joins the first identical one seen before it, or starts a new one
  std::unordered_map<uint64_t, std::vector<uint32_t>> seen;
  std::vector<uint32_t> first, cls(n);
  std::vector<uint64_t> ka, kb;
  for (uint64_t g = 0; g < n; g++) {
    std::vector<uint32_t>& bucket = seen[h[g]];
    uint32_t found = UINT32_MAX;
    if (!bucket.empty()) {
      key_of(g, kb);
      for (uint32_t d : bucket) {
        key_of(first[d], ka);
        if (ka == kb && gro[first[d] + 1] - gro[first[d]] == gro[g + 1] - gro[g]) { found = d; break; }
      }
    }
    if (found == UINT32_MAX) { found = (uint32_t)first.size(); first.push_back((uint32_t)g); bucket.push_back(found); }
    cls[g] = found;
  }
  const uint64_t un = first.size();
  std::vector<uint32_t> pos(un);   // output position of each distinct geometry
  for (uint64_t d = 0; d < un; d++) pos[d] = (uint32_t)d;
  if (morton && un > 1) {   // Z-order of the bbox centres, quantised to 32 bits per axis over their range
    std::vector<double> cx(un), cy(un);
    for (uint64_t d = 0; d < un; d++) {
      const uint32_t g = first[d];
      double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
      for (uint64_t v = rvo[gro[g]]; v < rvo[gro[g + 1]]; v++) {
        x0 = std::min(x0, xy[2 * v]); x1 = std::max(x1, xy[2 * v]); y0 = std::min(y0, xy[2 * v + 1]); y1 = std::max(y1, xy[2 * v + 1]);
      }
      cx[d] = 0.5 * (x0 + x1); cy[d] = 0.5 * (y0 + y1);
    }
    const auto [ax0, ax1] = std::minmax_element(cx.begin(), cx.end());
    const auto [ay0, ay1] = std::minmax_element(cy.begin(), cy.end());
    const double mx0 = *ax0, mx1 = *ax1, my0 = *ay0, my1 = *ay1;
    const double sx = mx1 > mx0 ? 4294967295.0 / (mx1 - mx0) : 0, sy = my1 > my0 ? 4294967295.0 / (my1 - my0) : 0;
    std::vector<uint64_t> z(un);
    for (uint64_t d = 0; d < un; d++)
      z[d] = (interleave((uint32_t)(uint64_t)((cx[d] - mx0) * sx)) << 1) | interleave((uint32_t)(uint64_t)((cy[d] - my0) * sy));
    std::vector<uint32_t> ord(un);
    for (uint64_t d = 0; d < un; d++) ord[d] = (uint32_t)d;
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return z[a] < z[b]; });
    for (uint64_t i = 0; i < un; i++) pos[ord[i]] = (uint32_t)i;
  }
  std::vector<uint64_t> moff(un + 1, 0);
  for (uint64_t g = 0; g < n; g++) moff[pos[cls[g]] + 1]++;
  for (uint64_t i = 0; i < un; i++) moff[i + 1] += moff[i];
  std::vector<uint32_t> midx(n);
  std::vector<uint64_t> fill(moff.begin(), moff.end() - 1);
  for (uint64_t g = 0; g < n; g++) midx[fill[pos[cls[g]]]++] = (uint32_t)g;
  std::vector<uint32_t> at(un);
  for (uint64_t d = 0; d < un; d++) at[pos[d]] = first[d];
  std::vector<uint64_t> og{0}, orv{0};
  std::vector<double> oxy;
  for (uint64_t i = 0; i < un; i++) {
    const uint32_t g = at[i];
    for (uint64_t r = gro[g]; r < gro[g + 1]; r++) {
      oxy.insert(oxy.end(), xy + 2 * rvo[r], xy + 2 * rvo[r + 1]);
      orv.push_back(oxy.size() / 2);
    }
    og.push_back(orv.size() - 1);
  }
  *out_gro = to_malloc(og); *out_rvo = to_malloc(orv); *out_xy = to_malloc(oxy); *out_moff = to_malloc(moff); *out_midx = to_malloc(midx);
  *out_nr = orv.size() - 1;
  *out_nv = oxy.size() / 2;
  return (int64_t)un;
}

}  // extern "C"
