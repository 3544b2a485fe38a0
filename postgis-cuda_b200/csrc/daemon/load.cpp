// Layer files for LOAD. The reference loads layers over libpq with parallel binary COPY (daemon/loader.h); this
// daemon reads the same rows from files: a PostgreSQL binary COPY file of (id text, geom) rows - the bytes
// `COPY (SELECT id::text, geom FROM t) TO 'f' (FORMAT binary)` writes, the stream the reference parses
// (CopyParser, loader.h:129-170) - or the flat .gset / .pset layouts of the reference's harness (engine/gset.h).
#include "load.h"

#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>

namespace gsjd {

double ring_area2(const double* xy, size_t n) {
  // Fan of triangles from the first vertex: differences to it are exact for the nearby vertices of one ring,
  // each cross product is kept as value + rounding error (an FMA recovers the error of a product), and all
  // terms are added with Neumaier's compensated summation, so the sign survives 1e-14 deg^2 slivers.
  if (n < 4) return 0;
  const double x0 = xy[0], y0 = xy[1];
  double sum = 0, comp = 0;
  auto acc = [&](double v) {
    const double t = sum + v;
    comp += std::fabs(sum) >= std::fabs(v) ? (sum - t) + v : (v - t) + sum;
    sum = t;
  };
  for (size_t i = 1; i + 2 < n; i++) {
    const double ax = xy[2 * i] - x0, ay = xy[2 * i + 1] - y0, bx = xy[2 * i + 2] - x0, by = xy[2 * i + 3] - y0;
    const double p = ax * by, q = ay * bx;
    acc(p);
    acc(-q);
    acc(std::fma(ax, by, -p));
    acc(-std::fma(ay, bx, -q));
  }
  return sum + comp;
}

namespace {

bool read_file(const std::string& path, std::string& data) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  data = ss.str();
  return true;
}

// ---- EWKB (PostGIS geometry_send): byte order, type with Z/M/SRID flags or ISO type codes, coordinates ----------
struct Reader {
  const uint8_t* p;
  const uint8_t* end;
  bool little = true;
  bool need(size_t k) const { return (size_t)(end - p) >= k; }
  uint32_t u32() {
    uint32_t v; std::memcpy(&v, p, 4); p += 4;
    return little ? v : __builtin_bswap32(v);
  }
  double f64() {
    uint64_t v; std::memcpy(&v, p, 8); p += 8;
    if (!little) v = __builtin_bswap64(v);
    double d; std::memcpy(&d, &v, 8);
    return d;
  }
};

enum Kind { kNothing = 0, kPolygonal = 1, kPoint = 2 };

// Geometry under assembly: rings appended to rvo / xy (one output geometry), or one point to pts.
struct Build {
  std::vector<uint64_t>& rvo;
  std::vector<double>& xy;
  std::vector<double>& pts;
  std::vector<double> ring;
  size_t rings = 0;
};

bool read_geometry(Reader& r, Build& b, int& kind) {   // loader.h:75-126
  if (!r.need(5)) return false;
  r.little = (*r.p++ == 1);
  const uint32_t type = r.u32();
  bool has_z = type & 0x80000000u, has_m = type & 0x40000000u;
  if (type & 0x20000000u) {   // SRID
    if (!r.need(4)) return false;
    r.u32();
  }
  uint32_t base = type & 0x0FFFFFFFu;
  if (base >= 1000) {   // ISO WKB: 1000 Z, 2000 M, 3000 ZM
    const uint32_t iso = base / 1000;
    base %= 1000;
    has_z = has_z || iso == 1 || iso == 3;
    has_m = has_m || iso == 2 || iso == 3;
  }
  const int dims = 2 + (has_z ? 1 : 0) + (has_m ? 1 : 0);
  if (base == 1) {   // POINT (NaN coordinates: POINT EMPTY)
    if (!r.need(8 * (size_t)dims)) return false;
    const double x = r.f64(), y = r.f64();
    for (int k = 2; k < dims; k++) r.f64();
    if (std::isnan(x) || std::isnan(y)) return true;
    b.pts.push_back(x); b.pts.push_back(y);
    kind = kPoint;
    return true;
  }
  if (base == 3) {   // POLYGON: first ring the shell (CCW), the others holes (CW); rings under 4 points dropped
    if (!r.need(4)) return false;
    const uint32_t nrings = r.u32();
    for (uint32_t k = 0; k < nrings; k++) {
      if (!r.need(4)) return false;
      const uint32_t np = r.u32();
      if (!r.need((size_t)np * 8 * dims)) return false;
      b.ring.resize(2 * (size_t)np);
      for (uint32_t i = 0; i < np; i++) {
        b.ring[2 * i] = r.f64(); b.ring[2 * i + 1] = r.f64();
        for (int d = 2; d < dims; d++) r.f64();
      }
      if (np < 4) continue;
      const bool ccw = ring_area2(b.ring.data(), np) > 0;
      if (ccw != (k == 0))
        for (uint32_t i = 0, j = np - 1; i < j; i++, j--) {
          std::swap(b.ring[2 * i], b.ring[2 * j]);
          std::swap(b.ring[2 * i + 1], b.ring[2 * j + 1]);
        }
      b.xy.insert(b.xy.end(), b.ring.begin(), b.ring.end());
      b.rvo.push_back(b.xy.size() / 2);
      b.rings++;
    }
    if (kind == kNothing) kind = kPolygonal;
    return true;
  }
  if (base == 6 || base == 7) {   // MULTIPOLYGON, GEOMETRYCOLLECTION: polygonal members only
    if (!r.need(4)) return false;
    const uint32_t ng = r.u32();
    for (uint32_t k = 0; k < ng; k++) {
      int sub = kNothing;
      if (!read_geometry(r, b, sub)) return false;
      if (sub == kPoint) return false;   // points mixed with polygons: unsupported
      if (sub == kPolygonal) kind = kPolygonal;
    }
    return true;
  }
  return false;   // lines and the rest
}

struct Parts {
  uint64_t polys = 0, points = 0;
  std::vector<double> pts;
};

// One row (id, geometry) of a COPY stream (loader.h:153-166).
void add_row(const uint8_t* id, int32_t id_len, const uint8_t* g, int32_t g_len, LoadedLayer& o, Parts& parts, Build& b) {
  o.rows++;
  if (id_len < 0 || g_len < 0) { o.skipped_null++; return; }
  Reader r{g, g + g_len};
  const size_t xy0 = o.xy.size(), rvo0 = o.rvo.size(), p0 = parts.pts.size();
  b.rings = 0;
  int kind = kNothing;
  const bool ok = read_geometry(r, b, kind);
  if (!ok || (parts.polys && kind == kPoint) || (parts.points && kind == kPolygonal)) {
    o.xy.resize(xy0); o.rvo.resize(rvo0); parts.pts.resize(p0);
    o.skipped_type++;
    return;
  }
  if (kind == kNothing || (kind == kPolygonal && b.rings == 0)) {
    o.xy.resize(xy0); o.rvo.resize(rvo0); parts.pts.resize(p0);
    o.skipped_empty++;
    return;
  }
  if (kind == kPolygonal) { o.gro.push_back(o.rvo.size() - 1); parts.polys++; }
  else parts.points++;
  o.ids.add(reinterpret_cast<const char*>(id), (size_t)id_len);
}

uint32_t be32(const uint8_t* p) { uint32_t v; std::memcpy(&v, p, 4); return __builtin_bswap32(v); }
uint16_t be16(const uint8_t* p) { uint16_t v; std::memcpy(&v, p, 2); return __builtin_bswap16(v); }

std::string load_copy(const std::string& data, LoadedLayer& o) {
  static const char sig[11] = {'P', 'G', 'C', 'O', 'P', 'Y', '\n', '\377', '\r', '\n', '\0'};
  const uint8_t* b = reinterpret_cast<const uint8_t*>(data.data());
  const size_t len = data.size();
  if (len < 19 || std::memcmp(b, sig, 11)) return "not a binary COPY file";
  const uint32_t ext = be32(b + 15);
  if (len < 19 + (size_t)ext) return "truncated COPY header";
  size_t pos = 19 + ext;
  Parts parts;
  Build bd{o.rvo, o.xy, parts.pts, {}, 0};
  for (;;) {
    if (len - pos < 2) return "COPY file ends without its trailer";
    const int16_t nf = (int16_t)be16(b + pos);
    pos += 2;
    if (nf == -1) break;
    if (nf != 2) return "COPY rows must have 2 columns (id text, geometry)";
    int32_t fl[2];
    size_t at[2];
    for (int k = 0; k < 2; k++) {
      if (len - pos < 4) return "truncated COPY row";
      fl[k] = (int32_t)be32(b + pos);
      pos += 4;
      at[k] = pos;
      if (fl[k] > 0) {
        if (len - pos < (size_t)fl[k]) return "truncated COPY row";
        pos += (size_t)fl[k];
      }
    }
    add_row(b + at[0], fl[0], b + at[1], fl[1], o, parts, bd);
  }
  if (parts.points) {
    o.is_points = true;
    o.xy.swap(parts.pts);
    o.gro.assign(1, 0); o.rvo.assign(1, 0);
  }
  return "";
}

std::string read_ids(const std::string& path, uint64_t n, IdTable& ids) {
  std::ifstream f(path + ".ids");
  if (!f) {
    for (uint64_t i = 0; i < n; i++) { const std::string s = std::to_string(i); ids.add(s.data(), s.size()); }
    return "";
  }
  std::string line;
  while (ids.size() < n && std::getline(f, line)) ids.add(line.data(), line.size());
  if (ids.size() != n) return "the .ids file has fewer lines than the layer has geometries";
  return "";
}

std::string load_gset(const std::string& path, const std::string& data, LoadedLayer& o) {
  if (data.size() < 32) return "truncated .gset header";
  uint64_t n, nr, nv;
  std::memcpy(&n, data.data() + 8, 8); std::memcpy(&nr, data.data() + 16, 8); std::memcpy(&nv, data.data() + 24, 8);
  if (n >= (1ull << 31) || nr >= (1ull << 40) || nv >= (1ull << 40)) return ".gset sizes out of range";
  const size_t need = 32 + 8 * (n + 1) + 8 * (nr + 1) + 16 * nv;
  if (data.size() < need) return "truncated .gset file";
  o.gro.resize(n + 1); o.rvo.resize(nr + 1); o.xy.resize(2 * nv);
  const char* p = data.data() + 32;
  std::memcpy(o.gro.data(), p, 8 * (n + 1)); p += 8 * (n + 1);
  std::memcpy(o.rvo.data(), p, 8 * (nr + 1)); p += 8 * (nr + 1);
  std::memcpy(o.xy.data(), p, 16 * nv);
  if (o.gro[0] != 0 || o.gro[n] != nr || o.rvo[0] != 0 || o.rvo[nr] != nv) return ".gset offsets are inconsistent";
  for (uint64_t g = 0; g < n; g++) if (o.gro[g + 1] < o.gro[g]) return ".gset geometry offsets decrease";
  for (uint64_t r = 0; r < nr; r++) if (o.rvo[r + 1] < o.rvo[r]) return ".gset ring offsets decrease";
  o.rows = n;
  return read_ids(path, n, o.ids);
}

std::string load_pset(const std::string& path, const std::string& data, LoadedLayer& o) {
  if (data.size() < 16) return "truncated .pset header";
  uint64_t n;
  std::memcpy(&n, data.data() + 8, 8);
  if (n >= (1ull << 32) || data.size() < 16 + 16 * n) return "truncated .pset file";
  o.is_points = true;
  o.xy.resize(2 * n);
  std::memcpy(o.xy.data(), data.data() + 16, 16 * n);
  o.rows = n;
  return read_ids(path, n, o.ids);
}

}  // namespace

std::string load_layer_file(const std::string& path, LoadedLayer& out) {
  std::string data;
  if (!read_file(path, data)) return "cannot read " + path;
  if (data.size() >= 4 && !std::memcmp(data.data(), "GSET", 4)) return load_gset(path, data, out);
  if (data.size() >= 4 && !std::memcmp(data.data(), "PSET", 4)) return load_pset(path, data, out);
  if (data.size() >= 6 && !std::memcmp(data.data(), "PGCOPY", 6)) return load_copy(data, out);
  return "unknown layer file format (expected a binary COPY file, .gset or .pset): " + path;
}

}  // namespace gsjd
