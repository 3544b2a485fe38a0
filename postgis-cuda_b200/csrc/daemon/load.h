// Layer files for LOAD: .gset / .pset (+ .ids) and PostgreSQL binary COPY files of (id, EWKB geometry) rows.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "rows.h"

namespace gsjd {

struct LoadedLayer {
  bool is_points = false;
  uint64_t rows = 0, skipped_null = 0, skipped_type = 0, skipped_empty = 0;
  std::vector<uint64_t> gro{0}, rvo{0};   // polygons: geometry -> ring, ring -> vertex offsets
  std::vector<double> xy;                 // polygon vertices, or points
  IdTable ids;                            // one per kept geometry / point
  uint64_t n() const { return is_points ? xy.size() / 2 : gro.size() - 1; }
};

// Returns "" on success, else the reason.
std::string load_layer_file(const std::string& path, LoadedLayer& out);

// Twice the signed area of a closed ring (n points, first == last), robust enough to orient sliver rings.
double ring_area2(const double* xy, size_t n);

}  // namespace gsjd
