// C ABI of the daemon's host rules (gsjd.h): row expansion, row counts, cluster numbering, layer files.
#include <cstdlib>
#include <cstring>
#include <new>

#include "../../../include/gsjd.h"
#include "load.h"
#include "rows.h"

using namespace gsjd;

extern "C" {

int gsjd_expand_rows(uint64_t n, const uint32_t* pairs, int same, int distinct, const uint64_t* moff_a, const uint32_t* midx_a,
                     const uint64_t* moff_b, const uint32_t* midx_b, uint64_t* out_n, uint32_t** out_rows, uint64_t** out_src,
                     uint8_t** out_tr) {
  if ((n && !pairs) || !out_n || !out_rows || !out_src || !out_tr) return 1;
  if ((moff_a && !midx_a) || (moff_b && !midx_b)) return 1;
  const Members A{moff_a, midx_a}, B{moff_b, midx_b};
  uint64_t total = 0;
  for (uint64_t i = 0; i < n; i++) total += pair_row_count(pairs[2 * i], pairs[2 * i + 1], A, B, same != 0, distinct != 0);
  uint32_t* rows = static_cast<uint32_t*>(std::malloc(8 * (total ? total : 1)));
  uint64_t* src = static_cast<uint64_t*>(std::malloc(8 * (total ? total : 1)));
  uint8_t* tr = static_cast<uint8_t*>(std::malloc(total ? total : 1));
  if (!rows || !src || !tr) { std::free(rows); std::free(src); std::free(tr); return 1; }
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; i++)
    pair_rows(pairs[2 * i], pairs[2 * i + 1], A, B, same != 0, distinct != 0, [&](uint32_t ra, uint32_t rb, bool t) {
      rows[2 * k] = ra; rows[2 * k + 1] = rb; src[k] = i; tr[k] = t ? 1 : 0; k++;
    });
  *out_n = k; *out_rows = rows; *out_src = src; *out_tr = tr;
  return 0;
}

uint64_t gsjd_count_rows(uint64_t n, const uint32_t* pairs, int same, int distinct, const uint64_t* moff_a, const uint64_t* moff_b) {
  const Members A{moff_a, nullptr}, B{moff_b, nullptr};
  uint64_t t = 0;
  for (uint64_t i = 0; i < n; i++) t += pair_row_count(pairs[2 * i], pairs[2 * i + 1], A, B, same != 0, distinct != 0);
  return t;
}

uint32_t gsjd_cluster_labels(uint32_t n_distinct, const uint32_t* root, uint64_t rows, const uint64_t* moff, const uint32_t* midx,
                             uint32_t* label) {
  // root per distinct geometry -> root per input row -> dense numbers in order of first row
  uint32_t* row_root = static_cast<uint32_t*>(std::malloc(4 * (rows ? rows : 1)));
  uint32_t* dense = static_cast<uint32_t*>(std::malloc(4 * (n_distinct ? n_distinct : 1)));
  if (!row_root || !dense) { std::free(row_root); std::free(dense); return 0; }
  const Members M{moff, midx};
  for (uint32_t g = 0; g < n_distinct; g++) M.each(g, [&](uint32_t r) { if (r < rows) row_root[r] = root[g]; });
  for (uint32_t g = 0; g < n_distinct; g++) dense[g] = UINT32_MAX;
  uint32_t k = 0;
  for (uint64_t r = 0; r < rows; r++) {
    const uint32_t rt = row_root[r];
    if (dense[rt] == UINT32_MAX) dense[rt] = k++;
    label[r] = dense[rt];
  }
  std::free(row_root); std::free(dense);
  return k;
}

struct gsjd_file {
  LoadedLayer L;
};

int gsjd_file_open(const char* path, gsjd_file** out, char* err, size_t errlen) {
  if (!path || !out) return 1;
  gsjd_file* f = new (std::nothrow) gsjd_file;
  if (!f) return 1;
  const std::string e = load_layer_file(path, f->L);
  if (!e.empty()) {
    if (err && errlen) { std::strncpy(err, e.c_str(), errlen - 1); err[errlen - 1] = 0; }
    delete f;
    return 1;
  }
  *out = f;
  return 0;
}

void gsjd_file_get_info(const gsjd_file* f, gsjd_file_info* info) {
  const LoadedLayer& L = f->L;
  info->is_points = L.is_points;
  info->rows = L.rows; info->skipped_null = L.skipped_null; info->skipped_type = L.skipped_type; info->skipped_empty = L.skipped_empty;
  info->n = L.n();
  info->nr = L.is_points ? 0 : L.rvo.size() - 1;
  info->nv = L.xy.size() / 2;
}

void gsjd_file_arrays(const gsjd_file* f, const uint64_t** gro, const uint64_t** rvo, const double** xy) {
  const LoadedLayer& L = f->L;
  if (gro) *gro = L.is_points ? nullptr : L.gro.data();
  if (rvo) *rvo = L.is_points ? nullptr : L.rvo.data();
  if (xy) *xy = L.xy.data();
}

const char* gsjd_file_id(const gsjd_file* f, uint64_t i, size_t* len) {
  if (i >= f->L.ids.size()) { if (len) *len = 0; return nullptr; }
  if (len) *len = f->L.ids.len(i);
  return f->L.ids.data(i);
}

void gsjd_file_close(gsjd_file* f) { delete f; }

void gsjd_free(void* p) { std::free(p); }

}  // extern "C"
