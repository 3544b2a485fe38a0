/* gsjd - the serving daemon over the gsj engine: the drop-in for landstats-us/postgis-cuda's gpujoind
 * (daemon/gpujoind.cu), speaking its wire protocol (gsp_protocol.h). Host code only; the GPU work goes through
 * gsj.h. This header exposes the daemon's host-side rules as a C ABI so they can be used and tested without a
 * GPU: the row rules that turn engine pairs into result rows, cluster numbering, and the layer file loader.
 */
#ifndef GSJD_H
#define GSJD_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Row expansion of engine pairs (distinct-geometry ids) into result rows (input row ids), the rules of op_join /
 * op_relate / op_dwithin (gpujoind.cu:271-283, 356-367, 471-481):
 *  - members: a deduplicated layer's distinct geometry g stands for rows midx[moff[g] .. moff[g+1]) (moff NULL:
 *    not deduplicated, g is its own row); rows are members(a) x members(b);
 *  - same (self-join over one layer, pairs reported once with b >= a):
 *      distinct = 0 ("all"): row (ra, rb) and, off the diagonal, the mirrored row (rb, ra);
 *      distinct = 1: rows (lo, hi) with lo < hi only (no row of an input row with itself);
 *  - tr[k] = 1 marks a row that reads the pair in the (b, a) order: a DE-9IM code must be transposed for it.
 * out_rows[2k] = (a row, b row), out_src[k] = index of the pair the row came from. Outputs are allocated by the
 * library (free with gsjd_free). Returns 0, or 1 on bad arguments. */
int gsjd_expand_rows(uint64_t n, const uint32_t* pairs, int same, int distinct, const uint64_t* moff_a, const uint32_t* midx_a,
                     const uint64_t* moff_b, const uint32_t* midx_b, uint64_t* out_n, uint32_t** out_rows, uint64_t** out_src,
                     uint8_t** out_tr);
/* Number of rows the pairs expand to (stats-only requests, gpujoind.cu:257-267, 454-463). */
uint64_t gsjd_count_rows(uint64_t n, const uint32_t* pairs, int same, int distinct, const uint64_t* moff_a, const uint64_t* moff_b);
/* Cluster labels per input row from the engine's roots per distinct geometry: dense numbers in order of first
 * row (op_cluster, gpujoind.cu:302-313). label[rows]; returns the number of clusters. */
uint32_t gsjd_cluster_labels(uint32_t n_distinct, const uint32_t* root, uint64_t rows, const uint64_t* moff, const uint32_t* midx,
                             uint32_t* label);

/* Layer files for LOAD (the file counterpart of the libpq COPY loader, daemon/loader.h): a `.gset` / `.pset`
 * (+ `.ids`, one id per line; indices when absent), or a PostgreSQL binary COPY file of (id text, geom) rows
 * as written by COPY (SELECT id::text, geom FROM t) TO 'file' (FORMAT binary), geometry as EWKB (geometry_send).
 * EWKB polygons, multipolygons and the polygons of collections become one geometry each with shells CCW and holes
 * CW (compensated orientation test); rings of fewer than 4 points are dropped; null ids/geometries, other types and
 * empty geometries are counted and skipped (loader.h:59-170). The first kind met (points or polygons) fixes the
 * layer's kind; rows of the other kind are skipped as wrong type. */
typedef struct gsjd_file gsjd_file;
int gsjd_file_open(const char* path, gsjd_file** out, char* err, size_t errlen);
typedef struct gsjd_file_info {
  int is_points;
  uint64_t rows, skipped_null, skipped_type, skipped_empty;
  uint64_t n, nr, nv;   /* kept geometries, rings, vertices (points: n = nv = points, nr = 0) */
} gsjd_file_info;
void gsjd_file_get_info(const gsjd_file* f, gsjd_file_info* info);
/* gro[n+1], rvo[nr+1], xy[2nv] for polygons; xy[2n] for points (gro, rvo NULL). Valid until gsjd_file_close. */
void gsjd_file_arrays(const gsjd_file* f, const uint64_t** gro, const uint64_t** rvo, const double** xy);
/* id of kept geometry i (not NUL-terminated). */
const char* gsjd_file_id(const gsjd_file* f, uint64_t i, size_t* len);
void gsjd_file_close(gsjd_file* f);

void gsjd_free(void* p);

/* The daemon: gsjd [--socket PATH] [--tcp HOST:PORT] [--token-file FILE] [--data-dir DIR] [--device N]
 *                  [--workers N] [--threads N] [--conninfo STR]. Runs until killed. */
int gsjd_main(int argc, char** argv);

#ifdef __cplusplus
}
#endif
#endif
