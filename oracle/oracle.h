/* CPU FP64 oracle for the spatial-join hot path - TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++ restatement of the reference engine's per-pair decisions (landstats-us/postgis-cuda,
 * engine/engine.cuh and engine/buffer.cuh), used by tests/ to check the CUDA engine, by the bench's
 * cpu_baseline leg and by its `--impl reference` arm. Nothing in the product links or calls it.
 *
 * Arithmetic contract shared with the CUDA engine: no implicit FMA contraction (-ffp-contract=off here,
 * --fmad=false there), explicit fma() exactly where the reference's `orient` uses it, and the area / relate
 * sums accumulated in the order of the reference's warp (lane l owns edges l, l+32, ...; A edges then B
 * edges; then the shfl_down tree 16, 8, 4, 2, 1). Under that contract pair sets, flags, DE-9IM codes and
 * areas are bit-identical between the oracle and the engine.
 */
#ifndef GSJ_ORACLE_H
#define GSJ_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_set orc_set;

/* Polygon set in the reference's host layout (engine/gset.h:5-11): gro[n+1], rvo[nr+1] (u64), xy[2nv] world
 * coordinates. parent[n] (piece -> geometry, sorted) and syn[nv] (edge v->v+1 made by subdivision) are optional
 * (NULL). Prepared as upload_set does (engine.cuh:42-89). */
orc_set* orc_set_create(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy,
                        const uint32_t* parent, const uint8_t* syn);
void orc_set_free(orc_set* s);
/* conservative float bbox (minx, miny, maxx, maxy) per geometry, as upload_set builds it */
void orc_set_bbox(const orc_set* s, float* bb4);

typedef struct orc_params {
  double tol_rel, eps_par, tol_abs;   /* RefineParams defaults: 1e-12, 1e-7, 1e-11 (engine.cuh:517) */
  int want_area, want_relate, snap_half_ulp;
} orc_params;

/* Candidate pairs (query a in P, leaf b in R) whose float bboxes overlap, as k_traverse reports them
 * (engine.cuh:233-259); upper: keep b >= a. Sorted by (a, b). Caller frees *out with orc_free. */
int64_t orc_candidates(const orc_set* P, const orc_set* R, int upper, uint32_t** out_pairs);
/* Same with explicit query boxes (points or expanded boxes). */
int64_t orc_candidates_bb(const float* qbb4, uint64_t nq, const orc_set* R, int upper, uint32_t** out_pairs);

/* Per candidate pair decision of k_refine (engine.cuh:530-636): flag 0/1/2, area, relate evidence
 * (ev[4*i] = inside/on length of A's real boundary, then of B's) and bits. Arrays may be NULL. */
void orc_refine_pairs(const orc_set* P, const orc_set* R, const uint32_t* pairs, int64_t np, const orc_params* rp,
                      uint8_t* flag, double* area, double* ev, uint32_t* evb, int nthreads);

/* Full join as join_stream produces it (engine.cuh:895-1061): parent pairs with area and DE-9IM code,
 * sorted by (a, b). Returns the number of rows; arrays freed with orc_free. */
int64_t orc_join(const orc_set* P, const orc_set* R, const orc_params* rp, int upper, int nthreads,
                 uint32_t** out_pairs, double** out_area, uint32_t** out_code, int64_t* n_candidates);

/* DE-9IM helpers (engine.cuh:848-888) */
uint32_t orc_de9im_code(const double* ev4, uint32_t bits, double la, double lb);
uint32_t orc_de9im_transpose(uint32_t code);
int orc_de9im_match(uint32_t code, const char* pat);
double orc_blen(const orc_set* s, uint32_t parent);

/* Point in polygon (k_pip_pairs, engine.cuh:1079-1106): where 1 interior / 2 boundary, per (point, parent),
 * boundary wins over interior (MaxU8 fold). */
int64_t orc_pip(const double* pts, uint64_t npts, const orc_set* R, int nthreads, uint32_t** out_pairs, uint8_t** out_where,
                int64_t* n_candidates);

/* ST_ClusterIntersecting (engine.cuh:1216-1234): root[g] = smallest parent index in g's component. */
void orc_cluster(const orc_set* P, uint32_t nparent, const orc_params* rp, int nthreads, uint32_t* root);

/* ST_DWithin(geography) polygon x polygon (buffer.cuh:185-273, 892-991): unique parent pairs. same: P and R are
 * one set (pieces of one parent shortcut, upper). */
int64_t orc_dwithin(const orc_set* P, const orc_set* R, double d, int same, int nthreads, uint32_t** out_pairs, int64_t* n_candidates);
/* points x polygons dwithin / in eroded polygon (buffer.cuh:1019-1132, 1137-1231): (point, parent) pairs. */
int64_t orc_pt_dwithin(const double* pts, uint64_t npts, const orc_set* R, double d, int nthreads, uint32_t** out_pairs);
int64_t orc_pt_erode(const double* pts, uint64_t npts, const orc_set* R, double r, int nthreads, uint32_t** out_pairs);
/* eroded intersects (buffer.cuh:499-889): parent pairs. need_self may be NULL. */
int64_t orc_erode(const orc_set* P, const orc_set* R, double ra, double rb, int same, const uint8_t* need_self, int nthreads,
                  uint32_t** out_pairs);

/* Layer preparation restated on the CPU (oracle_prep.cpp). Subdivision (engine/subdivide.h:14-129): pieces of at most
 * ~maxv vertices, parent[piece] = geometry, syn[v] = 1 for an edge on a cut line; returns the piece count.
 * Deduplication (engine/dedup.h:22-124): distinct geometries in order of first occurrence (morton: Z-order of their
 * bbox centres), members midx[moff[d] .. moff[d+1]); returns the distinct count. Arrays freed with orc_free. */
int64_t orc_subdivide(uint64_t n, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv, uint64_t** out_gro, uint64_t** out_rvo,
                      double** out_xy, uint32_t** out_parent, uint8_t** out_syn, uint64_t* out_nr, uint64_t* out_nv);
int64_t orc_dedup(uint64_t n, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton, uint64_t** out_gro, uint64_t** out_rvo,
                  double** out_xy, uint64_t** out_moff, uint32_t** out_midx, uint64_t* out_nr, uint64_t* out_nv);

void orc_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
