/* Synthetic parcel layers for tests and benchmarks (host only, no CUDA).
 *
 * Voronoi cells of seeded point sets, written in the flat polygon-set layout of the reference's
 * `.gset` files (engine/gset.h:5-30, scripts/dump_gset.py:6-12): u64 geometry->ring offsets, u64
 * ring->vertex offsets, closed rings, shells CCW and holes CW (the daemon/loader.h:100-102 invariant).
 *
 * Every Voronoi vertex is computed once from a canonical label (the sorted seed triple, or seed pair and
 * box side), and every edge subdivision point from the canonical orientation of its edge, so neighbouring
 * cells share bit-identical vertices along their common boundary - the property real parcel layers have and
 * the exact touch tests rely on. Output is a pure function of the parameters (seeded splitmix64 streams keyed
 * by seed index), independent of the thread count.
 */
#ifndef GSJGEN_H
#define GSJGEN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct gsjgen_params {
  uint64_t n;              /* number of seeds (cells) */
  double x0, y0, x1, y1;   /* box (lon/lat degrees) */
  uint64_t seed;           /* RNG seed */
  int jitter_grid;         /* 0: uniform random seeds; 1: jittered grid (+-jitter of a grid cell) */
  double jitter;           /* jitter amplitude in grid cells (e.g. 0.4) */
  int vmin, vmax;          /* target ring vertex count range (closed ring, incl. the closing vertex) */
  int log_uniform;         /* 0: uniform in [vmin, vmax]; 1: log-uniform */
  double mp_frac;          /* fraction of cells that become MultiPolygons */
  int mp_parts_min, mp_parts_max;
  double hole_frac;        /* fraction of cells with one interior hole (filled by an island geometry) */
} gsjgen_params;

typedef struct gsjgen_set {
  uint64_t n, nr, nv;
  uint64_t* gro;   /* [n+1] */
  uint64_t* rvo;   /* [nr+1] */
  double* xy;      /* [2*nv] */
  uint64_t n_mp, n_holes, n_inconsistent;   /* stats: multipolygons, holes, shared-edge mismatches found */
} gsjgen_set;

/* Returns 0 on success; fills *out (free with gsjgen_free). */
int gsjgen_voronoi(const gsjgen_params* p, gsjgen_set* out);
void gsjgen_free(gsjgen_set* s);
/* n points uniform in the box; xy must hold 2n doubles. */
void gsjgen_points(uint64_t n, double x0, double y0, double x1, double y1, uint64_t seed, double* xy);
/* .gset / .pset writers (reference layout); ids are written as decimal geometry indices. 0 on success. */
int gsjgen_write_gset(const char* path, const gsjgen_set* s);
int gsjgen_write_pset(const char* path, uint64_t n, const double* xy);
/* .gset reader: allocates; free with gsjgen_free. 0 on success. */
int gsjgen_read_gset(const char* path, gsjgen_set* out);

#ifdef __cplusplus
}
#endif
#endif
