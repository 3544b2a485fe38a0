/* gsj - B200-native (sm_100a) spatial-join engine: the C ABI.
 *
 * Drop-in for the engine entry points behind the gpujoind daemon of landstats-us/postgis-cuda (paths below are
 * relative to that project). Plain pointers and sizes only; every call returns an int status (0 = GSJ_OK) and
 * never exits the process (the reference's CK() aborts, engine/common.h:13-14); gsj_last_error() gives the
 * message. Host inputs are copied at upload; result pointers handed to a sink are valid only during the call
 * (as the reference's callback contract, engine/engine.cuh:1047-1055). One context per GPU; a context is used
 * by one host thread at a time (the serving loop owns it).
 */
#ifndef GSJ_H
#define GSJ_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSJ_OK 0
#define GSJ_ERR_ARG 1        /* invalid argument */
#define GSJ_ERR_CUDA 2       /* CUDA runtime error (message in gsj_last_error) */
#define GSJ_ERR_NOMEM 3      /* device or host allocation failed / admission refused */
#define GSJ_ERR_CANCELLED 4  /* the cancel flag was raised between batches */
#define GSJ_ERR_SINK 5       /* the sink returned non-zero */
#define GSJ_ERR_TIMEOUT 6    /* a bounded device-side wait expired */

typedef struct gsj_ctx gsj_ctx;
typedef struct gsj_layer gsj_layer;

/* Context on a CUDA device (replaces the daemon's process-global device state, daemon/gpujoind.cu:589-621). */
int gsj_ctx_create(int device, gsj_ctx** out);
/* The same, with the context's stream at the device's highest (high_priority != 0) or lowest priority: the kernels
 * of a high-priority context get SMs first as blocks of other contexts' kernels retire (serving: small requests
 * ahead of large ones). */
int gsj_ctx_create_prio(int device, int high_priority, gsj_ctx** out);
void gsj_ctx_destroy(gsj_ctx* ctx);
const char* gsj_last_error(const gsj_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t): every kernel and copy of the context runs on it, in call order.
 * Lets a caller bracket calls with its own CUDA events. */
void* gsj_ctx_stream(gsj_ctx* ctx);
/* Name, compute capability and memory of a CUDA device, without a context (the daemon's STATUS, gpujoind.cu:486-494).
 * GSJ_ERR_CUDA when no CUDA device can be used, GSJ_ERR_ARG for a device index out of range. */
int gsj_device_query(int device, char* name, size_t namelen, int* cc_major, int* cc_minor, uint64_t* free_bytes, uint64_t* total_bytes);
/* Free device memory and the number of SMs, for admission decisions (gpujoind.cu:133-137). */
int gsj_ctx_mem_info(gsj_ctx* ctx, uint64_t* free_bytes, uint64_t* total_bytes, int* sm_count);

/* Resident polygon layer + its LBVH: upload_set (engine/engine.cuh:42-89) followed by build_bvh (engine.cuh:197-228).
 * gro[n+1], rvo[nr+1], xy[2nv] world coordinates (closed rings, shells CCW, holes CW: daemon/loader.h:100-102).
 * parent[n] (piece -> geometry, non-decreasing) and syn[nv] (1: edge v->v+1 was created by subdivision) are
 * optional (NULL), as upload_set's parent/syn arguments. */
int gsj_layer_upload_polygons(gsj_ctx* ctx, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo,
                              const double* xy, const uint32_t* parent, const uint8_t* syn, gsj_layer** out);
/* Resident point layer + LBVH over the points' degenerate boxes: upload_points (engine.cuh:1068-1076). */
int gsj_layer_upload_points(gsj_ctx* ctx, uint64_t n, const double* xy, gsj_layer** out);
/* free_set / free_points / free_bvh (engine.cuh:91-97, 1077, 230). ctx may be NULL (no stream to drain first). */
void gsj_layer_free(gsj_ctx* ctx, gsj_layer* layer);

typedef struct gsj_layer_info {
  uint64_t n, nr, nv;     /* geometries (pieces), rings, vertices (points: n = nv, nr = 0) */
  uint32_t nparent;       /* parent geometries (== n when not subdivided) */
  int is_points;
  uint32_t max_geom_edges;
  uint64_t device_bytes;  /* resident bytes incl. the LBVH (Layer::gpu_bytes, gpujoind.cu:145) */
} gsj_layer_info;
int gsj_layer_get_info(const gsj_layer* layer, gsj_layer_info* info);

/* RefineParams (engine.cuh:517-518). Defaults: 1e-12, 1e-7, 1e-11, area on, relate off, snap off. */
typedef struct gsj_refine_params {
  double tol_rel, eps_par, tol_abs;
  int want_area, want_relate, snap_half_ulp;
} gsj_refine_params;
void gsj_refine_params_default(gsj_refine_params* p);

/* Refinement variants, the same results bit for bit: GSJ_REFINE_PLAIN = the reference's scheme (a warp per pair, every
 * lane sweeping all of the other polygon's local edges in FP64); GSJ_REFINE_FILTERED = the same FP64 decisions
 * reorganised around per-pair candidate edge-pair lists (only edge pairs whose boxes come within 2 tol are visited). */
#define GSJ_REFINE_PLAIN 0
#define GSJ_REFINE_FILTERED 1
/* GSJ_REFINE_FILTERED with its pure-sign orientation tests (the contact test, the probe point's crossing parity, the
 * point-in-ring tests of the area / relate sweeps) first decided in FP32 under a certified error bound, FP64 only
 * where the bound cannot decide: the same results, bit for bit (kept beside GSJ_REFINE_FILTERED for measured
 * comparison). Ops other than joins and clustering, and oversized pairs, run it as GSJ_REFINE_FILTERED. */
#define GSJ_REFINE_FILTERED_FP32 2

/* JoinOpts (engine.cuh:799-813). */
typedef struct gsj_join_opts {
  uint32_t batch_q;          /* probe geometries per batch (0: whole probe layer) */
  uint64_t max_pairs;        /* candidate pairs per refine launch (0: 128 Mi) */
  int upper;                 /* self-join: each unordered pair once (b >= a) */
  int no_agg;                /* report piece pairs instead of parent pairs */
  int refine_mode;           /* GSJ_REFINE_PLAIN / GSJ_REFINE_FILTERED */
  const volatile int* cancel;  /* checked between batches (Conn::broken, gpujoind.cu:225) */
  uint32_t shard, nshards;   /* probe shard `shard` of `nshards` (nshards <= 1: all probes): contiguous runs of the
                                probes' Morton order (index ranges kept whole per parent on subdivided layers); the
                                shards' results partition the join's (multi-GPU: one shard per GPU, R replicated) */
} gsj_join_opts;
void gsj_join_opts_default(gsj_join_opts* o);

/* JoinStats (engine.cuh:814) plus device-side timings of the phases. */
typedef struct gsj_join_stats {
  double traverse_ms, refine_ms, compact_ms, copy_ms;
  uint64_t candidates, hits, heavy, batches;
  uint64_t launches;     /* kernels of this library launched by the call */
  uint64_t node_visits;  /* LBVH nodes visited by the candidate search (48 bytes each) */
  uint64_t edge_pairs;   /* sum over the refined pairs of na x nb, their local edge counts (the refinement's work unit) */
} gsj_join_stats;

/* Sink for a finished batch (the host callback of join_stream): pairs[2n] = (P index, R index) in parent ids,
 * area[n] (NULL without want_area), code[n] DE-9IM codes of relate(P, R) (NULL without want_relate; 2 bits per
 * cell II IB IE BI BB BE EI EB EE, 0 = F, 1 = '0', 2 = '1', 3 = '2', engine.cuh:845-856). Return 0 to continue. */
typedef int (*gsj_join_sink)(void* user, const uint32_t* pairs, const double* area, const uint32_t* code, uint64_t n);

/* Intersects (+ area, + DE-9IM evidence) join of probe P against build R: join_stream (engine.cuh:895-1061).
 * Behind gpu_join / gpu_intersects and gpu_relate (op_join / op_relate, daemon/gpujoind.cu:210-388). */
int gsj_join(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rp, const gsj_join_opts* o,
             gsj_join_sink sink, void* user, gsj_join_stats* stats);

/* Points in polygons: join_points_stream (engine.cuh:1112-1178). Sink gets (point, parent polygon) pairs and
 * where[n] = 1 interior / 2 boundary (DE-9IM 0FFFFF212 / F0FFFF212, engine.cuh:337-338). */
typedef int (*gsj_points_sink)(void* user, const uint32_t* pairs, const uint8_t* where, uint64_t n);
int gsj_join_points(gsj_ctx* ctx, const gsj_layer* pts, const gsj_layer* R, const gsj_join_opts* o, gsj_points_sink sink,
                    void* user, gsj_join_stats* stats);

/* ST_ClusterIntersecting: cluster_intersecting (engine.cuh:1216-1234). root[nparent] = smallest parent index of each
 * parent's connected component in the intersects graph. */
int gsj_cluster(gsj_ctx* ctx, const gsj_layer* P, uint32_t nparent, const gsj_join_opts* o, uint32_t* root,
                gsj_join_stats* stats);
/* Clustering across GPUs: each GPU runs gsj_cluster on the same layer with o->shard / o->nshards (its probe shard;
 * every intersecting pair is found by exactly one shard), the root arrays are gathered, and this joins them:
 * roots[nforests * nparent] (forest f at f * nparent) -> root[nparent], the smallest parent index of each parent's
 * component in the union, i.e. gsj_cluster's answer for the whole layer. Runs on the context's GPU. */
int gsj_cluster_merge(gsj_ctx* ctx, uint32_t nparent, uint32_t nforests, const uint32_t* roots, uint32_t* root);

/* Layer preparation. Outputs are host arrays allocated by the library; free each with gsj_host_free. Both run on the
 * calling thread's current CUDA device (a context is made for the call; gsj_subdivide_gpu / gsj_dedup_gpu below take
 * one) and return GSJ_OK or an error code.
 * Subdivision (engine/subdivide.h:71-129): geometries with more than maxv vertices are cut recursively at the middle
 * of their bbox's longer side (Sutherland-Hodgman, FP64); parent[piece] = geometry, syn[v] = 1 for edges created
 * by a cut (ignored for boundary contact). Feed the result to gsj_layer_upload_polygons with parent and syn. */
int gsj_subdivide(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv,
                  uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy,
                  uint32_t** out_parent, uint8_t** out_syn);
/* Exact deduplication of identical geometries (engine/dedup.h:51-124): distinct geometries in order of first
 * occurrence (morton = 1: in Z-order of their bbox centres); members of distinct geometry g are the original
 * indices midx[moff[g] .. moff[g+1]). Results on the distinct set expand to members x members. */
int gsj_dedup(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton,
              uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy,
              uint64_t** out_moff, uint32_t** out_midx);
void gsj_host_free(void* p);
/* gsj_dedup on the context's GPU (hash, radix sort, exact comparison within equal-hash runs, gathers); the host
 * arrays are copied to the device and the results back. */
int gsj_dedup_gpu(gsj_ctx* ctx, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton,
                  uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy,
                  uint64_t** out_moff, uint32_t** out_midx);
/* gsj_subdivide on the context's GPU (breadth-first cut rounds, pieces sorted by geometry and cut path). */
int gsj_subdivide_gpu(gsj_ctx* ctx, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv,
                      uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy,
                      uint32_t** out_parent, uint8_t** out_syn);

/* Pair sink for distance / buffer joins: (P parent, R parent) pairs. */
typedef int (*gsj_pairs_sink)(void* user, const uint32_t* pairs, uint64_t n);
/* ST_DWithin(a::geography, b::geography, d) polygon x polygon: dwithin_join_stream (engine/buffer.cuh:892-991).
 * same: P and R are the same layer (pieces of one parent are within any distance; with upper). */
int gsj_dwithin(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, double d_m, int same, const gsj_join_opts* o,
                gsj_pairs_sink sink, void* user, gsj_join_stats* stats);
/* ST_Intersects(ST_Buffer(a::geography, -ra), ST_Buffer(b::geography, -rb)): erode_join_stream (buffer.cuh:765-889).
 * need_self[nparent] (host, optional): self pairs wanted for these parents (BufferQuery::need_self, buffer.cuh:694). */
int gsj_erode(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, double ra_m, double rb_m, int same, const uint8_t* need_self,
              const gsj_join_opts* o, gsj_pairs_sink sink, void* user, gsj_join_stats* stats);
/* points x polygons: ST_DWithin (k_pt_dwithin) and point in ST_Buffer(polygon, -r) (k_pt_erode):
 * points_buffer_join_stream (buffer.cuh:1137-1231). Sink gets (point, parent polygon) pairs. */
int gsj_points_dwithin(gsj_ctx* ctx, const gsj_layer* pts, const gsj_layer* R, double d_m, const gsj_join_opts* o,
                       gsj_pairs_sink sink, void* user, gsj_join_stats* stats);
int gsj_points_erode(gsj_ctx* ctx, const gsj_layer* pts, const gsj_layer* R, double r_m, const gsj_join_opts* o,
                     gsj_pairs_sink sink, void* user, gsj_join_stats* stats);

/* Parity / diagnostics: candidate pairs of the LBVH traversal (k_traverse, engine.cuh:233-259) and the per-pair
 * refinement outputs of k_refine (engine.cuh:530-636) for given piece pairs: flag 0/1/2, area, ev[4n]
 * (inside / on lengths of A's then B's real boundary), evb bits. Output arrays are host memory, NULL to skip. */
int gsj_candidates(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, int upper, gsj_pairs_sink sink, void* user);
int gsj_refine_pairs(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, const uint32_t* pairs, uint64_t np,
                     const gsj_refine_params* rp, int refine_mode, uint8_t* flag, double* area, double* ev, uint32_t* evb);

/* Refinement of candidate pairs for callers that cannot allocate device memory. No counterpart in the
 * reference: its engine allocates scratch on every call. For callers that must not call cudaMalloc once running
 * (a server working inside a device-memory budget reserved up front, or a request path that cannot take
 * cudaMalloc/cudaFree's implicit device synchronisation). Same outputs as gsj_refine_pairs, but every pointer is
 * DEVICE memory owned by the caller: d_pairs[2np] (P index, R index), d_flag[np], optional d_area[np], optional
 * d_ev[4np] with d_evb[np]. Its scratch is one static device array of GSJ_NOALLOC_SCRATCH_BYTES per GPU (held by
 * every GPU that loads the library, until exit); layers whose largest geometry needs a larger per-warp slab
 * (more than ~466k edges) are rejected with GSJ_ERR_ARG. All calls share that array: calls that overlap on the GPU
 * race and must be serialised. The address of the array is looked up on the first call on a device and kept until
 * the process exits: do not call this on a device after resetting it (cudaDeviceReset). Runs on the context's
 * stream and synchronises it before returning (it reads a status word back), so a call cannot be captured into a
 * CUDA graph. */
#define GSJ_NOALLOC_SCRATCH_BYTES (32u << 20)
int gsj_refine_pairs_noalloc(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, const uint32_t* d_pairs, uint64_t np,
                             const gsj_refine_params* rp, uint8_t* d_flag, double* d_area, double* d_ev, uint32_t* d_evb);

/* Launch shape of the refinement's two size bins, per context. No counterpart in the reference (its k_refine takes a
 * fixed grid, engine.cuh:963-975). Pairs whose local edge lists fit bin_edges per side run in the shared-memory bin
 * (a warp per pair, warps taking `run` consecutive pairs per fetch, at most `runs` fetches each); the others in the
 * global-scratch bin with scratch_warps_per_sm warps per SM. Every shape gives the same results, bit for bit; only
 * the time changes. Defaults: 4, 32, 128, 32. */
typedef struct gsj_refine_shape {
  int run;                   /* 1 - 64 */
  int runs;                  /* 1 - 4096 */
  int bin_edges;             /* 8 - 128 */
  int scratch_warps_per_sm;  /* 1 - 64 */
} gsj_refine_shape;
int gsj_get_refine_shape(const gsj_ctx* ctx, gsj_refine_shape* out);
int gsj_set_refine_shape(gsj_ctx* ctx, const gsj_refine_shape* shape);   /* GSJ_ERR_ARG when a field is out of range */

/* Autotuner: times the refinement of P x R's candidate pairs (upper: b >= a only, for self-joins) under launch
 * shapes searched one field at a time from the context's current shape, on a sample of at most max_pairs candidate
 * pairs (0: 2^20; 16 evenly spaced runs of consecutive pairs, keeping the traversal order's locality), and sets the
 * fastest on the context. Fields named in keep (GSJ_TUNE_KEEP_*) stay as they are: e.g. a server whose requests
 * share the GPU keeps `runs`, which bounds how long a block holds an SM before other streams' kernels get it.
 * Each shape's outputs are compared with the starting shape's, bit for bit; a difference fails the call
 * (GSJ_ERR_CUDA) and leaves the shape unchanged. Takes a few seconds at most on large samples. */
#define GSJ_TUNE_KEEP_RUN 1
#define GSJ_TUNE_KEEP_RUNS 2
#define GSJ_TUNE_KEEP_BIN 4
#define GSJ_TUNE_KEEP_SCRATCH 8
typedef struct gsj_tune_result {
  gsj_refine_shape best;
  double start_ms, best_ms;   /* device time of one refinement of the sample: starting shape, chosen shape */
  uint64_t sample_pairs;
  uint32_t shapes_tried;
} gsj_tune_result;
int gsj_tune_refine(gsj_ctx* ctx, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rp, int refine_mode, int upper,
                    uint64_t max_pairs, int keep, gsj_tune_result* out);

/* Row encoding on the device (replaces the daemon's host encoder, send_parallel / FrameBuf, gpujoind.cu:178-206).
 * A rowset is a device copy of a layer's row ids (id_blob bytes, id_off[n_rows + 1] offsets) and, for a deduplicated
 * layer, its members (moff[n_geoms + 1], midx: the rows each distinct geometry stands for; NULL: geometry = row).
 * gsj_encode_rows turns n engine results (host arrays as the sinks receive them) into the gpujoind byte stream of
 * frames {u32 nrows, rows}, rows as gpujoind writes them (u16 length + id, u16 length + id, then the payload), and
 * calls sink(user, bytes, nbytes, nrows) once with complete frames (not with an empty stream). Modes:
 *   GSJ_ENC_PAIRS   polygon pairs (a, b) of P x Q expanded by the row rules (members x members; same: "all"
 *                   mirrors, "distinct" keeps one of each; gpujoind.cu:271-283), payload f64 area[i] or NaN (area NULL)
 *   GSJ_ENC_RELATE  the same rows, payload the 9-char DE-9IM of code[i] (transposed for mirrored rows), kept when it
 *                   matches pattern (empty: all) (gpujoind.cu:356-367)
 *   GSJ_ENC_POINTS  (point p, polygon q) pairs: one row per member of q, payload f64 point_value; swapped: the
 *                   polygon's id first (gpujoind.cu:244-252, 460-468)
 *   GSJ_ENC_POINT_RELATE  the same rows, payload relate(point, polygon) from where[i] (2: boundary, else interior),
 *                   transposed when swapped, kept when it matches pattern
 * P holds the ids of the pairs' first members, Q of the second (for same, pass the same rowset twice).
 * Frames hold whole pairs' rows, ~1 MiB each for ids up to ~16 bytes; frame boundaries are not the host
 * encoder's, the rows are the same. Runs on the context's stream; returns after the sink returned. It may be called
 * from inside a join's sink on the same context (its scratch is its own; the join continues after it on the stream).
 * Ids longer than 65535 bytes are cut to 65535, as the host encoder does. */
typedef struct gsj_rowset gsj_rowset;
enum { GSJ_ENC_PAIRS = 0, GSJ_ENC_RELATE = 1, GSJ_ENC_POINTS = 2, GSJ_ENC_POINT_RELATE = 3 };
typedef struct {
  int mode, same, distinct, swapped;
  double point_value;
  char pattern[10];   /* 9 chars + NUL, or "" */
} gsj_encode_spec;
typedef int (*gsj_bytes_sink)(void* user, const uint8_t* bytes, uint64_t nbytes, uint64_t nrows);
int gsj_rowset_upload(gsj_ctx* ctx, uint64_t n_geoms, const uint64_t* moff, const uint32_t* midx, uint64_t n_rows, const char* id_blob,
                      const uint64_t* id_off, gsj_rowset** out);
void gsj_rowset_free(gsj_rowset* rs);
int gsj_encode_rows(gsj_ctx* ctx, const gsj_rowset* P, const gsj_rowset* Q, const gsj_encode_spec* spec, const uint32_t* pairs,
                    const double* area, const uint32_t* code, const uint8_t* where, uint64_t n, gsj_bytes_sink sink, void* user,
                    uint64_t* rows_out);

/* DE-9IM helpers: de9im_str / de9im_transpose / de9im_match (engine.cuh:871-888). out gets 9 chars (no NUL). */
void gsj_de9im_str(uint32_t code, char* out9);
uint32_t gsj_de9im_transpose(uint32_t code);
int gsj_de9im_match(uint32_t code, const char* pattern9);

#ifdef __cplusplus
}
#endif
#endif
