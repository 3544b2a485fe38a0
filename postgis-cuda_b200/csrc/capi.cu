// The C ABI (include/gsj.h): status codes instead of exits, exceptions stop here.
#include <cstdlib>
#include <cstring>
#include <functional>
#include "engine.h"

namespace gsj {
RefineArgs to_args(const gsj_refine_params* p);
void join_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rpp, const gsj_join_opts* op, gsj_join_sink sink,
               void* user, gsj_join_stats* stp);
void points_host(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, const gsj_join_opts* op, gsj_points_sink sink, void* user,
                 gsj_join_stats* stp);
void cluster_host(gsj_ctx* c, const gsj_layer* P, uint32_t nparent, const gsj_join_opts* op, uint32_t* root, gsj_join_stats* stp);
void cluster_merge_host(gsj_ctx* c, uint32_t nparent, uint32_t nforests, const uint32_t* roots, uint32_t* out);
void candidates_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, int upper, gsj_pairs_sink sink, void* user);
void refine_pairs_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint32_t* pairs, uint64_t np, const gsj_refine_params* rpp,
                       int mode, uint8_t* flag, double* area, double* ev, uint32_t* evb);
void dwithin_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double d, int same, const gsj_join_opts* op, gsj_pairs_sink sink, void* user,
                  gsj_join_stats* stp);
void erode_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double ra, double rb, int same, const uint8_t* need_self, const gsj_join_opts* op,
                gsj_pairs_sink sink, void* user, gsj_join_stats* stp);
void points_buffer_host(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, double d, int erode, const gsj_join_opts* op, gsj_pairs_sink sink,
                        void* user, gsj_join_stats* stp);
void dedup_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton,
               uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint64_t** out_moff,
               uint32_t** out_midx);
void subdivide_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv,
                   uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint32_t** out_parent,
                   uint8_t** out_syn);
}  // namespace gsj

using gsj::Error;

template <class F> static int guard(gsj_ctx* c, F&& f) {
  try {
    if (c) GSJ_CK(cudaSetDevice(c->device));
    f();
    if (c) c->err.clear();
    return GSJ_OK;
  } catch (const Error& e) {
    if (c) c->err = e.what();
    if (e.code == GSJ_ERR_CUDA || e.code == GSJ_ERR_NOMEM) (void)cudaGetLastError();   // clear a sticky-free error state
    return e.code;
  } catch (const std::bad_alloc&) {
    if (c) c->err = "host allocation failed";
    return GSJ_ERR_NOMEM;
  } catch (const std::exception& e) {
    if (c) c->err = e.what();
    return GSJ_ERR_ARG;
  }
}

extern "C" {

static int ctx_create(int device, int high_priority, gsj_ctx** out) {
  if (!out) return GSJ_ERR_ARG;
  *out = nullptr;
  gsj_ctx* c = new gsj_ctx();
  c->device = device;
  int rc = guard(c, [&] {
    int nd = 0;
    GSJ_CK(cudaGetDeviceCount(&nd));
    if (device < 0 || device >= nd) throw Error(GSJ_ERR_ARG, "no such CUDA device");
    GSJ_CK(cudaSetDevice(device));
    GSJ_CK(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    int lo = 0, hi = 0;
    GSJ_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));   // hi is the numerically smallest, most urgent
    GSJ_CK(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, high_priority ? hi : lo));
    // stream-ordered scratch: keep freed pool memory cached in the process (growth never goes back to the driver)
    cudaMemPool_t pool;
    GSJ_CK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    GSJ_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    c->each_buf([&](gsj::DevBuf& b) { b.s = c->stream; });
  });
  if (rc) { delete c; return rc; }
  *out = c;
  return GSJ_OK;
}

int gsj_ctx_create(int device, gsj_ctx** out) { return ctx_create(device, 0, out); }
int gsj_ctx_create_prio(int device, int high_priority, gsj_ctx** out) { return ctx_create(device, high_priority, out); }

void gsj_ctx_destroy(gsj_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) {
    c->each_buf([](gsj::DevBuf& b) { b.release(); });   // stream-ordered frees before the stream goes
    cudaStreamSynchronize(c->stream);
    for (auto& g : c->rgraph) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
    }
    cudaStreamDestroy(c->stream);
  }
  delete c;
}

const char* gsj_last_error(const gsj_ctx* c) { return c ? c->err.c_str() : "no context"; }

void* gsj_ctx_stream(gsj_ctx* c) { return c ? (void*)c->stream : nullptr; }

int gsj_device_query(int device, char* name, size_t namelen, int* cc_major, int* cc_minor, uint64_t* free_bytes, uint64_t* total_bytes) {
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess) { (void)cudaGetLastError(); return GSJ_ERR_CUDA; }
  if (device < 0 || device >= nd) return GSJ_ERR_ARG;
  cudaDeviceProp p;
  if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&p, device) != cudaSuccess) { (void)cudaGetLastError(); return GSJ_ERR_CUDA; }
  if (name && namelen) { std::strncpy(name, p.name, namelen - 1); name[namelen - 1] = 0; }
  if (cc_major) *cc_major = p.major;
  if (cc_minor) *cc_minor = p.minor;
  size_t f = 0, t = 0;
  if (cudaMemGetInfo(&f, &t) != cudaSuccess) { (void)cudaGetLastError(); return GSJ_ERR_CUDA; }
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return GSJ_OK;
}

int gsj_dedup_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton,
                  uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint64_t** out_moff,
                  uint32_t** out_midx) {
  if (!c) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::dedup_gpu(c, n, nr, nv, gro, rvo, xy, morton, out_n, out_nr, out_nv, out_gro, out_rvo, out_xy, out_moff, out_midx); });
}

int gsj_subdivide_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv,
                      uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy,
                      uint32_t** out_parent, uint8_t** out_syn) {
  if (!c) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::subdivide_gpu(c, n, nr, nv, gro, rvo, xy, maxv, out_n, out_nr, out_nv, out_gro, out_rvo, out_xy, out_parent, out_syn); });
}

// The context-free forms run on the calling thread's current CUDA device, with a context made for the call.
static int on_current_device(const std::function<int(gsj_ctx*)>& fn) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { (void)cudaGetLastError(); return GSJ_ERR_CUDA; }
  gsj_ctx* c = nullptr;
  const int rc = ctx_create(dev, 0, &c);
  if (rc) return rc;
  const int r = fn(c);
  gsj_ctx_destroy(c);
  return r;
}

int gsj_subdivide(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv, uint64_t* out_n,
                  uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint32_t** out_parent,
                  uint8_t** out_syn) {
  return on_current_device([&](gsj_ctx* c) {
    return gsj_subdivide_gpu(c, n, nr, nv, gro, rvo, xy, maxv, out_n, out_nr, out_nv, out_gro, out_rvo, out_xy, out_parent, out_syn);
  });
}

int gsj_dedup(uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton, uint64_t* out_n,
              uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint64_t** out_moff, uint32_t** out_midx) {
  return on_current_device([&](gsj_ctx* c) {
    return gsj_dedup_gpu(c, n, nr, nv, gro, rvo, xy, morton, out_n, out_nr, out_nv, out_gro, out_rvo, out_xy, out_moff, out_midx);
  });
}

void gsj_host_free(void* p) { free(p); }

int gsj_ctx_mem_info(gsj_ctx* c, uint64_t* fr, uint64_t* tot, int* sms) {
  if (!c) return GSJ_ERR_ARG;
  return guard(c, [&] {
    size_t f = 0, t = 0;
    GSJ_CK(cudaMemGetInfo(&f, &t));
    if (fr) *fr = f;
    if (tot) *tot = t;
    if (sms) *sms = c->sm_count;
  });
}

int gsj_layer_upload_polygons(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy,
                              const uint32_t* parent, const uint8_t* syn, gsj_layer** out) {
  if (!c || !out) return GSJ_ERR_ARG;
  *out = nullptr;
  gsj_layer* L = new gsj_layer();
  L->device = c->device;
  int rc = guard(c, [&] { gsj::layer_upload_polygons(c, n, nr, nv, gro, rvo, xy, parent, syn, L); });
  if (rc) { gsj::layer_free(L); delete L; return rc; }
  *out = L;
  return GSJ_OK;
}

int gsj_layer_upload_points(gsj_ctx* c, uint64_t n, const double* xy, gsj_layer** out) {
  if (!c || !out) return GSJ_ERR_ARG;
  *out = nullptr;
  gsj_layer* L = new gsj_layer();
  L->device = c->device;
  int rc = guard(c, [&] { gsj::layer_upload_points(c, n, xy, L); });
  if (rc) { gsj::layer_free(L); delete L; return rc; }
  *out = L;
  return GSJ_OK;
}

void gsj_layer_free(gsj_ctx* c, gsj_layer* L) {
  if (!L) return;
  if (c) { cudaSetDevice(c->device); if (c->stream) cudaStreamSynchronize(c->stream); }
  else cudaSetDevice(L->device);
  gsj::layer_free(L);
  delete L;
}

int gsj_layer_get_info(const gsj_layer* L, gsj_layer_info* info) {
  if (!L || !info) return GSJ_ERR_ARG;
  info->n = L->d.n; info->nr = L->d.nr; info->nv = L->d.nv; info->nparent = L->nparent; info->is_points = L->is_points;
  info->max_geom_edges = L->max_geom_edges; info->device_bytes = L->bytes;
  return GSJ_OK;
}

void gsj_refine_params_default(gsj_refine_params* p) {
  if (!p) return;
  p->tol_rel = 1e-12; p->eps_par = 1e-7; p->tol_abs = 1e-11;
  p->want_area = 1; p->want_relate = 0; p->snap_half_ulp = 0;
}

void gsj_join_opts_default(gsj_join_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->batch_q = 0; o->max_pairs = 0; o->upper = 0; o->no_agg = 0; o->refine_mode = GSJ_REFINE_FILTERED; o->cancel = nullptr;
}

int gsj_join(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rp, const gsj_join_opts* o, gsj_join_sink sink,
             void* user, gsj_join_stats* st) {
  if (!c || !P || !R) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::join_host(c, P, R, rp, o, sink, user, st); });
}

int gsj_join_points(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, const gsj_join_opts* o, gsj_points_sink sink, void* user,
                    gsj_join_stats* st) {
  if (!c || !pts || !R) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::points_host(c, pts, R, o, sink, user, st); });
}

int gsj_cluster(gsj_ctx* c, const gsj_layer* P, uint32_t nparent, const gsj_join_opts* o, uint32_t* root, gsj_join_stats* st) {
  if (!c || !P || !root) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::cluster_host(c, P, nparent, o, root, st); });
}
int gsj_cluster_merge(gsj_ctx* c, uint32_t nparent, uint32_t nforests, const uint32_t* roots, uint32_t* root) {
  if (!c || (nparent && (!root || (nforests && !roots)))) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::cluster_merge_host(c, nparent, nforests, roots, root); });
}

int gsj_dwithin(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double d, int same, const gsj_join_opts* o, gsj_pairs_sink sink, void* user,
                gsj_join_stats* st) {
  if (!c || !P || !R || !(d >= 0)) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::dwithin_host(c, P, R, d, same, o, sink, user, st); });
}

int gsj_erode(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, double ra, double rb, int same, const uint8_t* need_self, const gsj_join_opts* o,
              gsj_pairs_sink sink, void* user, gsj_join_stats* st) {
  if (!c || !P || !R || !(ra >= 0) || !(rb >= 0)) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::erode_host(c, P, R, ra, rb, same, need_self, o, sink, user, st); });
}

int gsj_points_dwithin(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, double d, const gsj_join_opts* o, gsj_pairs_sink sink, void* user,
                       gsj_join_stats* st) {
  if (!c || !pts || !R || !(d >= 0)) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::points_buffer_host(c, pts, R, d, 0, o, sink, user, st); });
}

int gsj_points_erode(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, double r, const gsj_join_opts* o, gsj_pairs_sink sink, void* user,
                     gsj_join_stats* st) {
  if (!c || !pts || !R || !(r >= 0)) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::points_buffer_host(c, pts, R, r, 1, o, sink, user, st); });
}

int gsj_candidates(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, int upper, gsj_pairs_sink sink, void* user) {
  if (!c || !P || !R) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::candidates_host(c, P, R, upper, sink, user); });
}

int gsj_refine_pairs(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint32_t* pairs, uint64_t np, const gsj_refine_params* rp,
                     int mode, uint8_t* flag, double* area, double* ev, uint32_t* evb) {
  if (!c || !P || !R || (np && !pairs)) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::refine_pairs_host(c, P, R, pairs, np, rp, mode, flag, area, ev, evb); });
}

int gsj_get_refine_shape(const gsj_ctx* c, gsj_refine_shape* out) {
  if (!c || !out) return GSJ_ERR_ARG;
  *out = gsj_refine_shape{c->shape.run, c->shape.runs, c->shape.bin_cap, c->shape.scratch_wpsm};
  return GSJ_OK;
}

int gsj_set_refine_shape(gsj_ctx* c, const gsj_refine_shape* sh) {
  if (!c || !sh) return GSJ_ERR_ARG;
  const gsj::RefineShape v{sh->run, sh->runs, sh->bin_edges, sh->scratch_warps_per_sm};
  if (!gsj::shape_valid(v)) { c->err = "refine shape field out of range"; return GSJ_ERR_ARG; }
  c->shape = v;
  return GSJ_OK;
}

int gsj_tune_refine(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rp, int mode, int upper, uint64_t max_pairs,
                    int keep, gsj_tune_result* out) {
  if (!c || !P || !R) return GSJ_ERR_ARG;
  return guard(c, [&] { gsj::tune_refine(c, P, R, gsj::to_args(rp), mode, upper, max_pairs, keep, out); });
}

int gsj_rowset_upload(gsj_ctx* c, uint64_t n_geoms, const uint64_t* moff, const uint32_t* midx, uint64_t n_rows, const char* id_blob,
                      const uint64_t* id_off, gsj_rowset** out) {
  if (!c || !out || !id_off || (moff && !midx) || (id_off[n_rows] && !id_blob)) return GSJ_ERR_ARG;
  *out = nullptr;
  return guard(c, [&] { *out = gsj::rowset_upload(c, n_geoms, moff, midx, n_rows, id_blob, id_off); });
}
void gsj_rowset_free(gsj_rowset* rs) { gsj::rowset_free(rs); }
int gsj_encode_rows(gsj_ctx* c, const gsj_rowset* P, const gsj_rowset* Q, const gsj_encode_spec* spec, const uint32_t* pairs, const double* area,
                    const uint32_t* code, const uint8_t* where, uint64_t n, gsj_bytes_sink sink, void* user, uint64_t* rows_out) {
  if (!c || !P || !Q || !spec || (n && !pairs)) return GSJ_ERR_ARG;
  if (rows_out) *rows_out = 0;
  return guard(c, [&] {
    const uint64_t r = gsj::encode_rows(c, P, Q, spec, pairs, area, code, where, n, sink, user);
    if (rows_out) *rows_out = r;
  });
}

void gsj_de9im_str(uint32_t code, char* out) {
  for (int k = 0; k < 9; k++) out[k] = "F012"[(code >> (2 * k)) & 3];
}

uint32_t gsj_de9im_transpose(uint32_t c) {
  uint32_t t = 0;
  for (int r = 0; r < 3; r++)
    for (int q = 0; q < 3; q++) t |= ((c >> (2 * (3 * r + q))) & 3) << (2 * (3 * q + r));
  return t;
}

int gsj_de9im_match(uint32_t code, const char* pat) {
  if (!pat) return 0;
  for (int k = 0; k < 9; k++) {
    const char p = pat[k];
    const uint32_t v = (code >> (2 * k)) & 3;
    if (p == '*') continue;
    if (p == 'T' || p == 't') { if (v == 0) return 0; continue; }
    if (p == 'F' || p == 'f') { if (v != 0) return 0; continue; }
    if (p >= '0' && p <= '2') { if (v != (uint32_t)(p - '0') + 1) return 0; continue; }
    return 0;
  }
  return 1;
}

}  // extern "C"
