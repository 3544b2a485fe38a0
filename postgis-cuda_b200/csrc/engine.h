// Host-side engine internals: context, resident layers, grow-only scratch pools, launch helpers.
// Errors are thrown as gsj::Error inside the library and turned into status codes at the C ABI (capi.cu).
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <functional>
#include <tuple>
#include <utility>
#include <vector>
#include "../../include/gsj.h"
#include "geom.cuh"

namespace gsj {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define GSJ_CK(x)                                                                                                   \
  do {                                                                                                              \
    cudaError_t e_ = (x);                                                                                           \
    if (e_ != cudaSuccess)                                                                                          \
      throw ::gsj::Error(e_ == cudaErrorMemoryAllocation ? GSJ_ERR_NOMEM : GSJ_ERR_CUDA,                            \
                         std::string(#x) + ": " + cudaGetErrorString(e_) + " (" __FILE__ ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

// grow-only device scratch: the pools live in the context, so steady-state requests allocate nothing. Bound to
// the context's stream, growth is stream-ordered (cudaMallocAsync / cudaFreeAsync): it never synchronises the
// device, so one request's growth does not stall the requests running on other contexts.
struct DevBuf {
  void* p = nullptr; size_t cap = 0;
  cudaStream_t s = nullptr;
  void* get(size_t n) {
    if (n > cap) {
      if (p) { if (s) cudaFreeAsync(p, s); else cudaFree(p); }
      p = nullptr; cap = 0;
      size_t want = n + n / 4 + 256;
      if (s) GSJ_CK(cudaMallocAsync(&p, want, s));
      else GSJ_CK(cudaMalloc(&p, want));
      cap = want;
    }
    return p;
  }
  template <class T> T* as(size_t count) { return reinterpret_cast<T*>(get(count * sizeof(T) + 16)); }
  void release() { if (p) { if (s) cudaFreeAsync(p, s); else cudaFree(p); } p = nullptr; cap = 0; }
  ~DevBuf() { release(); }
};
// grow-only pinned host staging. A buffer outgrown mid-request is retired, not freed: cudaFreeHost can wait for
// the whole device, which would stall the other contexts' requests; growth doubles, so the retired ones add up to
// less than the live one, and all are freed with the context.
struct PinnedBuf {
  void* p = nullptr; size_t cap = 0;
  std::vector<void*> retired;
  void* get(size_t n) {
    if (n > cap) {
      if (p) retired.push_back(p);
      p = nullptr;
      size_t want = std::max(n + n / 4 + 256, 2 * cap);
      cap = 0;
      GSJ_CK(cudaHostAlloc(&p, want, cudaHostAllocDefault));
      cap = want;
    }
    return p;
  }
  template <class T> T* as(size_t count) { return reinterpret_cast<T*>(get(count * sizeof(T) + 16)); }
  void release() {
    if (p) cudaFreeHost(p);
    for (void* q : retired) cudaFreeHost(q);
    retired.clear();
    p = nullptr; cap = 0;
  }
  ~PinnedBuf() { release(); }
};

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr; cudaStream_t s = nullptr;
  explicit Timer(cudaStream_t st) : s(st) { GSJ_CK(cudaEventCreate(&a)); GSJ_CK(cudaEventCreate(&b)); }
  ~Timer() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
  void start() { GSJ_CK(cudaEventRecord(a, s)); }
  float stop() { GSJ_CK(cudaEventRecord(b, s)); GSJ_CK(cudaEventSynchronize(b)); float ms = 0; GSJ_CK(cudaEventElapsedTime(&ms, a, b)); return ms; }
  // without a host wait: record the end now, read the time after a later stream sync
  void mark_end() { GSJ_CK(cudaEventRecord(b, s)); }
  float elapsed() { float ms = 0; GSJ_CK(cudaEventElapsedTime(&ms, a, b)); return ms; }
};

}  // namespace gsj

struct gsj_layer {
  gsj::DLayer d;
  gsj::DBvh bvh;
  int is_points = 0;
  uint32_t nparent = 0;
  uint32_t max_geom_edges = 0;
  uint64_t bytes = 0;
  std::vector<void*> allocs;           // owned device memory
  std::vector<uint32_t> h_parent;      // host copy (batches keep the pieces of one parent together)
  const double2* pts = nullptr;        // points layer: world coordinates
  int device = 0;
};

namespace gsj {
// Kernel arguments held for a graph kernel node: each value converted to the kernel's own parameter type (so the
// argument list is checked against the kernel's signature at compile time), ptr[] pointing at them.
template <class... A>
struct KernelArgs {
  std::tuple<A...> val;
  void* ptr[sizeof...(A) ? sizeof...(A) : 1];
  explicit KernelArgs(A... a) : val(a...) { fill(std::index_sequence_for<A...>{}); }
  KernelArgs(const KernelArgs&) = delete;
  KernelArgs& operator=(const KernelArgs&) = delete;
 private:
  template <size_t... I> void fill(std::index_sequence<I...>) { ((ptr[I] = &std::get<I>(val)), ...); }
};
template <class... A, class... V>
KernelArgs<A...> kernel_args(void (*)(A...), V&&... v) {
  static_assert(sizeof...(A) == sizeof...(V), "argument count differs from the kernel's parameters");
  return KernelArgs<A...>(static_cast<A>(v)...);
}

// Launch shape of the refinement's two size bins (set by gsj_set_refine_shape or chosen by gsj_tune_refine):
// run / runs = consecutive pairs a warp of the shared-memory bin takes per fetch / fetches per warp (grid size);
// bin_cap = local edges per side up to which a pair stays in the shared-memory bin (at most its list capacity);
// scratch_wpsm = warps per SM of the global-scratch bin.
struct RefineShape { int run = 4, runs = 32, bin_cap = 128, scratch_wpsm = 32; };
// The refinement's bins as one CUDA graph per variant (shared-memory bin, then scratch bin), instantiated once per
// context and re-parameterised per call.
struct RefineGraph {
  cudaGraph_t graph = nullptr; cudaGraphExec_t exec = nullptr;
  cudaGraphNode_t n_main = nullptr, n_scr = nullptr, n_idx = nullptr, n_self = nullptr;
};
}  // namespace gsj

struct gsj_ctx {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  std::string err;
  int refine_attr = 0, dw_attr = 0, er_attr = 0;
  uint64_t launches = 0;      // kernels launched by this context (reported per call in the stats)
  uint64_t node_visits = 0;   // LBVH nodes visited by traversals (roofline accounting)
  uint64_t edge_pairs = 0;    // local edge pairs (na x nb) of the pairs refined (the refinement's work unit)
  gsj::RefineShape shape;
  gsj::RefineGraph rgraph[12];   // [variant (plain, filtered, filtered FP32) x scratch bin or not x self bin or not]
  // scratch pools
  gsj::DevBuf counters, cand, flag, area, ev, evb, heavy, selfidx, scratch, keep, opairs, oarea, oev, oevb, ocode, tmp, keys, keys2, idx,
      idx2, agg_area, agg_ev, agg_evb, agg_flag, qbb, uf, misc1, misc2, misc3,
      er_pf, er_keep, er_off, er_pairs, er_flag, er_heavy, er_tiles, er_tiles2, er_slab, er_again, er_scr, er_ctr, er_tmp,
      enc_in, enc_cnt, enc_pre, enc_blk, enc_out;
  // every scratch pool, e.g. to bind them to the stream or release them before the stream goes
  template <class Fn> void each_buf(Fn&& fn) {
    for (gsj::DevBuf* b : {&counters, &cand, &flag, &area, &ev, &evb, &heavy, &selfidx, &scratch, &keep, &opairs, &oarea, &oev, &oevb, &ocode, &tmp, &keys, &keys2, &idx, &idx2, &agg_area, &agg_ev, &agg_evb, &agg_flag, &qbb, &uf, &misc1, &misc2, &misc3, &er_pf, &er_keep, &er_off, &er_pairs, &er_flag, &er_heavy, &er_tiles, &er_tiles2, &er_slab, &er_again, &er_scr, &er_ctr, &er_tmp, &enc_in, &enc_cnt, &enc_pre, &enc_blk, &enc_out}) fn(*b);
  }
  gsj::PinnedBuf h_counters, h_refine, h_pairs, h_area, h_code, h_where, h_enc;
  bool refine_pending = false;   // a refinement's counters are on their way to h_refine (refine_enqueue)
};

namespace gsj {

inline int grid_for(uint64_t n, int block) { return (int)std::min<uint64_t>((n + block - 1) / block, (uint64_t)1 << 30); }

// kernels / drivers implemented in the .cu files
void layer_upload_polygons(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy,
                           const uint32_t* parent, const uint8_t* syn, gsj_layer* L);
void layer_upload_points(gsj_ctx* c, uint64_t n, const double* xy, gsj_layer* L);
void build_bvh(gsj_ctx* c, gsj_layer* L);
void layer_free(gsj_layer* L);

// candidate pairs of probe boxes qbb[q0 .. q0+nq) (query order: qorder or identity) against the BVH; returns count.
// Writes at most cap pairs; a count above cap means the caller must grow the buffer and re-run.
uint64_t traverse(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper,
                  uint2* out, uint64_t cap);

struct RefineArgs {
  double tol_rel, eps_par, tol_abs;
  int want_area, want_relate, snap_half_ulp;
};
using PrefilterFn = std::function<uint64_t(uint2*, uint64_t)>;
using DeviceBatchFn = std::function<void(const uint2*, const double*, uint64_t)>;
void join_device(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const RefineArgs& rp, const gsj_join_opts& o, gsj_join_stats& st,
                 const PrefilterFn& pre, const DeviceBatchFn& on_batch);
uint64_t candidates_for(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper, uint2** out);
gsj_join_opts opts_or_default(const gsj_join_opts* o);

// per-pair refinement (flag, area, ev, evb); returns the number of pairs that took the oversized path
uint64_t refine(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint2* pairs, uint64_t np, const RefineArgs& rp, int mode,
                uint8_t* flag, double* area, double4* ev, uint32_t* evb);
// the same in two halves, for callers with a stream sync of their own after it: refine_enqueue puts the bins and the
// copy of their counters on the stream; refine_result, after the caller's next sync, checks the error word and
// returns the oversized-pair count (the outputs must not be used before it returned without throwing)
void refine_enqueue(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint2* pairs, uint64_t np, const RefineArgs& rp, int mode,
                    uint8_t* flag, double* area, double4* ev, uint32_t* evb);
uint64_t refine_result(gsj_ctx* c);

// refinement launch shapes (tune.cu)
bool shape_valid(const RefineShape& s);
void tune_refine(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const RefineArgs& rp, int mode, int upper, uint64_t max_pairs, int keep,
                 gsj_tune_result* out);

// device row encoding (encode.cu)
uint64_t encode_rows(gsj_ctx* c, const gsj_rowset* P, const gsj_rowset* Q, const gsj_encode_spec* spec, const uint32_t* pairs, const double* area,
                     const uint32_t* code, const uint8_t* where, uint64_t n, gsj_bytes_sink sink, void* user);
gsj_rowset* rowset_upload(gsj_ctx* c, uint64_t n_geoms, const uint64_t* moff, const uint32_t* midx, uint64_t n_rows, const char* blob,
                          const uint64_t* off);
void rowset_free(gsj_rowset* r);

}  // namespace gsj
