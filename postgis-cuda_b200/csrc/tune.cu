// Autotuner for the refinement's launch shape (run, runs, bin_edges, scratch warps per SM). No counterpart in the
// reference, whose refinement grid is fixed (engine/engine.cuh:963-975). It times the refinement of a sample of the
// layer pair's candidate pairs under each shape of a one-field-at-a-time search, checks every shape's outputs
// against the starting shape's bit for bit (the shape moves work between bins and warps, never changes a decision),
// and keeps the fastest on the context.
#include "engine.h"

namespace gsj {

// mismatches between two refinements of the same pairs (areas compared as bit patterns)
__global__ void k_refine_diff(const uint8_t* f0, const uint8_t* f1, const double* a0, const double* a1, const double4* e0, const double4* e1,
                              const uint32_t* b0, const uint32_t* b1, uint64_t n, unsigned long long* bad) {
  unsigned long long d = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    bool x = f0[i] != f1[i];
    if (a0) x |= __double_as_longlong(a0[i]) != __double_as_longlong(a1[i]);
    if (e0) {
      const double4 u = e0[i], v = e1[i];
      x |= __double_as_longlong(u.x) != __double_as_longlong(v.x) || __double_as_longlong(u.y) != __double_as_longlong(v.y) ||
           __double_as_longlong(u.z) != __double_as_longlong(v.z) || __double_as_longlong(u.w) != __double_as_longlong(v.w) || b0[i] != b1[i];
    }
    d += x;
  }
  if (d) atomicAdd(bad, d);
}

bool shape_valid(const RefineShape& s) {
  return s.run >= 1 && s.run <= 64 && s.runs >= 1 && s.runs <= 4096 && s.bin_cap >= 8 && s.bin_cap <= 128 && s.scratch_wpsm >= 1 &&
         s.scratch_wpsm <= 64;
}

namespace {
struct DevTmp {   // stream-ordered temporary, freed on the same stream
  void* p = nullptr; cudaStream_t s;
  DevTmp(size_t n, cudaStream_t st) : s(st) { GSJ_CK(cudaMallocAsync(&p, n ? n : 16, s)); }
  ~DevTmp() { if (p) cudaFreeAsync(p, s); }
  template <class T> T* as() { return static_cast<T*>(p); }
};
struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  Events() { GSJ_CK(cudaEventCreate(&a)); GSJ_CK(cudaEventCreate(&b)); }
  ~Events() { cudaEventDestroy(a); cudaEventDestroy(b); }
};
}  // namespace

void tune_refine(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const RefineArgs& rp, int mode, int upper, uint64_t max_pairs, int keep,
                 gsj_tune_result* out) {
  if (P->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "the refinement autotuner needs two polygon layers");
  if (mode != GSJ_REFINE_PLAIN && mode != GSJ_REFINE_FILTERED && mode != GSJ_REFINE_FILTERED_FP32) throw Error(GSJ_ERR_ARG, "unknown refine mode");
  cudaStream_t s = c->stream;
  if (!max_pairs) max_pairs = 1u << 20;
  // candidate pairs of the whole probe layer in its Morton order (the join's probe order)
  uint2* cand = nullptr;
  const uint64_t nc = candidates_for(c, P->d.bb, P->bvh.order, 0, P->d.n, R->bvh, upper, &cand);
  if (!nc) throw Error(GSJ_ERR_ARG, "the layers have no candidate pairs to tune on");
  const uint64_t n = std::min(nc, max_pairs);
  DevTmp sample(n * sizeof(uint2), s);
  if (n == nc) {
    GSJ_CK(cudaMemcpyAsync(sample.p, cand, n * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
  } else {   // 16 evenly spaced runs of consecutive pairs
    const int K = 16;
    uint64_t at = 0;
    for (int k = 0; k < K; k++) {
      const uint64_t len = n / K + (k < (int)(n % K) ? 1 : 0);
      const uint64_t src = (nc - len) * k / (K - 1);
      GSJ_CK(cudaMemcpyAsync(sample.as<uint2>() + at, cand + src, len * sizeof(uint2), cudaMemcpyDeviceToDevice, s));
      at += len;
    }
  }
  const bool rel = rp.want_relate != 0, ar = rp.want_area != 0;
  // the starting shape's outputs, kept for the comparisons
  DevTmp f0(n, s), a0(ar ? n * 8 : 0, s), e0(rel ? n * 32 : 0, s), b0(rel ? n * 4 : 0, s), bad(8, s);
  uint8_t* flag = c->flag.as<uint8_t>(n);
  double* area = ar ? c->area.as<double>(n) : nullptr;
  double4* ev = rel ? c->ev.as<double4>(n) : nullptr;
  uint32_t* evb = rel ? c->evb.as<uint32_t>(n) : nullptr;
  const RefineShape start = c->shape;
  Events ev_t;
  auto time_once = [&]() -> double {
    GSJ_CK(cudaEventRecord(ev_t.a, s));
    refine(c, P, R, sample.as<uint2>(), n, rp, mode, flag, area, ev, evb);   // returns after its stream sync
    GSJ_CK(cudaEventRecord(ev_t.b, s));
    GSJ_CK(cudaEventSynchronize(ev_t.b));
    float ms = 0;
    GSJ_CK(cudaEventElapsedTime(&ms, ev_t.a, ev_t.b));
    return ms;
  };
  auto measure = [&](const RefineShape& sh) -> double {   // one untimed run, then the best of three
    c->shape = sh;
    time_once();
    double best = 1e300;
    for (int r = 0; r < 3; r++) best = std::min(best, time_once());
    return best;
  };
  uint32_t tried = 0;
  double t_start = 0;
  try {
    t_start = measure(start);
    tried++;
    GSJ_CK(cudaMemcpyAsync(f0.p, flag, n, cudaMemcpyDeviceToDevice, s));
    if (ar) GSJ_CK(cudaMemcpyAsync(a0.p, area, n * 8, cudaMemcpyDeviceToDevice, s));
    if (rel) {
      GSJ_CK(cudaMemcpyAsync(e0.p, ev, n * 32, cudaMemcpyDeviceToDevice, s));
      GSJ_CK(cudaMemcpyAsync(b0.p, evb, n * 4, cudaMemcpyDeviceToDevice, s));
    }
    auto same_as_start = [&]() {
      unsigned long long h = 0;
      GSJ_CK(cudaMemsetAsync(bad.p, 0, 8, s));
      k_refine_diff<<<std::min<uint64_t>((n + 255) / 256, (uint64_t)c->sm_count * 8), 256, 0, s>>>(
          f0.as<uint8_t>(), flag, ar ? a0.as<double>() : nullptr, area, rel ? e0.as<double4>() : nullptr, ev, rel ? b0.as<uint32_t>() : nullptr, evb, n,
          bad.as<unsigned long long>());
      c->launches++;
      GSJ_CK(cudaMemcpyAsync(&h, bad.p, 8, cudaMemcpyDeviceToHost, s));
      GSJ_CK(cudaStreamSynchronize(s));
      return h;
    };
    RefineShape best = start;
    double t_best = t_start;
    const uint32_t maxe = std::max(P->max_geom_edges, R->max_geom_edges);
    // one field at a time; a shape replaces the best only when more than 1 % faster (timing noise)
    for (int field = 0; field < 4; field++) {
      if (keep & (1 << field)) continue;   // GSJ_TUNE_KEEP_RUN, _RUNS, _BIN, _SCRATCH
      std::vector<int> vals;
      if (field == 0) { if (mode == GSJ_REFINE_PLAIN) continue; vals = {1, 2, 4, 8, 16}; }
      if (field == 1) { if (mode == GSJ_REFINE_PLAIN) continue; vals = {8, 16, 32, 64, 128, 512, 4096}; }
      if (field == 2) vals = {32, 64, 96, 128};
      if (field == 3) { if (maxe <= (uint32_t)best.bin_cap) continue; vals = {8, 16, 32, 48}; }
      const RefineShape base = best;
      for (int v : vals) {
        RefineShape sh = base;
        (field == 0 ? sh.run : field == 1 ? sh.runs : field == 2 ? sh.bin_cap : sh.scratch_wpsm) = v;
        if (field == 0 && sh.run == base.run) continue;
        if (field == 1 && sh.runs == base.runs) continue;
        if (field == 2 && sh.bin_cap == base.bin_cap) continue;
        if (field == 3 && sh.scratch_wpsm == base.scratch_wpsm) continue;
        const double t = measure(sh);
        tried++;
        if (const unsigned long long d = same_as_start())
          throw Error(GSJ_ERR_CUDA, "autotuner: shape (" + std::to_string(sh.run) + ", " + std::to_string(sh.runs) + ", " + std::to_string(sh.bin_cap) +
                                        ", " + std::to_string(sh.scratch_wpsm) + ") changed " + std::to_string(d) + " refinement outputs");
        if (t < 0.99 * t_best) { t_best = t; best = sh; }
      }
    }
    c->shape = best;
    if (out) {
      out->best = gsj_refine_shape{best.run, best.runs, best.bin_cap, best.scratch_wpsm};
      out->start_ms = t_start;
      out->best_ms = t_best;
      out->sample_pairs = n;
      out->shapes_tried = tried;
    }
  } catch (...) {
    c->shape = start;
    throw;
  }
  GSJ_CK(cudaStreamSynchronize(s));
}

}  // namespace gsj
