// Join drivers: batching, traversal -> refinement -> compaction (+ piece -> parent folding, DE-9IM codes) ->
// host sink. The stream structure of the reference's join_stream / join_points_stream / cluster_intersecting
// (engine/engine.cuh:895-1234) on one CUDA stream, with grow-only scratch pools in the context instead of
// per-request allocations.
#include <algorithm>
#include <cub/cub.cuh>
#include "engine.h"

namespace gsj {

// ---- small kernels -------------------------------------------------------------------------------------------
__global__ void k_keep(const uint8_t* __restrict__ f, uint64_t n, int any_nonzero, uint32_t* keep) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep[i] = any_nonzero ? (f[i] != 0) : (f[i] == 1);
}

// DE-9IM code from boundary evidence (engine.cuh:848-856)
__device__ __forceinline__ uint32_t de9im_code(double4 e, uint32_t bits, double LA, double LB) {
  const double ta = 1e-9 * LA, tb = 1e-9 * LB;
  bool aIn = e.x > ta, aOut = (LA - e.x - e.y) > ta, bIn = e.z > tb, bOut = (LB - e.z - e.w) > tb;
  bool same = bits & REL_COIN_SAME, opp = bits & REL_COIN_OPP, touch = bits & REL_TOUCH;
  uint32_t II = (aIn || bIn || same) ? 3 : 0, IB = bIn ? 2 : 0, IE = (aOut || bIn || opp) ? 3 : 0;
  uint32_t BI = aIn ? 2 : 0, BB = (same || opp) ? 2 : (touch ? 1 : 0), BE = aOut ? 2 : 0;
  uint32_t EI = (bOut || aIn || opp) ? 3 : 0, EB = bOut ? 2 : 0, EE = 3;
  return II | IB << 2 | IE << 4 | BI << 6 | BB << 8 | BE << 10 | EI << 12 | EB << 14 | EE << 16;
}

// scatter kept pairs (exclusive scan offsets), with their area and DE-9IM code
__global__ void k_scatter_rows(const uint2* __restrict__ pairs, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off, uint64_t n,
                               const double* area, const double4* ev, const uint32_t* evb, const double* blA, const double* blB,
                               uint2* opairs, double* oarea, uint32_t* ocode) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  uint32_t o = off[i];
  uint2 p = pairs[i];
  opairs[o] = p;
  if (oarea) oarea[o] = area[i];
  if (ocode) ocode[o] = de9im_code(ev[i], evb[i], blA[p.x], blB[p.y]);
}

// pieces kept for folding: sort keys (piece pair, then parent pair) and the per-pair payload
__global__ void k_scatter_pieces(const uint2* __restrict__ pairs, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ off, uint64_t n,
                                 const uint32_t* parA, const uint32_t* parB, unsigned long long* kpiece, uint32_t* idx) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  uint32_t o = off[i];
  uint2 p = pairs[i];
  kpiece[o] = ((unsigned long long)p.x << 32) | p.y;
  idx[o] = (uint32_t)i;
  (void)parA; (void)parB;
}
__global__ void k_parent_keys(const uint32_t* __restrict__ idx, uint64_t n, const uint2* __restrict__ pairs, const uint32_t* parA, const uint32_t* parB,
                              unsigned long long* kpar) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint2 p = pairs[idx[i]];
  uint32_t a = parA ? parA[p.x] : p.x, b = parB ? parB[p.y] : p.y;
  kpar[i] = ((unsigned long long)a << 32) | b;
}
__global__ void k_seg_heads(const unsigned long long* __restrict__ k, uint64_t n, uint32_t* head) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = (i == 0 || k[i] != k[i - 1]) ? 1u : 0u;
}
__global__ void k_seg_starts(const uint32_t* __restrict__ head, const uint32_t* __restrict__ hoff, uint64_t n, uint32_t* start) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && head[i]) start[hoff[i]] = (uint32_t)i;
}
// one thread per parent pair: fold its piece pairs in (piece a, piece b) order: area sum, Sum4, OR, min flag
__global__ void k_fold(const unsigned long long* __restrict__ kpar, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ start, uint64_t nseg,
                       uint64_t n, const uint8_t* flag, const double* area, const double4* ev, const uint32_t* evb, uint2* opairs, double* oarea,
                       double4* oev, uint32_t* oevb, uint32_t* keep) {
  uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  uint64_t b = start[s], e = s + 1 < nseg ? start[s + 1] : n;
  double a = 0; double4 v = make_double4(0, 0, 0, 0); uint32_t bits = 0; uint8_t f = 255;
  for (uint64_t k = b; k < e; k++) {
    uint32_t i = idx[k];
    if (area) a += area[i];
    if (ev) { double4 x = ev[i]; v.x += x.x; v.y += x.y; v.z += x.z; v.w += x.w; bits |= evb[i]; }
    f = min(f, flag[i]);
  }
  unsigned long long key = kpar[b];
  opairs[s] = make_uint2((uint32_t)(key >> 32), (uint32_t)key);
  if (oarea) oarea[s] = a;
  if (oev) { oev[s] = v; oevb[s] = bits; }
  keep[s] = f == 1;
}

template <class T> static void exclusive_scan(gsj_ctx* c, const T* in, T* out, uint64_t n) {
  size_t tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int64_t)n, c->stream));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(c->tmp.get(tb), tb, in, out, (int64_t)n, c->stream));
}
static uint32_t read_last(gsj_ctx* c, const uint32_t* off, const uint32_t* flag, uint64_t n) {
  uint32_t* h = c->h_counters.as<uint32_t>(4);
  GSJ_CK(cudaMemcpyAsync(h, off + n - 1, 4, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaMemcpyAsync(h + 1, flag + n - 1, 4, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  return h[0] + h[1];
}

// Candidate search for probe rows [q0, q0 + nq) (in the given order), growing the pair buffer when needed.
uint64_t candidates_for(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper, uint2** out) {
  uint64_t cap = std::max<uint64_t>((uint64_t)nq * 16, 1 << 16);
  // reuse the whole pooled buffer: as<uint2>(cap + 1) needs (cap + 1) * 8 + 16 bytes
  const uint64_t pooled = c->cand.cap >= 64 ? (c->cand.cap - 16) / sizeof(uint2) - 1 : 0;
  if (pooled > cap) cap = pooled;
  for (;;) {
    uint2* buf = c->cand.as<uint2>(cap + 1);
    uint64_t np = traverse(c, qbb, qorder, q0, nq, T, upper, buf, cap);
    if (np <= cap) { *out = buf; return np; }
    cap = np + np / 8;
  }
}

struct Batch { uint32_t q0, nq; };
// Probe batches of one join: runs of Morton positions (layers without parents: each batch a compact region), or
// index ranges that keep a parent's pieces together. morton = the batches index P's Morton order.
static std::vector<Batch> make_batches(const gsj_layer* P, const gsj_join_opts& o, bool& morton) {
  std::vector<Batch> b;
  const uint32_t n = P->d.n;
  const auto& hp = P->h_parent;
  uint32_t lo = 0, hi = n;
  if (o.nshards > 1) {
    if (o.shard >= o.nshards) throw Error(GSJ_ERR_ARG, "shard >= nshards");
    lo = (uint32_t)((uint64_t)n * o.shard / o.nshards);
    hi = (uint32_t)((uint64_t)n * (o.shard + 1) / o.nshards);
    if (!hp.empty()) {   // a parent's pieces stay in the shard of its first piece
      while (lo > 0 && lo < n && hp[lo] == hp[lo - 1]) lo++;
      while (hi > 0 && hi < n && hp[hi] == hp[hi - 1]) hi++;
    }
  }
  const uint32_t bq = o.batch_q;
  // Morton order: the whole layer in one batch, or any batch or shard of a layer without parents
  morton = hp.empty() || (o.nshards <= 1 && (!bq || bq >= n));
  if (lo >= hi) return b;
  if (!bq || bq >= hi - lo) { b.push_back({lo, hi - lo}); return b; }
  for (uint32_t q0 = lo, qn; q0 < hi; q0 = qn) {
    qn = std::min<uint32_t>(q0 + bq, hi);
    if (!hp.empty()) while (qn < hi && hp[qn] == hp[qn - 1]) qn++;
    b.push_back({q0, qn - q0});
  }
  return b;
}

}  // namespace gsj

namespace gsj {

struct JoinOut {   // device pointers of one finished batch
  uint2* pairs; double* area; uint32_t* code; uint64_t n;
};

// Runs one join; calls on_batch(JoinOut) for every finished batch (device pointers, valid until the next batch).
// pre (optional) may drop candidate pairs in place before refinement and returns the new count.
template <class F>
void run_join(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const RefineArgs& rp, const gsj_join_opts& o, gsj_join_stats& st, F&& on_batch,
              const PrefilterFn* pre = nullptr) {
  if (P->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "polygon join needs two polygon layers");
  cudaStream_t s = c->stream;
  const bool agg = (P->d.parent || R->d.parent) && !o.no_agg;
  const bool rel = rp.want_relate != 0;
  Timer tm(s), tr(s);
  // Morton-ordered probes for coherent traversal; batches by index ranges keep a parent's pieces together
  bool whole = false;
  const std::vector<Batch> batches = make_batches(P, o, whole);
  for (const Batch& bt : batches) {
    if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
    tm.start();
    uint2* pairs = nullptr;
    uint64_t np = candidates_for(c, P->d.bb, whole ? P->bvh.order : nullptr, bt.q0, bt.nq, R->bvh, o.upper, &pairs);
    st.traverse_ms += tm.stop();
    st.candidates += np;
    st.batches++;
    if (pre && *pre && np) np = (*pre)(pairs, np);
    if (!np) continue;
    tr.start();
    uint8_t* flag = c->flag.as<uint8_t>(np);
    double* area = (rp.want_area) ? c->area.as<double>(np) : nullptr;
    double4* ev = rel ? c->ev.as<double4>(np) : nullptr;
    uint32_t* evb = rel ? c->evb.as<uint32_t>(np) : nullptr;
    // area is needed for the piece fold or the output; relate-only joins still fold (zero) areas.
    // The refinement's counters come back with the compaction's count: one host round trip for both.
    refine_enqueue(c, P, R, pairs, np, rp, o.refine_mode, flag, area, ev, evb);
    tr.mark_end();
    tm.start();
    uint32_t* keep = c->keep.as<uint32_t>(np);
    uint32_t* off = c->idx.as<uint32_t>(np);
    k_keep<<<grid_for(np, 256), 256, 0, s>>>(flag, np, agg ? 1 : 0, keep); c->launches++;
    exclusive_scan(c, keep, off, np);
    uint64_t nk = read_last(c, off, keep, np);
    st.heavy += refine_result(c);
    st.refine_ms += tr.elapsed();
    JoinOut out{nullptr, nullptr, nullptr, 0};
    if (!agg) {
      out.pairs = c->opairs.as<uint2>(nk);
      out.area = rp.want_area ? c->oarea.as<double>(nk) : nullptr;
      out.code = rel ? c->ocode.as<uint32_t>(nk) : nullptr;
      out.n = nk;
      if (nk) {
        k_scatter_rows<<<grid_for(np, 256), 256, 0, s>>>(pairs, keep, off, np, area, ev, evb, P->d.blen, R->d.blen, out.pairs, out.area, out.code);
        c->launches++;
      }
    } else if (nk) {
      // fold piece pairs into parent pairs in (parent pair, piece a, piece b) order
      unsigned long long* k1 = c->keys.as<unsigned long long>(nk);
      unsigned long long* k2 = c->keys2.as<unsigned long long>(nk);
      uint32_t* i1 = c->idx2.as<uint32_t>(nk);
      uint32_t* i2 = c->misc1.as<uint32_t>(nk);
      k_scatter_pieces<<<grid_for(np, 256), 256, 0, s>>>(pairs, keep, off, np, P->d.parent, R->d.parent, k1, i1); c->launches++;
      size_t tb = 0;
      GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, i1, i2, (int64_t)nk, 0, 64, s));
      GSJ_CK(cub::DeviceRadixSort::SortPairs(c->tmp.get(tb), tb, k1, k2, i1, i2, (int64_t)nk, 0, 64, s));
      k_parent_keys<<<grid_for(nk, 256), 256, 0, s>>>(i2, nk, pairs, P->d.parent, R->d.parent, k1); c->launches++;
      tb = 0;
      GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, i2, i1, (int64_t)nk, 0, 64, s));   // stable
      GSJ_CK(cub::DeviceRadixSort::SortPairs(c->tmp.get(tb), tb, k1, k2, i2, i1, (int64_t)nk, 0, 64, s));
      uint32_t* head = c->misc2.as<uint32_t>(nk);
      uint32_t* hoff = c->misc3.as<uint32_t>(nk);
      k_seg_heads<<<grid_for(nk, 256), 256, 0, s>>>(k2, nk, head); c->launches++;
      exclusive_scan(c, head, hoff, nk);
      uint64_t nseg = read_last(c, hoff, head, nk);
      uint32_t* start = c->keep.as<uint32_t>(std::max<uint64_t>(np, nseg));   // keep/off of the pieces are no longer needed
      k_seg_starts<<<grid_for(nk, 256), 256, 0, s>>>(head, hoff, nk, start); c->launches++;
      uint2* fp = c->agg_flag.as<uint2>(nseg);
      double* fa = c->agg_area.as<double>(nseg);
      double4* fe = rel ? c->agg_ev.as<double4>(nseg) : nullptr;
      uint32_t* fb = rel ? c->agg_evb.as<uint32_t>(nseg) : nullptr;
      uint32_t* fk = c->misc2.as<uint32_t>(nseg);
      k_fold<<<grid_for(nseg, 256), 256, 0, s>>>(k2, i1, start, nseg, nk, flag, area, ev, evb, fp, area ? fa : nullptr, fe, fb, fk); c->launches++;
      uint32_t* foff = c->misc3.as<uint32_t>(nseg);
      exclusive_scan(c, fk, foff, nseg);
      uint64_t nout = read_last(c, foff, fk, nseg);
      out.pairs = c->opairs.as<uint2>(nout);
      out.area = rp.want_area ? c->oarea.as<double>(nout) : nullptr;
      out.code = rel ? c->ocode.as<uint32_t>(nout) : nullptr;
      out.n = nout;
      if (nout) {
        k_scatter_rows<<<grid_for(nseg, 256), 256, 0, s>>>(fp, fk, foff, nseg, area ? fa : nullptr, fe, fb,
                                                           P->d.blen, R->d.blen, out.pairs, out.area, out.code);
        c->launches++;
      }
    }
    st.compact_ms += tm.stop();
    st.hits += out.n;
    on_batch(out);
  }
}

// ---- points in polygons (k_pip_pairs, engine.cuh:1079-1106) ---------------------------------------------------
__global__ void k_pip(const double2* __restrict__ pts, DLayer R, const uint2* __restrict__ pairs, uint64_t np, uint8_t* hit) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const uint2 pr = pairs[i];
  const double2 pt = pts[pr.x], o = R.origin[pr.y];
  const Frame B = frame_of(R, pr.y, o.x, o.y);
  const double px = (double)(pt.x - o.x), py = (double)(pt.y - o.y);
  const double ox = B.shx - (double)1;
  bool par = false, on = false;
  for (uint32_t r = B.r0; r < B.r1 && !on; r++) {
    const uint64_t s0 = R.rvo[r], e = R.rvo[r + 1];
    double x0, y0; B.v(s0, x0, y0);
    for (uint64_t j = s0 + 1; j < e; j++) {
      double x1, y1; B.v(j, x1, y1);
      if (!((y0 > py) == (y1 > py) && y0 != py && y1 != py)) {
        const double o_ = orient(x0, y0, x1, y1, px, py);
        if (o_ == 0 && !R.syn(j - 1) && onseg(x0, y0, x1, y1, px, py)) { on = true; break; }
        bool so = left_of(x0, y0, x1, y1, ox, py), sp = left_of(x0, y0, x1, y1, px, py);
        if (so != sp) {
          bool su = orient(ox, py, px, py, x0, y0) > 0, sv = orient(ox, py, px, py, x1, y1) > 0;
          if (su != sv) par = !par;
        }
      }
      x0 = x1; y0 = y1;
    }
  }
  hit[i] = on ? 2 : (par ? 1 : 0);
}
__global__ void k_u8_nonzero(const uint8_t* f, uint64_t n, uint32_t* keep) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keep[i] = f[i] != 0;
}
__global__ void k_scatter_pts(const uint2* __restrict__ pairs, const uint8_t* __restrict__ hit, const uint32_t* keep, const uint32_t* off,
                              uint64_t n, const uint32_t* parR, unsigned long long* key, uint8_t* val) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !keep[i]) return;
  uint2 p = pairs[i];
  uint32_t o = off[i];
  key[o] = ((unsigned long long)p.x << 32) | (parR ? parR[p.y] : p.y);
  val[o] = hit[i];
}
// sorted (point, parent) keys: max fold per key (boundary wins over interior)
__global__ void k_fold_max(const unsigned long long* __restrict__ k, const uint8_t* __restrict__ v, const uint32_t* start, uint64_t nseg, uint64_t n,
                           uint2* opairs, uint8_t* owhere) {
  uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nseg) return;
  uint64_t b = start[s], e = s + 1 < nseg ? start[s + 1] : n;
  uint8_t m = 0;
  for (uint64_t q = b; q < e; q++) m = max(m, v[q]);
  opairs[s] = make_uint2((uint32_t)(k[b] >> 32), (uint32_t)k[b]);
  owhere[s] = m;
}

template <class F>
void run_points(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, const gsj_join_opts& o, gsj_join_stats& st, F&& on_batch) {
  if (!pts->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "point join needs a point layer and a polygon layer");
  cudaStream_t s = c->stream;
  Timer tm(s);
  const uint32_t n = pts->d.n;
  uint32_t lo = 0, hi = n;   // probe shard: a run of Morton positions
  if (o.nshards > 1) {
    if (o.shard >= o.nshards) throw Error(GSJ_ERR_ARG, "shard >= nshards");
    lo = (uint32_t)((uint64_t)n * o.shard / o.nshards);
    hi = (uint32_t)((uint64_t)n * (o.shard + 1) / o.nshards);
  }
  const uint32_t span = hi - lo;
  const uint32_t bq = (o.batch_q && o.batch_q < span) ? o.batch_q : span;
  for (uint32_t q0 = lo; q0 < hi; q0 += bq) {
    if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
    const uint32_t nq = std::min(bq, hi - q0);
    tm.start();
    uint2* pairs = nullptr;
    uint64_t np = candidates_for(c, pts->d.bb, pts->bvh.order, q0, nq, R->bvh, 0, &pairs);   // runs of Morton positions
    st.traverse_ms += tm.stop(); st.candidates += np; st.batches++;
    if (!np) continue;
    tm.start();
    uint8_t* hit = c->flag.as<uint8_t>(np);
    // one thread per (point, piece) in both modes: a warp per pair measured slower (1.59 vs 1.37 ms for 2M pairs)
    k_pip<<<grid_for(np, 128), 128, 0, s>>>(pts->pts, R->d, pairs, np, hit); c->launches++;
    GSJ_CK(cudaGetLastError());
    st.refine_ms += tm.stop();
    tm.start();
    uint32_t* keep = c->keep.as<uint32_t>(np);
    uint32_t* off = c->idx.as<uint32_t>(np);
    k_u8_nonzero<<<grid_for(np, 256), 256, 0, s>>>(hit, np, keep); c->launches++;
    exclusive_scan(c, keep, off, np);
    uint64_t nk = read_last(c, off, keep, np);
    uint2* opairs = c->opairs.as<uint2>(nk);
    uint8_t* owhere = reinterpret_cast<uint8_t*>(c->ocode.as<uint32_t>(nk / 4 + 1));
    uint64_t nout = 0;
    if (nk) {
      unsigned long long* k1 = c->keys.as<unsigned long long>(nk);
      unsigned long long* k2 = c->keys2.as<unsigned long long>(nk);
      uint8_t* v1 = reinterpret_cast<uint8_t*>(c->misc1.as<uint32_t>(nk / 4 + 1));
      uint8_t* v2 = reinterpret_cast<uint8_t*>(c->misc2.as<uint32_t>(nk / 4 + 1));
      k_scatter_pts<<<grid_for(np, 256), 256, 0, s>>>(pairs, hit, keep, off, np, R->d.parent, k1, v1); c->launches++;
      size_t tb = 0;
      GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, v1, v2, (int64_t)nk, 0, 64, s));
      GSJ_CK(cub::DeviceRadixSort::SortPairs(c->tmp.get(tb), tb, k1, k2, v1, v2, (int64_t)nk, 0, 64, s));
      uint32_t* head = c->misc3.as<uint32_t>(nk);
      uint32_t* hoff = c->idx2.as<uint32_t>(nk);
      k_seg_heads<<<grid_for(nk, 256), 256, 0, s>>>(k2, nk, head); c->launches++;
      exclusive_scan(c, head, hoff, nk);
      nout = read_last(c, hoff, head, nk);
      uint32_t* start = c->keep.as<uint32_t>(std::max<uint64_t>(np, nout));
      k_seg_starts<<<grid_for(nk, 256), 256, 0, s>>>(head, hoff, nk, start); c->launches++;
      k_fold_max<<<grid_for(nout, 256), 256, 0, s>>>(k2, v2, start, nout, nk, opairs, owhere); c->launches++;
      GSJ_CK(cudaGetLastError());
    }
    st.compact_ms += tm.stop();
    st.hits += nout;
    on_batch(opairs, owhere, nout);
  }
}

// ---- ST_ClusterIntersecting: lock-free union-find on the device (engine.cuh:1180-1234) -------------------------
// parent[] through L2 (ld.cg / st.cg): L1 is not coherent with other SMs' atomics
__device__ __forceinline__ uint32_t uf_find(uint32_t* par, uint32_t x) {
  for (;;) {
    uint32_t p = __ldcg(par + x);
    if (p == x) return x;
    uint32_t gp = __ldcg(par + p);
    if (gp != p) __stcg(par + x, gp);   // path halving; a stale write still points at an ancestor
    x = p;
  }
}
__global__ void k_uf_init(uint32_t* par, uint32_t n) { uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; if (i < n) par[i] = i; }
__global__ void k_uf_union(const uint2* __restrict__ pairs, uint64_t n, uint32_t* par) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t a = pairs[i].x, b = pairs[i].y;
  if (a == b) return;
  for (;;) {
    uint32_t ra = uf_find(par, a), rb = uf_find(par, b);
    if (ra == rb) return;
    if (ra > rb) { uint32_t t = ra; ra = rb; rb = t; }
    if (atomicCAS(&par[rb], rb, ra) == rb) return;   // the larger root goes under the smaller: roots are component minima
  }
}
constexpr uint32_t CLUSTER_ROUNDS = 8;
// Cluster rounds (filtered mode): candidate i = t * R + r belongs to round r; it is refined only while its two
// parents are still in different components. A skipped pair joins two geometries that are already connected, so
// the components (and root[]) are those of the full intersects graph.
__global__ void k_cl_select(const uint2* __restrict__ pairs, uint64_t n, uint32_t r, uint32_t R, const uint32_t* __restrict__ parent,
                            uint32_t* par, uint32_t* keep) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, i = t * R + r;
  if (i >= n) return;
  const uint2 p = pairs[i];
  const uint32_t a = parent ? parent[p.x] : p.x, b = parent ? parent[p.y] : p.y;
  keep[t] = a != b && uf_find(par, a) != uf_find(par, b);
}
__global__ void k_cl_gather(const uint2* __restrict__ pairs, uint64_t n, uint32_t r, uint32_t R, const uint32_t* __restrict__ keep,
                            const uint32_t* __restrict__ off, uint2* out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x, i = t * R + r;
  if (i < n && keep[t]) out[off[t]] = pairs[i];
}
__global__ void k_cl_union(const uint2* __restrict__ pairs, const uint8_t* __restrict__ flag, uint64_t n, const uint32_t* __restrict__ parent,
                           uint32_t* par, unsigned long long* hits) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool h = i < n && flag[i];
  const unsigned m = __ballot_sync(0xffffffffu, h);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(hits, (unsigned long long)__popc(m));
  if (!h) return;
  uint32_t a = parent ? parent[pairs[i].x] : pairs[i].x, b = parent ? parent[pairs[i].y] : pairs[i].y;
  for (;;) {
    uint32_t ra = uf_find(par, a), rb = uf_find(par, b);
    if (ra == rb) return;
    if (ra > rb) { uint32_t t = ra; ra = rb; rb = t; }
    if (atomicCAS(&par[rb], rb, ra) == rb) return;
  }
}
__global__ void k_uf_flatten(uint32_t* par, uint32_t n) {   // concurrent readers see an ancestor either way
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) par[i] = uf_find(par, i);
}
// one forest of a probe shard's cluster (root[i] = smallest index of i's component there): joined into par
__global__ void k_uf_union_roots(const uint32_t* __restrict__ root, uint32_t n, uint32_t* par) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t a = i, b = root[i];
  if (a == b) return;
  for (;;) {
    uint32_t ra = uf_find(par, a), rb = uf_find(par, b);
    if (ra == rb) return;
    if (ra > rb) { uint32_t t = ra; ra = rb; rb = t; }
    if (atomicCAS(&par[rb], rb, ra) == rb) return;
  }
}
__global__ void k_uf_roots(uint32_t* par, uint32_t n, uint32_t* root) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) root[i] = uf_find(par, i);
}

}  // namespace gsj

// ---- C ABI entry points of the joins -------------------------------------------------------------------------
namespace gsj {
RefineArgs to_args(const gsj_refine_params* p) {
  gsj_refine_params d;
  gsj_refine_params_default(&d);
  if (!p) p = &d;
  return RefineArgs{p->tol_rel, p->eps_par, p->tol_abs, p->want_area, p->want_relate, p->snap_half_ulp};
}
gsj_join_opts opts_or_default(const gsj_join_opts* o) {
  gsj_join_opts d;
  gsj_join_opts_default(&d);
  return o ? *o : d;
}

void join_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const gsj_refine_params* rpp, const gsj_join_opts* op, gsj_join_sink sink, void* user,
               gsj_join_stats* stp) {
  RefineArgs rp = to_args(rpp);
  gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches, v0 = c->node_visits, e0 = c->edge_pairs;
  Timer tm(c->stream);
  run_join(c, P, R, rp, o, st, [&](const JoinOut& out) {
    if (!out.n) return;
    tm.start();
    uint32_t* hp = c->h_pairs.as<uint32_t>(2 * out.n);
    double* ha = out.area ? c->h_area.as<double>(out.n) : nullptr;
    uint32_t* hc = out.code ? c->h_code.as<uint32_t>(out.n) : nullptr;
    GSJ_CK(cudaMemcpyAsync(hp, out.pairs, out.n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (ha) GSJ_CK(cudaMemcpyAsync(ha, out.area, out.n * 8, cudaMemcpyDeviceToHost, c->stream));
    if (hc) GSJ_CK(cudaMemcpyAsync(hc, out.code, out.n * 4, cudaMemcpyDeviceToHost, c->stream));
    st.copy_ms += tm.stop();
    if (sink && sink(user, hp, ha, hc, out.n)) throw Error(GSJ_ERR_SINK, "sink stopped the join");
  });
  st.launches = c->launches - l0;
  st.node_visits = c->node_visits - v0;
  st.edge_pairs = c->edge_pairs - e0;
  if (stp) *stp = st;
}

void points_host(gsj_ctx* c, const gsj_layer* pts, const gsj_layer* R, const gsj_join_opts* op, gsj_points_sink sink, void* user, gsj_join_stats* stp) {
  gsj_join_opts o = opts_or_default(op);
  gsj_join_stats st{};
  const uint64_t l0 = c->launches, v0 = c->node_visits, e0 = c->edge_pairs;
  Timer tm(c->stream);
  run_points(c, pts, R, o, st, [&](const uint2* dp, const uint8_t* dw, uint64_t n) {
    if (!n) return;
    tm.start();
    uint32_t* hp = c->h_pairs.as<uint32_t>(2 * n);
    uint8_t* hw = reinterpret_cast<uint8_t*>(c->h_where.as<uint32_t>(n / 4 + 1));
    GSJ_CK(cudaMemcpyAsync(hp, dp, n * 8, cudaMemcpyDeviceToHost, c->stream));
    GSJ_CK(cudaMemcpyAsync(hw, dw, n, cudaMemcpyDeviceToHost, c->stream));
    st.copy_ms += tm.stop();
    if (sink && sink(user, hp, hw, n)) throw Error(GSJ_ERR_SINK, "sink stopped the join");
  });
  st.launches = c->launches - l0;
  st.node_visits = c->node_visits - v0;
  st.edge_pairs = c->edge_pairs - e0;
  if (stp) *stp = st;
}

void cluster_host(gsj_ctx* c, const gsj_layer* P, uint32_t nparent, const gsj_join_opts* op, uint32_t* root, gsj_join_stats* stp) {
  if (P->is_points) throw Error(GSJ_ERR_ARG, "cluster needs a polygon layer");
  if (nparent < P->nparent) throw Error(GSJ_ERR_ARG, "nparent is smaller than the layer's parent count");
  gsj_join_opts o = opts_or_default(op);
  o.upper = 1; o.no_agg = 0;
  RefineArgs rp = to_args(nullptr);
  rp.want_area = 0; rp.want_relate = 0;
  gsj_join_stats st{};
  const uint64_t l0 = c->launches, v0 = c->node_visits, e0 = c->edge_pairs;
  cudaStream_t s = c->stream;
  uint32_t* par = c->uf.as<uint32_t>(2 * (size_t)nparent);
  uint32_t* droot = par + nparent;
  k_uf_init<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent); c->launches++;
  if (o.refine_mode == GSJ_REFINE_PLAIN) {   // every candidate refined, as the reference does
    run_join(c, P, P, rp, o, st, [&](const JoinOut& out) {
      if (out.n) { k_uf_union<<<grid_for(out.n, 256), 256, 0, s>>>(out.pairs, out.n, par); c->launches++; }
    });
  } else {   // rounds that skip pairs whose parents are already connected
    Timer tm(s);
    bool whole = false;
    const std::vector<Batch> batches = make_batches(P, o, whole);
    unsigned long long* hits = c->misc3.as<unsigned long long>(1);
    GSJ_CK(cudaMemsetAsync(hits, 0, sizeof(unsigned long long), s));
    for (const Batch& bt : batches) {
      if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
      tm.start();
      uint2* pairs = nullptr;
      const uint64_t np = candidates_for(c, P->d.bb, whole ? P->bvh.order : nullptr, bt.q0, bt.nq, P->bvh, 1, &pairs);
      st.traverse_ms += tm.stop();
      st.candidates += np;
      st.batches++;
      if (!np) continue;
      const uint32_t R = np < (1u << 16) ? 1 : CLUSTER_ROUNDS;
      for (uint32_t r = 0; r < R; r++) {
        if (o.cancel && *o.cancel) throw Error(GSJ_ERR_CANCELLED, "cancelled");
        tm.start();
        const uint64_t nt = (np - r + R - 1) / R;   // candidates r, r + R, ... < np
        uint32_t* keep = c->keep.as<uint32_t>(nt);
        uint32_t* off = c->idx.as<uint32_t>(nt);
        k_cl_select<<<grid_for(nt, 256), 256, 0, s>>>(pairs, np, r, R, P->d.parent, par, keep); c->launches++;
        exclusive_scan(c, keep, off, nt);
        const uint64_t ns = read_last(c, off, keep, nt);
        uint2* sel = c->opairs.as<uint2>(ns);
        if (ns) { k_cl_gather<<<grid_for(nt, 256), 256, 0, s>>>(pairs, np, r, R, keep, off, sel); c->launches++; }
        st.compact_ms += tm.stop();
        if (!ns) continue;
        tm.start();
        uint8_t* flag = c->flag.as<uint8_t>(ns);
        st.heavy += refine(c, P, P, sel, ns, rp, o.refine_mode, flag, nullptr, nullptr, nullptr);
        st.refine_ms += tm.stop();
        tm.start();
        k_cl_union<<<grid_for(ns, 256), 256, 0, s>>>(sel, flag, ns, P->d.parent, par, hits); c->launches++;
        k_uf_flatten<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent); c->launches++;
        st.compact_ms += tm.stop();
      }
    }
    unsigned long long hh = 0;
    GSJ_CK(cudaMemcpyAsync(&hh, hits, sizeof(hh), cudaMemcpyDeviceToHost, s));
    GSJ_CK(cudaStreamSynchronize(s));
    st.hits = hh;
  }
  k_uf_roots<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent, droot); c->launches++;
  GSJ_CK(cudaGetLastError());
  GSJ_CK(cudaMemcpyAsync(root, droot, (size_t)nparent * 4, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  st.launches = c->launches - l0;
  st.node_visits = c->node_visits - v0;
  st.edge_pairs = c->edge_pairs - e0;
  if (stp) *stp = st;
}

// Components of the union of several forests (the clusters of the probe shards of one layer, computed by
// cluster_host with shard / nshards on several GPUs and gathered): every i joined with its root in every forest.
void cluster_merge_host(gsj_ctx* c, uint32_t nparent, uint32_t nforests, const uint32_t* roots, uint32_t* out) {
  if (!nparent) return;
  for (uint64_t k = 0; k < (uint64_t)nforests * nparent; k++)
    if (roots[k] >= nparent) throw Error(GSJ_ERR_ARG, "a root index is out of range");
  cudaStream_t s = c->stream;
  uint32_t* par = c->uf.as<uint32_t>(2 * (size_t)nparent);
  uint32_t* droot = par + nparent;
  uint32_t* din = c->misc1.as<uint32_t>(nparent);
  k_uf_init<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent); c->launches++;
  for (uint32_t f = 0; f < nforests; f++) {
    GSJ_CK(cudaMemcpyAsync(din, roots + (uint64_t)f * nparent, (size_t)nparent * 4, cudaMemcpyHostToDevice, s));
    k_uf_union_roots<<<grid_for(nparent, 256), 256, 0, s>>>(din, nparent, par); c->launches++;
    k_uf_flatten<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent); c->launches++;
  }
  k_uf_roots<<<grid_for(nparent, 256), 256, 0, s>>>(par, nparent, droot); c->launches++;
  GSJ_CK(cudaGetLastError());
  GSJ_CK(cudaMemcpyAsync(out, droot, (size_t)nparent * 4, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
}

// the intersects + area join with device-side results: pass 1 of the erosion join
void join_device(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const RefineArgs& rp, const gsj_join_opts& o, gsj_join_stats& st,
                 const PrefilterFn& pre, const DeviceBatchFn& on_batch) {
  run_join(c, P, R, rp, o, st, [&](const JoinOut& out) { if (out.n) on_batch(out.pairs, out.area, out.n); }, &pre);
}

void candidates_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, int upper, gsj_pairs_sink sink, void* user) {
  uint2* pairs = nullptr;
  uint64_t np = candidates_for(c, P->d.bb, P->bvh.order, 0, P->d.n, R->bvh, upper, &pairs);
  uint32_t* hp = c->h_pairs.as<uint32_t>(2 * np + 2);
  GSJ_CK(cudaMemcpyAsync(hp, pairs, np * 8, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  if (sink && np && sink(user, hp, np)) throw Error(GSJ_ERR_SINK, "sink stopped");
}

void refine_pairs_host(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint32_t* pairs, uint64_t np, const gsj_refine_params* rpp, int mode,
                       uint8_t* flag, double* area, double* ev, uint32_t* evb) {
  if (!np) return;
  RefineArgs rp = to_args(rpp);
  cudaStream_t s = c->stream;
  uint2* dp = c->cand.as<uint2>(np);
  for (uint64_t i = 0; i < np; i++)
    if (pairs[2 * i] >= P->d.n || pairs[2 * i + 1] >= R->d.n) throw Error(GSJ_ERR_ARG, "pair index out of range");
  GSJ_CK(cudaMemcpyAsync(dp, pairs, np * 8, cudaMemcpyHostToDevice, s));
  uint8_t* dflag = c->flag.as<uint8_t>(np);
  double* darea = c->area.as<double>(np);
  double4* dev = c->ev.as<double4>(np);
  uint32_t* devb = c->evb.as<uint32_t>(np);
  GSJ_CK(cudaMemsetAsync(darea, 0, np * 8, s));
  GSJ_CK(cudaMemsetAsync(dev, 0, np * 32, s));
  GSJ_CK(cudaMemsetAsync(devb, 0, np * 4, s));
  refine(c, P, R, dp, np, rp, mode, dflag, darea, dev, devb);
  if (flag) GSJ_CK(cudaMemcpyAsync(flag, dflag, np, cudaMemcpyDeviceToHost, s));
  if (area) GSJ_CK(cudaMemcpyAsync(area, darea, np * 8, cudaMemcpyDeviceToHost, s));
  if (ev) GSJ_CK(cudaMemcpyAsync(ev, dev, np * 32, cudaMemcpyDeviceToHost, s));
  if (evb) GSJ_CK(cudaMemcpyAsync(evb, devb, np * 4, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
}

}  // namespace gsj
