// Row encoding on the device: the gpujoind result stream (frames of rows) built from the engine's result pairs by
// the daemon's row rules, in place of the host encoder (send_parallel / FrameBuf, daemon/gpujoind.cu:178-206;
// rules gpujoind.cu:244-283, 356-367, 460-481). One thread per result pair counts its rows and bytes, scans give
// every pair its offset in one output buffer and every block of pairs a frame header, a second pass writes the rows.
#include <cub/cub.cuh>
#include <cmath>
#include <cstring>
#include "engine.h"
#include "../../include/gsp_protocol.h"

struct gsj_rowset {
  int device = 0;
  uint64_t n_geoms = 0, n_rows = 0;
  uint64_t* moff = nullptr;   // device, n_geoms + 1, or null: geometry = row
  uint32_t* midx = nullptr;
  char* blob = nullptr;
  uint64_t* off = nullptr;    // device, n_rows + 1
  uint32_t max_id = 0;        // longest id (bytes, capped at 65535)
};

namespace gsj {
namespace {

constexpr uint32_t kPtInterior = 1u | (3u << 12) | (2u << 14) | (3u << 16);          // 0FFFFF212
constexpr uint32_t kPtBoundary = (1u << 2) | (3u << 12) | (2u << 14) | (3u << 16);   // F0FFFF212

struct RowsDev {
  const uint64_t* moff; const uint32_t* midx; const char* blob; const uint64_t* off;
  __device__ uint64_t count(uint32_t g) const { return moff ? moff[g + 1] - moff[g] : 1; }
  __device__ uint32_t member(uint32_t g, uint64_t k) const { return moff ? midx[moff[g] + k] : g; }
  __device__ uint32_t len(uint32_t r) const { const uint64_t l = off[r + 1] - off[r]; return l < 65535 ? (uint32_t)l : 65535u; }
};
struct Spec { int mode, same, distinct, swapped; double value; char pat[9]; int has_pat; };

__device__ uint32_t transpose(uint32_t c) {   // gsj_de9im_transpose
  uint32_t t = 0;
  for (int r = 0; r < 3; r++)
    for (int q = 0; q < 3; q++) t |= ((c >> (2 * (3 * r + q))) & 3) << (2 * (3 * q + r));
  return t;
}
__device__ bool matches(uint32_t code, const Spec& S) {   // gsj_de9im_match (an empty pattern keeps every row)
  if (!S.has_pat) return true;
  for (int k = 0; k < 9; k++) {
    const char p = S.pat[k];
    const uint32_t v = (code >> (2 * k)) & 3;
    if (p == '*') continue;
    if (p == 'T' || p == 't') { if (v == 0) return false; continue; }
    if (p == 'F' || p == 'f') { if (v != 0) return false; continue; }
    if (p >= '0' && p <= '2') { if (v != (uint32_t)(p - '0') + 1) return false; continue; }
    return false;
  }
  return true;
}

// the rows of result pair i: out(x row, y row, code) with x's id from X and y's from Y (code only for relate modes)
template <class F>
__device__ void rows_of(uint64_t i, const Spec& S, const uint2* pairs, const uint32_t* code, const uint8_t* where, const RowsDev& P,
                        const RowsDev& Q, F&& out) {
  const uint2 p = pairs[i];
  if (S.mode == GSJ_ENC_PAIRS || S.mode == GSJ_ENC_RELATE) {   // pair_rows (rows.h)
    const uint32_t cd = S.mode == GSJ_ENC_RELATE ? code[i] : 0u, ct = S.mode == GSJ_ENC_RELATE ? transpose(cd) : 0u;
    const bool diag = S.same && p.x == p.y;
    const uint64_t na = P.count(p.x), nb = Q.count(p.y);
    for (uint64_t u = 0; u < na; u++) {
      const uint32_t ra = P.member(p.x, u);
      for (uint64_t v = 0; v < nb; v++) {
        const uint32_t rb = Q.member(p.y, v);
        if (!S.same) { out(ra, rb, cd); continue; }
        if (S.distinct) {
          if (ra == rb || (diag && ra > rb)) continue;
          if (ra < rb) out(ra, rb, cd); else out(rb, ra, diag ? cd : ct);
          continue;
        }
        out(ra, rb, cd);
        if (!diag) out(rb, ra, ct);
      }
    }
    return;
  }
  // (point, polygon): one row per member of the polygon
  const uint32_t pc = S.mode == GSJ_ENC_POINT_RELATE ? (where[i] == 2 ? kPtBoundary : kPtInterior) : 0u;
  const uint64_t nb = Q.count(p.y);
  for (uint64_t v = 0; v < nb; v++) {
    const uint32_t rb = Q.member(p.y, v);
    if (S.swapped) out(rb, p.x, S.mode == GSJ_ENC_POINT_RELATE ? transpose(pc) : 0u);
    else out(p.x, rb, pc);
  }
}
__host__ __device__ __forceinline__ bool relate_mode(const Spec& S) { return S.mode == GSJ_ENC_RELATE || S.mode == GSJ_ENC_POINT_RELATE; }

// x ids come from P, y ids from Q, except that a swapped points row has the polygon (Q) first
__device__ __forceinline__ const RowsDev& xset(const Spec& S, const RowsDev& P, const RowsDev& Q) {
  return (S.swapped && (S.mode == GSJ_ENC_POINTS || S.mode == GSJ_ENC_POINT_RELATE)) ? Q : P;
}
__device__ __forceinline__ const RowsDev& yset(const Spec& S, const RowsDev& P, const RowsDev& Q) {
  return (S.swapped && (S.mode == GSJ_ENC_POINTS || S.mode == GSJ_ENC_POINT_RELATE)) ? P : Q;
}

}  // namespace

__global__ void k_enc_count(Spec S, const uint2* __restrict__ pairs, const uint32_t* __restrict__ code, const uint8_t* __restrict__ where,
                            uint64_t n, RowsDev P, RowsDev Q, unsigned long long* rows, unsigned long long* bytes) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i > n) return;
  unsigned long long r = 0, b = 0;
  if (i < n) {
    const RowsDev& X = xset(S, P, Q);
    const RowsDev& Y = yset(S, P, Q);
    const int pl = relate_mode(S) ? 9 : 8;
    rows_of(i, S, pairs, code, where, P, Q, [&](uint32_t xr, uint32_t yr, uint32_t cd) {
      if (relate_mode(S) && !matches(cd, S)) return;
      r++;
      b += 4 + X.len(xr) + Y.len(yr) + pl;
    });
  }
  rows[i] = r; bytes[i] = b;   // entry n: 0, so the exclusive scans end with the totals
}
// frame headers: block k of K pairs gets one when it has rows (an empty frame would end the stream)
__global__ void k_enc_blocks(const unsigned long long* __restrict__ rpre, uint64_t n, uint64_t K, uint64_t nb, unsigned long long* hdr) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nb) return;
  if (k == nb) { hdr[k] = 0; return; }
  const uint64_t a = k * K, e = a + K < n ? a + K : n;
  hdr[k] = rpre[e] > rpre[a] ? 4ull : 0ull;
}
__global__ void k_enc_headers(const unsigned long long* __restrict__ rpre, const unsigned long long* __restrict__ bpre,
                              const unsigned long long* __restrict__ hpre, uint64_t n, uint64_t K, uint64_t nb, uint8_t* out) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nb) return;
  const uint64_t a = k * K, e = a + K < n ? a + K : n;
  const unsigned long long nr = rpre[e] - rpre[a];
  if (!nr) return;
  const uint32_t v = (uint32_t)nr;
  uint8_t* d = out + bpre[a] + hpre[k];
  d[0] = (uint8_t)v; d[1] = (uint8_t)(v >> 8); d[2] = (uint8_t)(v >> 16); d[3] = (uint8_t)(v >> 24);
}
__device__ __forceinline__ void put_bytes(uint8_t*& d, const void* src, uint32_t n) {
  const uint8_t* s = static_cast<const uint8_t*>(src);
  for (uint32_t k = 0; k < n; k++) d[k] = s[k];
  d += n;
}
__global__ void k_enc_write(Spec S, const uint2* __restrict__ pairs, const double* __restrict__ area, const uint32_t* __restrict__ code,
                            const uint8_t* __restrict__ where, uint64_t n, RowsDev P, RowsDev Q, const unsigned long long* __restrict__ bpre,
                            const unsigned long long* __restrict__ hpre, const unsigned long long* __restrict__ hdr, uint64_t K, uint8_t* out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = i / K;
  uint8_t* d = out + bpre[i] + hpre[k] + hdr[k];
  const RowsDev& X = xset(S, P, Q);
  const RowsDev& Y = yset(S, P, Q);
  const double val = S.mode == GSJ_ENC_PAIRS ? (area ? area[i] : (double)NAN) : S.value;
  rows_of(i, S, pairs, code, where, P, Q, [&](uint32_t xr, uint32_t yr, uint32_t cd) {
    if (relate_mode(S) && !matches(cd, S)) return;
    const uint16_t lx = (uint16_t)X.len(xr), ly = (uint16_t)Y.len(yr);
    put_bytes(d, &lx, 2); put_bytes(d, X.blob + X.off[xr], lx);
    put_bytes(d, &ly, 2); put_bytes(d, Y.blob + Y.off[yr], ly);
    if (relate_mode(S)) {
      char m[9];
      for (int q = 0; q < 9; q++) m[q] = "F012"[(cd >> (2 * q)) & 3];
      put_bytes(d, m, 9);
    } else {
      put_bytes(d, &val, 8);
    }
  });
}

namespace {

RowsDev dev_of(const gsj_rowset* r) { return RowsDev{r->moff, r->midx, r->blob, r->off}; }

template <class T> void exscan(gsj_ctx* c, const T* in, T* out, uint64_t n) {
  size_t tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int64_t)n, c->stream));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(c->tmp.get(tb), tb, in, out, (int64_t)n, c->stream));
}

}  // namespace

uint64_t encode_rows(gsj_ctx* c, const gsj_rowset* P, const gsj_rowset* Q, const gsj_encode_spec* spec, const uint32_t* pairs, const double* area,
                     const uint32_t* code, const uint8_t* where, uint64_t n, gsj_bytes_sink sink, void* user) {
  if (!n) return 0;
  Spec S{spec->mode, spec->same, spec->distinct, spec->swapped, spec->point_value, {0}, 0};
  const size_t pl = strnlen(spec->pattern, sizeof spec->pattern);
  if (pl && pl != 9) throw Error(GSJ_ERR_ARG, "pattern must have 9 characters");
  if (pl) { memcpy(S.pat, spec->pattern, 9); S.has_pat = 1; }
  if (S.mode < GSJ_ENC_PAIRS || S.mode > GSJ_ENC_POINT_RELATE) throw Error(GSJ_ERR_ARG, "unknown encode mode");
  const bool rel = relate_mode(S), pts = S.mode >= GSJ_ENC_POINTS;
  if ((S.mode == GSJ_ENC_RELATE && !code) || (S.mode == GSJ_ENC_POINT_RELATE && !where)) throw Error(GSJ_ERR_ARG, "missing relate input");
  for (uint64_t i = 0; i < n; i++)   // indices checked on the host: the kernels trust them
    if ((pts ? pairs[2 * i] >= P->n_rows : pairs[2 * i] >= P->n_geoms) || pairs[2 * i + 1] >= Q->n_geoms)
      throw Error(GSJ_ERR_ARG, "pair index out of range of its rowset");
  cudaStream_t s = c->stream;
  // inputs: pairs, then the payload array of the mode
  const size_t pb = n * 8, vb = S.mode == GSJ_ENC_PAIRS && area ? n * 8 : (S.mode == GSJ_ENC_RELATE ? n * 4 : (S.mode == GSJ_ENC_POINT_RELATE ? n : 0));
  uint8_t* din = c->enc_in.as<uint8_t>(pb + vb + 16);
  GSJ_CK(cudaMemcpyAsync(din, pairs, pb, cudaMemcpyHostToDevice, s));
  const uint2* dp = reinterpret_cast<const uint2*>(din);
  const double* da = nullptr; const uint32_t* dc = nullptr; const uint8_t* dw = nullptr;
  if (vb) {
    const void* src = S.mode == GSJ_ENC_PAIRS ? (const void*)area : (S.mode == GSJ_ENC_RELATE ? (const void*)code : (const void*)where);
    GSJ_CK(cudaMemcpyAsync(din + pb, src, vb, cudaMemcpyHostToDevice, s));
    if (S.mode == GSJ_ENC_PAIRS) da = reinterpret_cast<const double*>(din + pb);
    else if (S.mode == GSJ_ENC_RELATE) dc = reinterpret_cast<const uint32_t*>(din + pb);
    else dw = din + pb;
  }
  const RowsDev RP = dev_of(P), RQ = dev_of(Q);
  unsigned long long* cnt = c->enc_cnt.as<unsigned long long>(2 * (n + 1));
  unsigned long long* pre = c->enc_pre.as<unsigned long long>(2 * (n + 1));
  k_enc_count<<<grid_for(n + 1, 256), 256, 0, s>>>(S, dp, dc, dw, n, RP, RQ, cnt, cnt + n + 1); c->launches++;
  exscan(c, cnt, pre, n + 1);                   // rows
  exscan(c, cnt + n + 1, pre + n + 1, n + 1);   // bytes
  const uint64_t row_max = 4ull + P->max_id + Q->max_id + (rel ? 9 : 8);
  const uint64_t K = std::max<uint64_t>(1, (uint64_t)GSP_FRAME_BYTES / (2 * row_max));   // pairs per frame
  const uint64_t nb = (n + K - 1) / K;
  unsigned long long* blk = c->enc_blk.as<unsigned long long>(2 * (nb + 1));
  k_enc_blocks<<<grid_for(nb + 1, 256), 256, 0, s>>>(pre, n, K, nb, blk); c->launches++;
  exscan(c, blk, blk + nb + 1, nb + 1);
  unsigned long long* h = c->h_counters.as<unsigned long long>(4);
  GSJ_CK(cudaMemcpyAsync(h, pre + n, 8, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(h + 1, pre + n + 1 + n, 8, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(h + 2, blk + nb + 1 + nb, 8, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  const uint64_t nrows = h[0], total = h[1] + h[2];
  if (!nrows) return 0;
  uint8_t* out = c->enc_out.as<uint8_t>(total);
  k_enc_headers<<<grid_for(nb, 256), 256, 0, s>>>(pre, pre + n + 1, blk + nb + 1, n, K, nb, out); c->launches++;
  k_enc_write<<<grid_for(n, 128), 128, 0, s>>>(S, dp, da, dc, dw, n, RP, RQ, pre + n + 1, blk + nb + 1, blk, K, out); c->launches++;
  GSJ_CK(cudaGetLastError());
  uint8_t* ho = c->h_enc.as<uint8_t>(total);
  GSJ_CK(cudaMemcpyAsync(ho, out, total, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  if (sink && sink(user, ho, total, nrows)) throw Error(GSJ_ERR_SINK, "sink stopped the stream");
  return nrows;
}

gsj_rowset* rowset_upload(gsj_ctx* c, uint64_t n_geoms, const uint64_t* moff, const uint32_t* midx, uint64_t n_rows, const char* blob,
                          const uint64_t* off) {
  auto* r = new gsj_rowset;
  r->device = c->device; r->n_geoms = n_geoms; r->n_rows = n_rows;
  try {
    if (moff) {
      if (moff[0] != 0 || moff[n_geoms] > (uint64_t)UINT32_MAX) throw Error(GSJ_ERR_ARG, "bad member offsets");
      for (uint64_t k = 0; k < moff[n_geoms]; k++) if (midx[k] >= n_rows) throw Error(GSJ_ERR_ARG, "member index out of range");
      GSJ_CK(cudaMalloc(&r->moff, (n_geoms + 1) * 8));
      GSJ_CK(cudaMalloc(&r->midx, std::max<uint64_t>(moff[n_geoms], 1) * 4));
      GSJ_CK(cudaMemcpy(r->moff, moff, (n_geoms + 1) * 8, cudaMemcpyHostToDevice));
      if (moff[n_geoms]) GSJ_CK(cudaMemcpy(r->midx, midx, moff[n_geoms] * 4, cudaMemcpyHostToDevice));
    } else if (n_geoms != n_rows) {
      throw Error(GSJ_ERR_ARG, "without members, geometries and rows are the same");
    }
    if (off[0] != 0) throw Error(GSJ_ERR_ARG, "id offsets must start at 0");
    uint64_t mx = 0;
    for (uint64_t k = 0; k < n_rows; k++) {
      if (off[k + 1] < off[k]) throw Error(GSJ_ERR_ARG, "id offsets must not decrease");
      mx = std::max<uint64_t>(mx, off[k + 1] - off[k]);
    }
    r->max_id = (uint32_t)std::min<uint64_t>(mx, 65535);
    GSJ_CK(cudaMalloc(&r->off, (n_rows + 1) * 8));
    GSJ_CK(cudaMalloc(&r->blob, std::max<uint64_t>(off[n_rows], 1)));
    GSJ_CK(cudaMemcpy(r->off, off, (n_rows + 1) * 8, cudaMemcpyHostToDevice));
    if (off[n_rows]) GSJ_CK(cudaMemcpy(r->blob, blob, off[n_rows], cudaMemcpyHostToDevice));
  } catch (...) {
    rowset_free(r);
    throw;
  }
  return r;
}
void rowset_free(gsj_rowset* r) {
  if (!r) return;
  cudaSetDevice(r->device);
  for (void* p : {(void*)r->moff, (void*)r->midx, (void*)r->blob, (void*)r->off}) if (p) cudaFree(p);
  delete r;
}

}  // namespace gsj
