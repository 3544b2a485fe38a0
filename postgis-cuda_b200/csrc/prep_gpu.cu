// Exact deduplication of identical geometries on the GPU: the outputs of gsj_dedup (restating engine/dedup.h:51-124
// of landstats-us/postgis-cuda) computed on the device.
//
// A geometry's representative is the lowest-index geometry bitwise identical to it (ring count, ring sizes, vertex
// words). Identical geometries hash alike, so each equality class lies inside one run of equal hashes; a geometry
// compares itself with the earlier members of its run (ids increase along a run after a stable sort) and takes the
// first identical one, which is the class minimum. The result therefore does not depend on the hash function:
// distinct geometries in order of first occurrence (or in Z-order of their bbox centres), members of each in
// increasing input order - the same arrays as the host routine, bit for bit.
#include <cub/cub.cuh>

#include "engine.h"

namespace gsj {

struct MaxU32 {
  __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {   // splitmix64 finaliser
  x ^= x >> 30; x *= 0xBF58476D1CE4E5B9ull;
  x ^= x >> 27; x *= 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// warp per geometry: sum over rings and vertices of position-salted mixes (order-sensitive, warp-parallel)
__global__ void k_geom_hash(const uint64_t* __restrict__ gro, const uint64_t* __restrict__ rvo, const double2* __restrict__ xy, uint32_t n,
                            unsigned long long* h, uint32_t* ids) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t g = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < n; g += nw) {
    const uint64_t r0 = gro[g], r1 = gro[g + 1], v0 = rvo[r0], v1 = rvo[r1];
    uint64_t acc = 0;
    for (uint64_t r = r0 + lane; r < r1; r += 32) acc += mix64((rvo[r + 1] - rvo[r]) + ((r - r0 + 1) << 40));
    for (uint64_t v = v0 + lane; v < v1; v += 32) {
      const double2 p = xy[v];
      const uint64_t bx = (uint64_t)__double_as_longlong(p.x), by = (uint64_t)__double_as_longlong(p.y);
      acc += mix64(bx ^ mix64(by + 0x9E3779B97F4A7C15ull * (v - v0 + 1)));
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) { h[g] = mix64(acc ^ (r1 - r0)); ids[g] = (uint32_t)g; }
  }
}

__device__ bool same_geom_warp(const uint64_t* gro, const uint64_t* rvo, const double2* xy, uint32_t a, uint32_t b, int lane) {
  const uint64_t na = gro[a + 1] - gro[a];
  if (na != gro[b + 1] - gro[b]) return false;
  bool diff = false;
  for (uint64_t k = lane; k < na; k += 32)
    if (rvo[gro[a] + k + 1] - rvo[gro[a] + k] != rvo[gro[b] + k + 1] - rvo[gro[b] + k]) diff = true;
  if (__any_sync(0xffffffffu, diff)) return false;
  const uint64_t va = rvo[gro[a]], vb = rvo[gro[b]], nv = rvo[gro[a + 1]] - va;
  for (uint64_t i = lane; i < nv && !diff; i += 32) {
    const double2 p = xy[va + i], q = xy[vb + i];
    diff = __double_as_longlong(p.x) != __double_as_longlong(q.x) || __double_as_longlong(p.y) != __double_as_longlong(q.y);
  }
  return !__any_sync(0xffffffffu, diff);
}

// run starts along the hash-sorted order: rs[p] = p at a run head, else 0 (a max-scan spreads the heads)
__global__ void k_run_heads(const unsigned long long* __restrict__ hs, uint32_t n, uint32_t* rs) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) rs[p] = (p == 0 || hs[p] != hs[p - 1]) ? p : 0;
}
// warp per sorted position: the representative is the first identical earlier member of the run
__global__ void k_reps(const uint64_t* gro, const uint64_t* rvo, const double2* xy, const uint32_t* __restrict__ ids, const uint32_t* __restrict__ rs,
                       uint32_t n, uint32_t* rep) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < n; p += nw) {
    const uint32_t g = ids[p];
    uint32_t r = g;
    for (uint64_t q = rs[p]; q < p; q++)
      if (same_geom_warp(gro, rvo, xy, ids[q], g, lane)) { r = ids[q]; break; }
    if (lane == 0) rep[g] = r;
  }
}
__global__ void k_rep_flags(const uint32_t* __restrict__ rep, uint32_t n, uint32_t* flag) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) flag[g] = rep[g] == g;
}
__global__ void k_first(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ uid, uint32_t n, uint32_t* first) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n && flag[g]) first[uid[g]] = g;
}
// bbox centre of each distinct geometry (Z-order variant, dedup.h:81-96)
__global__ void k_centres(const uint64_t* gro, const uint64_t* rvo, const double2* xy, const uint32_t* __restrict__ first, uint32_t un, double* cx,
                          double* cy) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < un; i += nw) {
    const uint32_t g = first[i];
    double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
    for (uint64_t v = rvo[gro[g]] + lane; v < rvo[gro[g + 1]]; v += 32) {
      const double2 p = xy[v];
      x0 = fmin(x0, p.x); x1 = fmax(x1, p.x); y0 = fmin(y0, p.y); y1 = fmax(y1, p.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
      x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o)); x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
      y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o)); y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) { cx[i] = 0.5 * (x0 + x1); cy[i] = 0.5 * (y0 + y1); }
  }
}
__device__ __forceinline__ uint64_t spread32(uint64_t v) {
  v &= 0xFFFFFFFFull;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull; v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full; v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}
__global__ void k_zkeys(const double* __restrict__ cx, const double* __restrict__ cy, uint32_t un, const double* __restrict__ mm, unsigned long long* key) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= un) return;
  const double mx0 = mm[0], mx1 = mm[1], my0 = mm[2], my1 = mm[3];
  const double sx = mx1 > mx0 ? 4294967295.0 / (mx1 - mx0) : 0, sy = my1 > my0 ? 4294967295.0 / (my1 - my0) : 0;
  key[i] = (spread32((uint64_t)((cx[i] - mx0) * sx)) << 1) | spread32((uint64_t)((cy[i] - my0) * sy));
}
__global__ void k_uid_of_first(const uint32_t* __restrict__ first, uint32_t un, uint32_t* uid) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < un) uid[first[i]] = i;
}
__global__ void k_member_keys(const uint32_t* __restrict__ rep, const uint32_t* __restrict__ uid, uint32_t n, uint32_t* key, uint32_t* val,
                              unsigned long long* cnt) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t u = uid[rep[g]];
  key[g] = u; val[g] = g;
  atomicAdd(&cnt[u], 1ull);
}
__global__ void k_sizes(const uint64_t* __restrict__ gro, const uint64_t* __restrict__ rvo, const uint32_t* __restrict__ first, uint32_t un,
                        unsigned long long* nr, unsigned long long* nv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > un) return;
  if (i == un) { nr[i] = 0; nv[i] = 0; return; }
  const uint32_t g = first[i];
  nr[i] = gro[g + 1] - gro[g];
  nv[i] = rvo[gro[g + 1]] - rvo[gro[g]];
}
// warp per distinct geometry: its ring offsets and vertices in the distinct arrays
__global__ void k_gather(const uint64_t* gro, const uint64_t* rvo, const double2* xy, const uint32_t* __restrict__ first,
                         const unsigned long long* __restrict__ og, const unsigned long long* __restrict__ ov, uint32_t un, uint64_t* orv, double2* oxy) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < un; i += nw) {
    const uint32_t g = first[i];
    const uint64_t r0 = gro[g], r1 = gro[g + 1], vb = rvo[r0], ve = rvo[r1];
    for (uint64_t r = r0 + lane; r < r1; r += 32) orv[og[i] + (r - r0)] = ov[i] + (rvo[r] - vb);
    for (uint64_t v = vb + lane; v < ve; v += 32) oxy[ov[i] + (v - vb)] = xy[v];
  }
}

void dedup_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int morton,
               uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint64_t** out_moff,
               uint32_t** out_midx) {
  if (!gro || !rvo || !xy || !out_n || !out_gro || !out_rvo || !out_xy || !out_moff || !out_midx) throw Error(GSJ_ERR_ARG, "NULL argument");
  if (n == 0 || n >= (1ull << 31) || gro[0] != 0 || gro[n] != nr || rvo[0] != 0 || rvo[nr] != nv) throw Error(GSJ_ERR_ARG, "inconsistent offsets");
  cudaStream_t s = c->stream;
  const uint32_t N = (uint32_t)n;
  DevBuf bgro, brvo, bxy, bh, bh2, bid, bid2, brs, brep, bflag, buid, bfirst, bcx, bcy, bmm, bkey, bkey2, bf2, bk32, bv32, bk32b, bmidx, bcnt, bmoff,
      bnr, bnv, bog, bov, borv, boxy, btmp;
  for (DevBuf* b : {&bgro, &brvo, &bxy, &bh, &bh2, &bid, &bid2, &brs, &brep, &bflag, &buid, &bfirst, &bcx, &bcy, &bmm, &bkey, &bkey2, &bf2, &bk32,
                    &bv32, &bk32b, &bmidx, &bcnt, &bmoff, &bnr, &bnv, &bog, &bov, &borv, &boxy, &btmp})
    b->s = s;
  uint64_t* dgro = bgro.as<uint64_t>(n + 1);
  uint64_t* drvo = brvo.as<uint64_t>(nr + 1);
  double2* dxy = bxy.as<double2>(nv + 1);
  GSJ_CK(cudaMemcpyAsync(dgro, gro, 8 * (n + 1), cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(drvo, rvo, 8 * (nr + 1), cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(dxy, xy, 16 * nv, cudaMemcpyHostToDevice, s));
  const int wgrid = (int)std::min<uint64_t>((n * 32 + 255) / 256, (uint64_t)c->sm_count * 64);
  unsigned long long* h = bh.as<unsigned long long>(n);
  unsigned long long* hs = bh2.as<unsigned long long>(n);
  uint32_t* ids = bid.as<uint32_t>(n);
  uint32_t* ids_s = bid2.as<uint32_t>(n);
  k_geom_hash<<<wgrid, 256, 0, s>>>(dgro, drvo, dxy, N, h, ids); c->launches++;
  size_t tb = 0;
  GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, h, hs, ids, ids_s, (int64_t)n, 0, 64, s));
  GSJ_CK(cub::DeviceRadixSort::SortPairs(btmp.get(tb), tb, h, hs, ids, ids_s, (int64_t)n, 0, 64, s));
  uint32_t* rs = brs.as<uint32_t>(n);
  k_run_heads<<<grid_for(n, 256), 256, 0, s>>>(hs, N, rs); c->launches++;
  tb = 0;
  GSJ_CK(cub::DeviceScan::InclusiveScan(nullptr, tb, rs, rs, MaxU32(), (int64_t)n, s));
  GSJ_CK(cub::DeviceScan::InclusiveScan(btmp.get(tb), tb, rs, rs, MaxU32(), (int64_t)n, s));
  uint32_t* rep = brep.as<uint32_t>(n);
  k_reps<<<wgrid, 256, 0, s>>>(dgro, drvo, dxy, ids_s, rs, N, rep); c->launches++;
  uint32_t* flag = bflag.as<uint32_t>(n + 1);
  uint32_t* uid = buid.as<uint32_t>(n + 1);
  k_rep_flags<<<grid_for(n, 256), 256, 0, s>>>(rep, N, flag); c->launches++;
  GSJ_CK(cudaMemsetAsync(flag + n, 0, 4, s));
  tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, uid, (int64_t)n + 1, s));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(btmp.get(tb), tb, flag, uid, (int64_t)n + 1, s));
  uint32_t hun = 0;
  GSJ_CK(cudaMemcpyAsync(&hun, uid + n, 4, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  const uint32_t un = hun;
  uint32_t* first = bfirst.as<uint32_t>(un);
  k_first<<<grid_for(n, 256), 256, 0, s>>>(flag, uid, N, first); c->launches++;
  if (morton && un > 1) {
    double* cx = bcx.as<double>(un);
    double* cy = bcy.as<double>(un);
    const int ugrid = (int)std::min<uint64_t>(((uint64_t)un * 32 + 255) / 256, (uint64_t)c->sm_count * 64);
    k_centres<<<ugrid, 256, 0, s>>>(dgro, drvo, dxy, first, un, cx, cy); c->launches++;
    double* mm = bmm.as<double>(4);
    tb = 0;
    GSJ_CK(cub::DeviceReduce::Min(nullptr, tb, cx, mm, (int64_t)un, s));
    size_t tb2 = tb;
    GSJ_CK(cub::DeviceReduce::Max(nullptr, tb2, cx, mm + 1, (int64_t)un, s));
    void* tmp = btmp.get(std::max(tb, tb2));
    tb = std::max(tb, tb2);
    GSJ_CK(cub::DeviceReduce::Min(tmp, tb, cx, mm, (int64_t)un, s));
    GSJ_CK(cub::DeviceReduce::Max(tmp, tb, cx, mm + 1, (int64_t)un, s));
    GSJ_CK(cub::DeviceReduce::Min(tmp, tb, cy, mm + 2, (int64_t)un, s));
    GSJ_CK(cub::DeviceReduce::Max(tmp, tb, cy, mm + 3, (int64_t)un, s));
    unsigned long long* key = bkey.as<unsigned long long>(un);
    unsigned long long* key2 = bkey2.as<unsigned long long>(un);
    uint32_t* first2 = bf2.as<uint32_t>(un);
    k_zkeys<<<grid_for(un, 256), 256, 0, s>>>(cx, cy, un, mm, key); c->launches++;
    tb = 0;
    GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, first, first2, (int64_t)un, 0, 64, s));
    GSJ_CK(cub::DeviceRadixSort::SortPairs(btmp.get(tb), tb, key, key2, first, first2, (int64_t)un, 0, 64, s));
    GSJ_CK(cudaMemcpyAsync(first, first2, 4 * (size_t)un, cudaMemcpyDeviceToDevice, s));
    k_uid_of_first<<<grid_for(un, 256), 256, 0, s>>>(first, un, uid); c->launches++;
  }
  // members: (uid of the representative, g) sorted stably by uid; counts -> offsets
  uint32_t* k32 = bk32.as<uint32_t>(n);
  uint32_t* v32 = bv32.as<uint32_t>(n);
  uint32_t* k32b = bk32b.as<uint32_t>(n);
  uint32_t* midx = bmidx.as<uint32_t>(n);
  unsigned long long* cnt = bcnt.as<unsigned long long>((size_t)un + 1);
  unsigned long long* moff = bmoff.as<unsigned long long>((size_t)un + 1);
  GSJ_CK(cudaMemsetAsync(cnt, 0, 8 * ((size_t)un + 1), s));
  k_member_keys<<<grid_for(n, 256), 256, 0, s>>>(rep, uid, N, k32, v32, cnt); c->launches++;
  tb = 0;
  GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k32, k32b, v32, midx, (int64_t)n, 0, 32, s));
  GSJ_CK(cub::DeviceRadixSort::SortPairs(btmp.get(tb), tb, k32, k32b, v32, midx, (int64_t)n, 0, 32, s));
  tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, moff, (int64_t)un + 1, s));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(btmp.get(tb), tb, cnt, moff, (int64_t)un + 1, s));
  // distinct geometry arrays
  unsigned long long* dnr = bnr.as<unsigned long long>((size_t)un + 1);
  unsigned long long* dnv = bnv.as<unsigned long long>((size_t)un + 1);
  unsigned long long* og = bog.as<unsigned long long>((size_t)un + 1);
  unsigned long long* ov = bov.as<unsigned long long>((size_t)un + 1);
  k_sizes<<<grid_for((uint64_t)un + 1, 256), 256, 0, s>>>(dgro, drvo, first, un, dnr, dnv); c->launches++;
  tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, dnr, og, (int64_t)un + 1, s));
  void* tmp = btmp.get(tb);
  GSJ_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, dnr, og, (int64_t)un + 1, s));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, dnv, ov, (int64_t)un + 1, s));
  unsigned long long tot[2];
  GSJ_CK(cudaMemcpyAsync(&tot[0], og + un, 8, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(&tot[1], ov + un, 8, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  const uint64_t onr = tot[0], onv = tot[1];
  uint64_t* orv = borv.as<uint64_t>(onr + 1);
  double2* oxy = boxy.as<double2>(onv + 1);
  const int ugrid = (int)std::min<uint64_t>(((uint64_t)un * 32 + 255) / 256, (uint64_t)c->sm_count * 64);
  k_gather<<<ugrid, 256, 0, s>>>(dgro, drvo, dxy, first, og, ov, un, orv, oxy); c->launches++;
  GSJ_CK(cudaMemcpyAsync(orv + onr, &tot[1], 8, cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaGetLastError());
  // results to library-allocated host arrays (freed with gsj_host_free)
  uint64_t* hgro = (uint64_t*)malloc(8 * ((size_t)un + 1));
  uint64_t* hrvo = (uint64_t*)malloc(8 * (onr + 1));
  double* hxy = (double*)malloc(16 * (onv ? onv : 1));
  uint64_t* hmoff = (uint64_t*)malloc(8 * ((size_t)un + 1));
  uint32_t* hmidx = (uint32_t*)malloc(4 * n);
  if (!hgro || !hrvo || !hxy || !hmoff || !hmidx) {
    free(hgro); free(hrvo); free(hxy); free(hmoff); free(hmidx);
    throw Error(GSJ_ERR_NOMEM, "host allocation failed");
  }
  GSJ_CK(cudaMemcpyAsync(hgro, og, 8 * ((size_t)un + 1), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hrvo, orv, 8 * (onr + 1), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hxy, oxy, 16 * onv, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hmoff, moff, 8 * ((size_t)un + 1), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hmidx, midx, 4 * n, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  *out_n = un;
  if (out_nr) *out_nr = onr;
  if (out_nv) *out_nv = onv;
  *out_gro = hgro; *out_rvo = hrvo; *out_xy = hxy; *out_moff = hmoff; *out_midx = hmidx;
}

}  // namespace gsj
