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

#include <vector>

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


// ---- subdivision on the GPU: the outputs of gsj_subdivide (engine/subdivide.h:16-129 of the reference) ---------------
// Breadth-first rounds instead of the host's recursion: each round, a warp per piece takes its vertex count and bbox
// and decides leaf or split (the longer side halved); split pieces clip every ring against both half-planes (thread
// per ring and side; the same FP64 steps as the host's Sutherland-Hodgman clip, run once to count and once to write).
// A leaf carries (geometry << 24 | cut path, MSB = first cut, 0 = low side): sorting the keys gives the host's
// depth-first order, so the arrays come out the same, bit for bit.
namespace {

constexpr int SUB_MAX_DEPTH = 24;

struct ClipOut {   // one clipped ring: count and (write pass) the points
  double2* xy = nullptr;
  uint8_t* syn = nullptr;
};

// Sutherland-Hodgman clip of closed ring (src, n points) against coord[axis] <= m (le) or >= m; returns the kept
// point count, 0 when the ring is dropped (fewer than 4 points or zero shoelace area, summed while the points are
// appended, in the host's order). With out.xy set, also writes the points and their cut flags.
__device__ uint32_t clip_ring_dev(const double2* src, const uint8_t* ssyn, uint32_t n, int axis, double m, bool le, ClipOut out) {
  uint32_t k = 0;
  double lx = 0, ly = 0, fx = 0, fy = 0, area = 0;
  auto push = [&](double x, double y, uint8_t f) {
    if (k >= 1 && lx == x && ly == y) { if (out.syn) out.syn[k - 1] = f; return; }   // repeated point: keep one
    if (k == 0) { fx = x; fy = y; }
    else area += lx * y - x * ly;
    if (out.xy) { out.xy[k] = make_double2(x, y); out.syn[k] = f; }
    lx = x; ly = y; k++;
  };
  auto inside = [&](const double2& p) { const double v = axis == 0 ? p.x : p.y; return le ? v <= m : v >= m; };
  for (uint32_t i = 0; i + 1 < n; i++) {
    const double2 p = src[i], q = src[i + 1];
    const bool pin = inside(p), qin = inside(q);
    const uint8_t f = ssyn ? ssyn[i] : 0;
    double ix = 0, iy = 0;
    if (pin != qin) {
      if (axis == 0) { ix = m; iy = p.y + (m - p.x) * (q.y - p.y) / (q.x - p.x); }
      else { iy = m; ix = p.x + (m - p.y) * (q.x - p.x) / (q.y - p.y); }
    }
    if (pin) push(p.x, p.y, f);
    if (pin && !qin) push(ix, iy, 1);       // leaving: the next edge runs along the cut
    else if (!pin && qin) push(ix, iy, f);  // entering
  }
  if (k < 3) return 0;
  if (fx != lx || fy != ly) {   // close the ring
    area += lx * fy - fx * ly;
    if (out.xy) { out.xy[k] = make_double2(fx, fy); out.syn[k] = 0; }
    k++;
  } else if (out.syn) {
    out.syn[k - 1] = 0;
  }
  if (k < 4 || area == 0.0) return 0;   // degenerate slivers are dropped
  return k;
}

}  // namespace

namespace {

struct Pieces {   // one round's pieces, their rings, and the vertex pool the rings point into
  uint32_t* g; uint32_t* path; uint32_t* depth; uint32_t* r0; uint32_t* nr;
  uint64_t* rv0; uint32_t* rn;
  const double2* xy; const uint8_t* syn;   // syn == nullptr: no cut edges yet
};

// warp per piece: vertex count, bbox, leaf or split (subdivide.h:52-67)
__global__ void k_sub_stats(Pieces P, uint32_t np, int maxv, uint8_t* leaf, uint8_t* axis, double* mid, unsigned long long* nv_out) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw) {
    uint64_t nv = 0;
    double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
    for (uint32_t r = P.r0[p]; r < P.r0[p] + P.nr[p]; r++) {
      const uint64_t v0 = P.rv0[r], n = P.rn[r];
      nv += n;
      for (uint64_t i = lane; i < n; i += 32) {
        const double2 q = P.xy[v0 + i];
        x0 = fmin(x0, q.x); x1 = fmax(x1, q.x); y0 = fmin(y0, q.y); y1 = fmax(y1, q.y);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o)); x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
      y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o)); y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) {
      const bool lf = nv <= (uint64_t)maxv || P.depth[p] >= SUB_MAX_DEPTH || (x1 - x0 <= 0 && y1 - y0 <= 0);
      leaf[p] = lf;
      axis[p] = (x1 - x0) >= (y1 - y0) ? 0 : 1;
      mid[p] = axis[p] == 0 ? 0.5 * (x0 + x1) : 0.5 * (y0 + y1);
      nv_out[p] = nv;
    }
  }
}

__global__ void k_sub_leaf_sizes(const Pieces P, uint32_t np, const uint8_t* __restrict__ leaf, const unsigned long long* __restrict__ nv,
                                 unsigned long long* lv, unsigned long long* lr, uint32_t* lf) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p > np) return;
  if (p == np) { lv[p] = 0; lr[p] = 0; lf[p] = 0; return; }
  lv[p] = leaf[p] ? nv[p] : 0;
  lr[p] = leaf[p] ? P.nr[p] : 0;
  lf[p] = leaf[p];
}

// warp per leaf piece: its rings into the leaf pool, its key and ring range into the leaf list
__global__ void k_sub_emit_leaves(const Pieces P, uint32_t np, const uint8_t* __restrict__ leaf, const unsigned long long* __restrict__ lvo,
                                  const unsigned long long* __restrict__ lro, const uint32_t* __restrict__ lfo, uint64_t vbase, uint64_t rbase,
                                  uint64_t lbase, double2* lxy, uint8_t* lsyn, uint64_t* lrv0, uint32_t* lrn, unsigned long long* lkey, uint64_t* lr0,
                                  uint32_t* lnr) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw) {
    if (!leaf[p]) continue;
    uint64_t vo = vbase + lvo[p];
    const uint64_t ro = rbase + lro[p];
    for (uint32_t k = 0; k < P.nr[p]; k++) {
      const uint32_t r = P.r0[p] + k;
      const uint64_t v0 = P.rv0[r], n = P.rn[r];
      for (uint64_t i = lane; i < n; i += 32) {
        lxy[vo + i] = P.xy[v0 + i];
        lsyn[vo + i] = P.syn ? P.syn[v0 + i] : 0;
      }
      if (lane == 0) { lrv0[ro + k] = vo; lrn[ro + k] = (uint32_t)n; }
      vo += n;
    }
    if (lane == 0) {
      const uint64_t l = lbase + lfo[p];
      lkey[l] = ((unsigned long long)P.g[p] << 24) | P.path[p];
      lr0[l] = ro; lnr[l] = P.nr[p];
    }
  }
}

// thread per (side, ring of a split piece): clipped point count (pass 1) or the points (pass 2)
__global__ void k_sub_clip(const Pieces P, const uint32_t* __restrict__ rpiece, uint32_t nrings, const uint8_t* __restrict__ leaf,
                           const uint8_t* __restrict__ axis, const double* __restrict__ mid, uint32_t* cnt, const unsigned long long* voff,
                           double2* oxy, uint8_t* osyn) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2ull * nrings) return;
  const uint32_t side = (uint32_t)(e / nrings), r = (uint32_t)(e % nrings);
  const uint32_t p = rpiece[r];
  if (leaf[p]) { if (!oxy) cnt[e] = 0; return; }
  ClipOut out;
  if (oxy) {
    if (cnt[e] == 0) return;
    out.xy = oxy + voff[e]; out.syn = osyn + voff[e];
  }
  const uint32_t k = clip_ring_dev(P.xy + P.rv0[r], P.syn ? P.syn + P.rv0[r] : nullptr, P.rn[r], axis[p], mid[p], side == 0, out);
  if (!oxy) cnt[e] = k;
}

__global__ void k_u32_to_u64(const uint32_t* __restrict__ a, uint64_t n, unsigned long long* b, uint32_t* nz) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) { b[i] = a[i]; nz[i] = a[i] != 0; }
  else if (i == n) { b[i] = 0; nz[i] = 0; }
}

// new pieces: (side, split piece) with at least one kept ring; ring range = the nonzero-ring scan across its entries
__global__ void k_sub_new_pieces(const Pieces P, uint32_t np, uint32_t nrings, const uint8_t* __restrict__ leaf, const uint32_t* __restrict__ rix,
                                 uint32_t* exists) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q > 2ull * np) return;
  if (q == 2ull * np) { exists[q] = 0; return; }
  const uint32_t side = (uint32_t)(q / np), p = (uint32_t)(q % np);
  if (leaf[p]) { exists[q] = 0; return; }
  const uint64_t e0 = (uint64_t)side * nrings + P.r0[p], e1 = e0 + P.nr[p];
  exists[q] = rix[e1] > rix[e0];
}
__global__ void k_sub_fill_pieces(const Pieces P, uint32_t np, uint32_t nrings, const uint32_t* __restrict__ rix, const uint32_t* __restrict__ exists,
                                  const uint32_t* __restrict__ qix, Pieces N) {
  const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2ull * np || !exists[q]) return;
  const uint32_t side = (uint32_t)(q / np), p = (uint32_t)(q % np);
  const uint64_t e0 = (uint64_t)side * nrings + P.r0[p], e1 = e0 + P.nr[p];
  const uint32_t k = qix[q];
  N.g[k] = P.g[p];
  N.path[k] = P.path[p] | (side << (SUB_MAX_DEPTH - 1 - P.depth[p]));
  N.depth[k] = P.depth[p] + 1;
  N.r0[k] = rix[e0];
  N.nr[k] = rix[e1] - rix[e0];
}
// thread per kept entry: the new ring table (vertex offset, count, owning new piece)
__global__ void k_sub_fill_rings(const Pieces P, uint32_t np, uint32_t nrings, const uint32_t* __restrict__ rpiece, const uint32_t* __restrict__ cnt,
                                 const unsigned long long* __restrict__ voff, const uint32_t* __restrict__ rix, const uint32_t* __restrict__ qix,
                                 uint64_t* nrv0, uint32_t* nrn, uint32_t* nrpiece) {
  const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 2ull * nrings || cnt[e] == 0) return;
  const uint32_t side = (uint32_t)(e / nrings), r = (uint32_t)(e % nrings);
  const uint32_t k = rix[e];
  nrv0[k] = voff[e]; nrn[k] = cnt[e];
  nrpiece[k] = qix[(uint64_t)side * np + rpiece[r]];
}

// the output in key order: warp per sorted leaf
__global__ void k_sub_leaf_counts(const uint32_t* __restrict__ order, uint32_t nl, const uint64_t* __restrict__ lr0, const uint32_t* __restrict__ lnr,
                                  const uint32_t* __restrict__ lrn, unsigned long long* onr, unsigned long long* onv) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > nl) return;
  if (i == nl) { onr[i] = 0; onv[i] = 0; return; }
  const uint32_t l = order[i];
  uint64_t nv = 0;
  for (uint32_t k = 0; k < lnr[l]; k++) nv += lrn[lr0[l] + k];
  onr[i] = lnr[l]; onv[i] = nv;
}
__global__ void k_sub_gather(const uint32_t* __restrict__ order, const unsigned long long* __restrict__ skey, uint32_t nl, const uint64_t* __restrict__ lr0,
                             const uint32_t* __restrict__ lnr, const uint64_t* __restrict__ lrv0, const uint32_t* __restrict__ lrn,
                             const double2* __restrict__ lxy, const uint8_t* __restrict__ lsyn, const unsigned long long* __restrict__ gro,
                             const unsigned long long* __restrict__ vbase, uint64_t* orvo, double2* oxy, uint8_t* osyn, uint32_t* opar) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < nl; i += nw) {
    const uint32_t l = order[i];
    uint64_t vo = vbase[i];
    for (uint32_t k = 0; k < lnr[l]; k++) {
      const uint64_t src = lrv0[lr0[l] + k], n = lrn[lr0[l] + k];
      if (lane == 0) orvo[gro[i] + k] = vo;
      for (uint64_t j = lane; j < n; j += 32) { oxy[vo + j] = lxy[src + j]; osyn[vo + j] = lsyn[src + j]; }
      vo += n;
    }
    if (lane == 0) opar[i] = (uint32_t)(skey[i] >> 24);
  }
}

}  // namespace

namespace {

__global__ void k_sub_init(const uint64_t* __restrict__ gro, const uint64_t* __restrict__ rvo, uint32_t n, Pieces P, uint32_t* rpiece) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  P.g[g] = g; P.path[g] = 0; P.depth[g] = 0;
  P.r0[g] = (uint32_t)gro[g]; P.nr[g] = (uint32_t)(gro[g + 1] - gro[g]);
  for (uint64_t r = gro[g]; r < gro[g + 1]; r++) { P.rv0[r] = rvo[r]; P.rn[r] = (uint32_t)(rvo[r + 1] - rvo[r]); rpiece[r] = g; }
}

// grow keeping the first `used` bytes (stream-ordered)
void* grow_keep(DevBuf& b, size_t used, size_t need, cudaStream_t s) {
  if (need <= b.cap && b.p) return b.p;
  const size_t want = need + need / 2 + 256;
  void* p = nullptr;
  GSJ_CK(cudaMallocAsync(&p, want, s));
  if (used && b.p) GSJ_CK(cudaMemcpyAsync(p, b.p, used, cudaMemcpyDeviceToDevice, s));
  if (b.p) cudaFreeAsync(b.p, s);
  b.p = p; b.cap = want;
  return p;
}

template <class T> uint64_t exscan_total(gsj_ctx* c, const T* in, T* out, uint64_t n, DevBuf& tmp) {   // out[0..n]: in has n + 1 entries
  size_t tb = 0;
  GSJ_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, (int64_t)n + 1, c->stream));
  GSJ_CK(cub::DeviceScan::ExclusiveSum(tmp.get(tb), tb, in, out, (int64_t)n + 1, c->stream));
  T h = 0;
  GSJ_CK(cudaMemcpyAsync(&h, out + n, sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  return (uint64_t)h;
}

}  // namespace

void subdivide_gpu(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy, int maxv,
                   uint64_t* out_n, uint64_t* out_nr, uint64_t* out_nv, uint64_t** out_gro, uint64_t** out_rvo, double** out_xy, uint32_t** out_parent,
                   uint8_t** out_syn) {
  if (!gro || !rvo || !xy || maxv < 4 || !out_n || !out_nr || !out_nv || !out_gro || !out_rvo || !out_xy || !out_parent || !out_syn)
    throw Error(GSJ_ERR_ARG, "bad arguments");
  if (n == 0 || n >= (1ull << 32) - 1 || nr >= (1ull << 32) - 1 || gro[0] != 0 || gro[n] != nr || rvo[0] != 0 || rvo[nr] != nv)
    throw Error(GSJ_ERR_ARG, "inconsistent offsets");
  cudaStream_t s = c->stream;
  DevBuf bgro, brvo, bxy, tmp, st_leaf, st_axis, st_mid, st_nv, lv, lr, lf, lvo, lro, lfo, cnt, cnt64, nz, voff, rix, ex, qix;
  DevBuf LXY, LSYN, LRV0, LRN, LKEY, LR0, LNR;
  DevBuf pg[2], ppath[2], pdepth[2], pr0[2], pnr[2], prv0[2], prn[2], prp[2], pxy[2], psyn[2];
  for (DevBuf* b : {&bgro, &brvo, &bxy, &tmp, &st_leaf, &st_axis, &st_mid, &st_nv, &lv, &lr, &lf, &lvo, &lro, &lfo, &cnt, &cnt64, &nz, &voff, &rix,
                    &ex, &qix, &LXY, &LSYN, &LRV0, &LRN, &LKEY, &LR0, &LNR})
    b->s = s;
  for (int k = 0; k < 2; k++)
    for (DevBuf* b : {&pg[k], &ppath[k], &pdepth[k], &pr0[k], &pnr[k], &prv0[k], &prn[k], &prp[k], &pxy[k], &psyn[k]}) b->s = s;
  uint64_t* dgro = bgro.as<uint64_t>(n + 1);
  uint64_t* drvo = brvo.as<uint64_t>(nr + 1);
  double2* dxy = bxy.as<double2>(nv + 1);
  GSJ_CK(cudaMemcpyAsync(dgro, gro, 8 * (n + 1), cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(drvo, rvo, 8 * (nr + 1), cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(dxy, xy, 16 * nv, cudaMemcpyHostToDevice, s));
  auto bind = [&](int k, uint64_t np_, uint64_t nrg) {
    Pieces P;
    P.g = pg[k].as<uint32_t>(np_); P.path = ppath[k].as<uint32_t>(np_); P.depth = pdepth[k].as<uint32_t>(np_);
    P.r0 = pr0[k].as<uint32_t>(np_); P.nr = pnr[k].as<uint32_t>(np_);
    P.rv0 = prv0[k].as<uint64_t>(nrg); P.rn = prn[k].as<uint32_t>(nrg);
    P.xy = nullptr; P.syn = nullptr;
    return P;
  };
  int cur = 0;
  Pieces P = bind(cur, n, nr);
  uint32_t* rpiece = prp[cur].as<uint32_t>(nr);
  P.xy = dxy; P.syn = nullptr;
  k_sub_init<<<grid_for(n, 256), 256, 0, s>>>(dgro, drvo, (uint32_t)n, P, rpiece); c->launches++;
  uint64_t np = n, nrings = nr, LV = 0, LR = 0, NL = 0;
  for (int round = 0; np > 0; round++) {
    if (round > SUB_MAX_DEPTH + 1) throw Error(GSJ_ERR_CUDA, "subdivision did not terminate");
    uint8_t* leaf = st_leaf.as<uint8_t>(np);
    uint8_t* axis = st_axis.as<uint8_t>(np);
    double* mid = st_mid.as<double>(np);
    unsigned long long* nvp = st_nv.as<unsigned long long>(np);
    const int wgrid = (int)std::min<uint64_t>((np * 32 + 255) / 256, (uint64_t)c->sm_count * 64);
    k_sub_stats<<<wgrid, 256, 0, s>>>(P, (uint32_t)np, maxv, leaf, axis, mid, nvp); c->launches++;
    unsigned long long* dlv = lv.as<unsigned long long>(np + 1);
    unsigned long long* dlr = lr.as<unsigned long long>(np + 1);
    uint32_t* dlf = lf.as<uint32_t>(np + 1);
    k_sub_leaf_sizes<<<grid_for(np + 1, 256), 256, 0, s>>>(P, (uint32_t)np, leaf, nvp, dlv, dlr, dlf); c->launches++;
    unsigned long long* dlvo = lvo.as<unsigned long long>(np + 1);
    unsigned long long* dlro = lro.as<unsigned long long>(np + 1);
    uint32_t* dlfo = lfo.as<uint32_t>(np + 1);
    const uint64_t dv = exscan_total(c, dlv, dlvo, np, tmp), dr = exscan_total(c, dlr, dlro, np, tmp), dl = exscan_total(c, dlf, dlfo, np, tmp);
    if (dl) {
      double2* lxy = (double2*)grow_keep(LXY, 16 * LV, 16 * (LV + dv) + 16, s);
      uint8_t* lsyn = (uint8_t*)grow_keep(LSYN, LV, LV + dv + 16, s);
      uint64_t* lrv0 = (uint64_t*)grow_keep(LRV0, 8 * LR, 8 * (LR + dr) + 16, s);
      uint32_t* lrn = (uint32_t*)grow_keep(LRN, 4 * LR, 4 * (LR + dr) + 16, s);
      unsigned long long* lkey = (unsigned long long*)grow_keep(LKEY, 8 * NL, 8 * (NL + dl) + 16, s);
      uint64_t* lr0 = (uint64_t*)grow_keep(LR0, 8 * NL, 8 * (NL + dl) + 16, s);
      uint32_t* lnr = (uint32_t*)grow_keep(LNR, 4 * NL, 4 * (NL + dl) + 16, s);
      k_sub_emit_leaves<<<wgrid, 256, 0, s>>>(P, (uint32_t)np, leaf, dlvo, dlro, dlfo, LV, LR, NL, lxy, lsyn, lrv0, lrn, lkey, lr0, lnr); c->launches++;
      LV += dv; LR += dr; NL += dl;
    }
    if (dl == np) break;   // no split pieces left
    // split pieces: count pass, offsets, write pass
    const uint64_t ne = 2 * nrings;
    uint32_t* dcnt = cnt.as<uint32_t>(ne + 1);
    k_sub_clip<<<grid_for(ne, 128), 128, 0, s>>>(P, rpiece, (uint32_t)nrings, leaf, axis, mid, dcnt, nullptr, nullptr, nullptr); c->launches++;
    unsigned long long* dc64 = cnt64.as<unsigned long long>(ne + 1);
    uint32_t* dnz = nz.as<uint32_t>(ne + 1);
    k_u32_to_u64<<<grid_for(ne + 1, 256), 256, 0, s>>>(dcnt, ne, dc64, dnz); c->launches++;
    unsigned long long* dvoff = voff.as<unsigned long long>(ne + 1);
    uint32_t* drix = rix.as<uint32_t>(ne + 1);
    const uint64_t NV = exscan_total(c, dc64, dvoff, ne, tmp), NR = exscan_total(c, dnz, drix, ne, tmp);
    uint32_t* dex = ex.as<uint32_t>(2 * np + 1);
    uint32_t* dqix = qix.as<uint32_t>(2 * np + 1);
    k_sub_new_pieces<<<grid_for(2 * np + 1, 256), 256, 0, s>>>(P, (uint32_t)np, (uint32_t)nrings, leaf, drix, dex); c->launches++;
    const uint64_t NP = exscan_total(c, dex, dqix, 2 * np, tmp);
    if (NR >= (1ull << 32) - 1 || NP >= (1ull << 32) - 1) throw Error(GSJ_ERR_NOMEM, "subdivision too large");
    const int nxt = cur ^ 1;
    Pieces N = bind(nxt, NP, NR);
    double2* nxy = pxy[nxt].as<double2>(NV + 1);
    uint8_t* nsyn = psyn[nxt].as<uint8_t>(NV + 1);
    N.xy = nxy; N.syn = nsyn;
    uint32_t* nrp = prp[nxt].as<uint32_t>(NR);
    k_sub_clip<<<grid_for(ne, 128), 128, 0, s>>>(P, rpiece, (uint32_t)nrings, leaf, axis, mid, dcnt, dvoff, nxy, nsyn); c->launches++;
    k_sub_fill_pieces<<<grid_for(2 * np, 256), 256, 0, s>>>(P, (uint32_t)np, (uint32_t)nrings, drix, dex, dqix, N); c->launches++;
    k_sub_fill_rings<<<grid_for(ne, 256), 256, 0, s>>>(P, (uint32_t)np, (uint32_t)nrings, rpiece, dcnt, dvoff, drix, dqix, N.rv0, N.rn, nrp); c->launches++;
    GSJ_CK(cudaGetLastError());
    cur = nxt; P = N; rpiece = nrp; np = NP; nrings = NR;
  }
  // leaves in (geometry, cut path) order -> the output arrays
  unsigned long long* skey = reinterpret_cast<unsigned long long*>(cnt64.get(8 * (NL + 1)));
  uint32_t* ord_in = reinterpret_cast<uint32_t*>(nz.get(4 * (NL + 1)));
  uint32_t* order = reinterpret_cast<uint32_t*>(ex.get(4 * (NL + 1)));
  {
    std::vector<uint32_t> iota(NL);
    for (uint64_t i = 0; i < NL; i++) iota[i] = (uint32_t)i;
    GSJ_CK(cudaMemcpyAsync(ord_in, iota.data(), 4 * NL, cudaMemcpyHostToDevice, s));
    size_t tb = 0;
    GSJ_CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, (const unsigned long long*)LKEY.p, skey, ord_in, order, (int64_t)NL, 0, 56, s));
    GSJ_CK(cub::DeviceRadixSort::SortPairs(tmp.get(tb), tb, (const unsigned long long*)LKEY.p, skey, ord_in, order, (int64_t)NL, 0, 56, s));
    GSJ_CK(cudaStreamSynchronize(s));
  }
  unsigned long long* onr = lv.as<unsigned long long>(NL + 1);
  unsigned long long* onv = lr.as<unsigned long long>(NL + 1);
  k_sub_leaf_counts<<<grid_for(NL + 1, 256), 256, 0, s>>>(order, (uint32_t)NL, (const uint64_t*)LR0.p, (const uint32_t*)LNR.p, (const uint32_t*)LRN.p, onr, onv);
  c->launches++;
  unsigned long long* ogro = lvo.as<unsigned long long>(NL + 1);
  unsigned long long* ovb = lro.as<unsigned long long>(NL + 1);
  const uint64_t TR = exscan_total(c, onr, ogro, NL, tmp), TV = exscan_total(c, onv, ovb, NL, tmp);
  uint64_t* orvo = reinterpret_cast<uint64_t*>(voff.get(8 * (TR + 1)));
  double2* oxy = reinterpret_cast<double2*>(pxy[0].get(16 * (TV + 1)));   // the round pools are free now (leaves hold copies)
  uint8_t* osyn = reinterpret_cast<uint8_t*>(psyn[0].get(TV + 1));
  uint32_t* opar = reinterpret_cast<uint32_t*>(rix.get(4 * (NL + 1)));
  const int lgrid = (int)std::min<uint64_t>((NL * 32 + 255) / 256, (uint64_t)c->sm_count * 64);
  k_sub_gather<<<lgrid, 256, 0, s>>>(order, skey, (uint32_t)NL, (const uint64_t*)LR0.p, (const uint32_t*)LNR.p, (const uint64_t*)LRV0.p,
                                    (const uint32_t*)LRN.p, (const double2*)LXY.p, (const uint8_t*)LSYN.p, ogro, ovb, orvo, oxy, osyn, opar);
  c->launches++;
  GSJ_CK(cudaMemcpyAsync(orvo + TR, &TV, 8, cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaGetLastError());
  uint64_t* hgro = (uint64_t*)malloc(8 * (NL + 1));
  uint64_t* hrvo = (uint64_t*)malloc(8 * (TR + 1));
  double* hxy = (double*)malloc(16 * (TV ? TV : 1));
  uint32_t* hpar = (uint32_t*)malloc(4 * (NL ? NL : 1));
  uint8_t* hsyn = (uint8_t*)malloc(TV ? TV : 1);
  if (!hgro || !hrvo || !hxy || !hpar || !hsyn) {
    free(hgro); free(hrvo); free(hxy); free(hpar); free(hsyn);
    throw Error(GSJ_ERR_NOMEM, "host allocation failed");
  }
  GSJ_CK(cudaMemcpyAsync(hgro, ogro, 8 * (NL + 1), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hrvo, orvo, 8 * (TR + 1), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hxy, oxy, 16 * TV, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hpar, opar, 4 * NL, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaMemcpyAsync(hsyn, osyn, TV, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  *out_n = NL; *out_nr = TR; *out_nv = TV;
  *out_gro = hgro; *out_rvo = hrvo; *out_xy = hxy; *out_parent = hpar; *out_syn = hsyn;
}

}  // namespace gsj
