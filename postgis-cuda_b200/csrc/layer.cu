// Resident layers: upload + on-device preparation (engine/engine.cuh:42-97 of the reference does this on the
// host) and the LBVH build (Karras 2012: Morton keys, device radix sort, internal nodes from key prefixes,
// bottom-up refit; the reference's build_bvh, engine.cuh:99-228).
#include <algorithm>
#include <cmath>
#include <cub/cub.cuh>
#include <omp.h>
#include <thread>
#include "engine.h"

namespace gsj {

// warp per geometry: bbox over its vertices -> origin / extent / outward-rounded float box, then vertices made
// relative to the origin in place (exact by Sterbenz for the pair frames; engine.cuh:49-64)
__global__ void k_prep_polygons(uint32_t n, const uint32_t* __restrict__ gro, const uint64_t* __restrict__ rvo, double2* xy,
                                double2* origin, double2* ext, float4* bb) {
  const int lane = threadIdx.x & 31;
  const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t g = w; g < n; g += nw) {
    uint64_t v0 = rvo[gro[g]], v1 = rvo[gro[g + 1]];
    double x0 = 1e300, y0 = 1e300, x1 = -1e300, y1 = -1e300;
    for (uint64_t v = v0 + lane; v < v1; v += 32) {
      double2 p = xy[v];
      x0 = fmin(x0, p.x); x1 = fmax(x1, p.x); y0 = fmin(y0, p.y); y1 = fmax(y1, p.y);
    }
    for (int o = 16; o > 0; o >>= 1) {
      x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o)); x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
      y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o)); y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
    }
    if (lane == 0) {
      origin[g] = make_double2(x0, y0);
      ext[g] = make_double2(x1 - x0, y1 - y0);
      // largest float <= v and smallest float >= v (the reference's f_down / f_up, engine.cuh:34-35)
      bb[g] = make_float4(__double2float_rd(x0), __double2float_rd(y0), __double2float_ru(x1), __double2float_ru(y1));
    }
    for (uint64_t v = v0 + lane; v < v1; v += 32) {
      double2 p = xy[v];
      xy[v] = make_double2(p.x - x0, p.y - y0);
    }
  }
}

__global__ void k_prep_points(uint64_t n, const double2* __restrict__ xy, float4* bb) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double2 p = xy[i];
  bb[i] = make_float4(__double2float_rd(p.x), __double2float_rd(p.y), __double2float_ru(p.x), __double2float_ru(p.y));
}

// a layer's arrays come from the device's stream-ordered pool (the contexts keep it cached, so re-uploading a layer
// of the same size allocates nothing new); the upload ends with a stream synchronisation, after which every
// context's stream may use them
template <class T> static T* dmalloc(gsj_layer* L, size_t count, cudaStream_t s = nullptr) {
  void* p = nullptr;
  const size_t b = std::max<size_t>(count * sizeof(T), 16);
  if (s) GSJ_CK(cudaMallocAsync(&p, b, s));
  else GSJ_CK(cudaMalloc(&p, b));
  L->allocs.push_back(p);
  L->bytes += count * sizeof(T);
  return reinterpret_cast<T*>(p);
}

void layer_free(gsj_layer* L) {
  for (void* p : L->allocs) cudaFree(p);
  L->allocs.clear();
}

// cut-edge flags (one byte per vertex) packed into bits, one warp per 32 vertices
__global__ void k_pack_syn(uint64_t nv, const uint8_t* __restrict__ syn, uint32_t* bits) {
  const uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned m = __ballot_sync(0xffffffffu, v < nv && syn[v] != 0);
  if ((threadIdx.x & 31) == 0 && v < nv) bits[v >> 5] = m;
}

// thread per geometry: 32-bit ring offsets, edge count (the largest goes to *maxe), and the length of its real
// boundary (edges not made by subdivision) summed edge by edge in ring order from the world coordinates, as the
// reference's host loop does (engine.cuh:69-82)
__global__ void k_geom_setup(uint32_t n, const uint64_t* __restrict__ gro, const uint64_t* __restrict__ rvo, const double2* __restrict__ xy,
                             const uint32_t* __restrict__ synb, uint32_t* gro32, double* glen, unsigned int* maxe) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g > n) return;
  gro32[g] = (uint32_t)gro[g];
  if (g == n) return;
  uint64_t e = 0;
  double len = 0;
  for (uint64_t r = gro[g]; r < gro[g + 1]; r++) {
    const uint64_t v0 = rvo[r], v1 = rvo[r + 1];
    e += v1 > v0 ? v1 - v0 - 1 : 0;
    for (uint64_t v = v0; v + 1 < v1; v++) {
      if (synb && ((synb[v >> 5] >> (v & 31)) & 1u)) continue;
      const double2 p = xy[v], q = xy[v + 1];
      len += hypot(q.x - p.x, q.y - p.y);
    }
  }
  glen[g] = len;
  atomicMax(maxe, (unsigned int)(e < 0xFFFFFFFFull ? e : 0xFFFFFFFFull));
}

// per parent geometry: its pieces' lengths summed in piece order (pieces of a parent are contiguous)
__global__ void k_parent_len(uint32_t n, const uint32_t* __restrict__ parent, const double* __restrict__ glen, double* blen) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n || (g > 0 && parent[g] == parent[g - 1])) return;
  const uint32_t p = parent[g];
  double s = 0;
  for (uint32_t h = g; h < n && parent[h] == p; h++) s += glen[h];
  blen[p] = s;
}

void layer_upload_polygons(gsj_ctx* c, uint64_t n, uint64_t nr, uint64_t nv, const uint64_t* gro, const uint64_t* rvo, const double* xy,
                           const uint32_t* parent, const uint8_t* syn, gsj_layer* L) {
  if (n == 0 || n >= (1ull << 31) || nr >= (1ull << 32)) throw Error(GSJ_ERR_ARG, "layer size out of range (0 < n < 2^31 geometries, rings < 2^32)");
  if (!gro || !rvo || !xy) throw Error(GSJ_ERR_ARG, "gro / rvo / xy must not be NULL");
  if (gro[0] != 0 || gro[n] != nr || rvo[0] != 0 || rvo[nr] != nv) throw Error(GSJ_ERR_ARG, "offset arrays are inconsistent with n / nr / nv");
  int bad_g = 0, bad_r = 0, bad_p = 0;
#pragma omp parallel for reduction(| : bad_g) schedule(static)
  for (int64_t g = 0; g < (int64_t)n; g++) bad_g |= gro[g + 1] < gro[g];
#pragma omp parallel for reduction(| : bad_r) schedule(static)
  for (int64_t r = 0; r < (int64_t)nr; r++) bad_r |= rvo[r + 1] < rvo[r];
  if (parent) {
#pragma omp parallel for reduction(| : bad_p) schedule(static)
    for (int64_t g = 1; g < (int64_t)n; g++) bad_p |= parent[g] < parent[g - 1];
  }
  if (bad_g) throw Error(GSJ_ERR_ARG, "gro must be non-decreasing");
  if (bad_r) throw Error(GSJ_ERR_ARG, "rvo must be non-decreasing");
  if (bad_p) throw Error(GSJ_ERR_ARG, "parent must be non-decreasing");
  L->is_points = 0;
  L->d.n = (uint32_t)n; L->d.nr = (uint32_t)nr; L->d.nv = nv;
  cudaStream_t s = c->stream;
  const uint32_t np = parent ? parent[n - 1] + 1 : (uint32_t)n;
  L->nparent = np;
  // every copy starts from the caller's arrays; the rest of the preparation runs on the device
  uint32_t* d_gro = dmalloc<uint32_t>(L, n + 1, s);
  uint64_t* d_rvo = dmalloc<uint64_t>(L, nr + 1, s);
  double2* d_xy = dmalloc<double2>(L, nv, s);
  double2* d_origin = dmalloc<double2>(L, n, s);
  double2* d_ext = dmalloc<double2>(L, n, s);
  float4* d_bb = dmalloc<float4>(L, n, s);
  double* d_len = dmalloc<double>(L, n, s);   // per geometry; also the per-parent lengths of a layer without parents
  DevBuf t_gro, t_syn, t_max;
  t_gro.s = t_syn.s = t_max.s = s;
  uint64_t* d_gro64 = t_gro.as<uint64_t>(n + 1);
  unsigned int* d_maxe = t_max.as<unsigned int>(1);
  GSJ_CK(cudaMemcpyAsync(d_gro64, gro, (n + 1) * 8, cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(d_rvo, rvo, (nr + 1) * 8, cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemcpyAsync(d_xy, xy, nv * 16, cudaMemcpyHostToDevice, s));
  GSJ_CK(cudaMemsetAsync(d_maxe, 0, 4, s));
  uint32_t* d_synb = nullptr;
  if (syn) {
    uint8_t* d_syn8 = t_syn.as<uint8_t>(nv);
    GSJ_CK(cudaMemcpyAsync(d_syn8, syn, nv, cudaMemcpyHostToDevice, s));
    d_synb = dmalloc<uint32_t>(L, (nv + 31) / 32, s);
    k_pack_syn<<<grid_for(nv, 256), 256, 0, s>>>(nv, d_syn8, d_synb); c->launches++;
    L->d.synb = d_synb;
  }
  k_geom_setup<<<grid_for(n + 1, 128), 128, 0, s>>>((uint32_t)n, d_gro64, d_rvo, d_xy, d_synb, d_gro, d_len, d_maxe); c->launches++;
  k_prep_polygons<<<grid_for((uint64_t)n * 32, 256), 256, 0, s>>>((uint32_t)n, d_gro, d_rvo, d_xy, d_origin, d_ext, d_bb); c->launches++;
  GSJ_CK(cudaGetLastError());
  L->d.gro = d_gro; L->d.rvo = d_rvo; L->d.xy = d_xy; L->d.origin = d_origin; L->d.ext = d_ext; L->d.bb = d_bb;
  if (parent) {
    uint32_t* d_par = dmalloc<uint32_t>(L, n, s);
    GSJ_CK(cudaMemcpyAsync(d_par, parent, n * 4, cudaMemcpyHostToDevice, s));
    L->d.parent = d_par;
    L->h_parent.assign(parent, parent + n);
    double* d_blen = dmalloc<double>(L, np, s);
    GSJ_CK(cudaMemsetAsync(d_blen, 0, (size_t)np * 8, s));
    k_parent_len<<<grid_for(n, 256), 256, 0, s>>>((uint32_t)n, d_par, d_len, d_blen); c->launches++;
    L->d.blen = d_blen;
  } else {
    L->d.blen = d_len;
  }
  build_bvh(c, L);
  unsigned int* h = c->h_counters.as<unsigned int>(1);
  GSJ_CK(cudaMemcpyAsync(h, d_maxe, 4, cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));   // the caller's arrays may go when this returns; other streams may use the layer
  L->max_geom_edges = h[0];
}

void layer_upload_points(gsj_ctx* c, uint64_t n, const double* xy, gsj_layer* L) {
  if (n == 0 || n >= (1ull << 31)) throw Error(GSJ_ERR_ARG, "point layer size out of range (0 < n < 2^31)");
  if (!xy) throw Error(GSJ_ERR_ARG, "xy must not be NULL");
  cudaStream_t s = c->stream;
  L->is_points = 1;
  L->d.n = (uint32_t)n; L->d.nv = n; L->nparent = (uint32_t)n;
  double2* d_xy = dmalloc<double2>(L, n, s);
  float4* d_bb = dmalloc<float4>(L, n, s);
  GSJ_CK(cudaMemcpyAsync(d_xy, xy, n * 16, cudaMemcpyHostToDevice, s));
  k_prep_points<<<grid_for(n, 256), 256, 0, s>>>(n, d_xy, d_bb); c->launches++;
  GSJ_CK(cudaGetLastError());
  L->d.xy = d_xy; L->d.bb = d_bb; L->pts = d_xy;
  build_bvh(c, L);
  GSJ_CK(cudaStreamSynchronize(s));   // the caller's array may go when this returns; other streams may use the layer
}

// ---- LBVH ---------------------------------------------------------------------------------------------------
__device__ __forceinline__ int ord_f(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7FFFFFFF; }
__device__ __forceinline__ float unord_f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }

__global__ void k_centroid_bounds(const float4* __restrict__ bb, uint32_t n, int* cmm) {
  float x0 = INFINITY, y0 = INFINITY, x1 = -INFINITY, y1 = -INFINITY;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 b = bb[i];
    float cx = 0.5f * (b.x + b.z), cy = 0.5f * (b.y + b.w);
    x0 = fminf(x0, cx); x1 = fmaxf(x1, cx); y0 = fminf(y0, cy); y1 = fmaxf(y1, cy);
  }
  for (int o = 16; o > 0; o >>= 1) {
    x0 = fminf(x0, __shfl_xor_sync(0xffffffffu, x0, o)); x1 = fmaxf(x1, __shfl_xor_sync(0xffffffffu, x1, o));
    y0 = fminf(y0, __shfl_xor_sync(0xffffffffu, y0, o)); y1 = fmaxf(y1, __shfl_xor_sync(0xffffffffu, y1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(cmm + 0, ord_f(x0)); atomicMin(cmm + 1, ord_f(y0)); atomicMax(cmm + 2, ord_f(x1)); atomicMax(cmm + 3, ord_f(y1));
  }
}

__device__ __forceinline__ uint32_t spread16(uint32_t v) {
  v = (v | (v << 8)) & 0x00FF00FFu; v = (v | (v << 4)) & 0x0F0F0F0Fu;
  v = (v | (v << 2)) & 0x33333333u; v = (v | (v << 1)) & 0x55555555u;
  return v;
}

// 64-bit keys: 32-bit Morton code of the box centre (16 bits per axis) above the geometry id, so every key is unique
__global__ void k_morton_keys(const float4* __restrict__ bb, uint32_t n, const int* cmm, unsigned long long* keys) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float minx = unord_f(cmm[0]), miny = unord_f(cmm[1]), maxx = unord_f(cmm[2]), maxy = unord_f(cmm[3]);
  float4 b = bb[i];
  float cx = 0.5f * (b.x + b.z), cy = 0.5f * (b.y + b.w);
  float sx = maxx > minx ? 1.f / (maxx - minx) : 0.f, sy = maxy > miny ? 1.f / (maxy - miny) : 0.f;
  uint32_t ix = (uint32_t)fminf(fmaxf((cx - minx) * sx * 65535.f, 0.f), 65535.f);
  uint32_t iy = (uint32_t)fminf(fmaxf((cy - miny) * sy * 65535.f, 0.f), 65535.f);
  uint32_t m = (spread16(ix) << 1) | spread16(iy);
  keys[i] = ((unsigned long long)m << 32) | i;
}

__device__ __forceinline__ int kdelta(const unsigned long long* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return __clzll(k[i] ^ k[j]);
}

// internal node i of the Karras hierarchy over sorted unique keys; children encoded (leaf: ~geometry id)
__global__ void k_karras(const unsigned long long* __restrict__ keys, int n, BNode* nodes, int* par_int, int* par_leaf, uint32_t* order) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) order[i] = (uint32_t)keys[i];
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = kdelta(keys, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int gamma = i + s * d + min(d, 0);
  int lo = min(i, j), hi = max(i, j);
  int lc, rc;
  if (lo == gamma) { lc = ~(int)(uint32_t)keys[gamma]; par_leaf[gamma] = i; } else { lc = gamma; par_int[gamma] = i; }
  if (hi == gamma + 1) { rc = ~(int)(uint32_t)keys[gamma + 1]; par_leaf[gamma + 1] = i; } else { rc = gamma + 1; par_int[gamma + 1] = i; }
  nodes[i].l = lc; nodes[i].r = rc;
}

// bottom-up boxes: the second child to arrive at a node merges (the first stops); one writer per node
__global__ void k_refit(int n, const float4* __restrict__ bb, BNode* nodes, float4* nbb, const int* par_int, const int* par_leaf, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int p = par_leaf[i];
  while (p >= 0) {
    __threadfence();
    if (atomicAdd(&flags[p], 1) == 0) return;
    __threadfence();
    int l = nodes[p].l, r = nodes[p].r;
    float4 a = l < 0 ? bb[~l] : __ldcg(nbb + l);
    float4 b = r < 0 ? bb[~r] : __ldcg(nbb + r);
    nodes[p].lb = a; nodes[p].rb = b;
    __stcg(nbb + p, make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)));
    p = par_int[p];
  }
}

__global__ void k_single_leaf(const float4* bb, BNode* nodes, uint32_t* order) {
  nodes[0].lb = bb[0]; nodes[0].l = ~0;
  nodes[0].rb = make_float4(INFINITY, INFINITY, -INFINITY, -INFINITY); nodes[0].r = ~0;
  order[0] = 0;
}

void build_bvh(gsj_ctx* c, gsj_layer* L) {
  cudaStream_t s = c->stream;
  const int n = (int)L->d.n;
  BNode* nodes = dmalloc<BNode>(L, std::max(n - 1, 1), s);
  uint32_t* order = dmalloc<uint32_t>(L, n, s);
  L->bvh.nodes = nodes; L->bvh.order = order; L->bvh.n = (uint32_t)n;
  if (n == 1) {
    k_single_leaf<<<1, 1, 0, s>>>(L->d.bb, nodes, order);
    GSJ_CK(cudaGetLastError());
    GSJ_CK(cudaStreamSynchronize(s));
    return;
  }
  DevBuf keys, keys2, tmp, par, flags, nbb, cmm;   // stream-ordered temporaries: freed behind the build on the stream
  for (DevBuf* b : {&keys, &keys2, &tmp, &par, &flags, &nbb, &cmm}) b->s = s;
  int* d_cmm = cmm.as<int>(4);
  int init[4];
  { auto ord = [](float f) { int i; memcpy(&i, &f, 4); return i >= 0 ? i : i ^ 0x7FFFFFFF; };
    init[0] = init[1] = ord(INFINITY); init[2] = init[3] = ord(-INFINITY); }
  int* h_init = c->h_counters.as<int>(4);   // pinned: the copy may still be pending when this returns
  memcpy(h_init, init, 16);
  GSJ_CK(cudaMemcpyAsync(d_cmm, h_init, 16, cudaMemcpyHostToDevice, s));
  k_centroid_bounds<<<std::min(grid_for(n, 256), c->sm_count * 8), 256, 0, s>>>(L->d.bb, n, d_cmm);
  unsigned long long* k1 = keys.as<unsigned long long>(n);
  unsigned long long* k2 = keys2.as<unsigned long long>(n);
  k_morton_keys<<<grid_for(n, 256), 256, 0, s>>>(L->d.bb, n, d_cmm, k1);
  GSJ_CK(cudaGetLastError());
  size_t tb = 0;
  GSJ_CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, k1, k2, n, 0, 64, s));
  GSJ_CK(cub::DeviceRadixSort::SortKeys(tmp.get(tb), tb, k1, k2, n, 0, 64, s));
  int* par_int = par.as<int>(2 * (size_t)n);
  int* par_leaf = par_int + n;
  GSJ_CK(cudaMemsetAsync(par_int, 0xFF, 2 * (size_t)n * sizeof(int), s));
  int* d_flags = flags.as<int>(n);
  GSJ_CK(cudaMemsetAsync(d_flags, 0, n * sizeof(int), s));
  float4* d_nbb = nbb.as<float4>(n);
  k_karras<<<grid_for(n, 256), 256, 0, s>>>(k2, n, nodes, par_int, par_leaf, order);
  k_refit<<<grid_for(n, 256), 256, 0, s>>>(n, L->d.bb, nodes, d_nbb, par_int, par_leaf, d_flags);
  c->launches += 4;
  GSJ_CK(cudaGetLastError());
}

}  // namespace gsj
