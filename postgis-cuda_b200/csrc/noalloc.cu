// Refinement of caller-supplied candidate pairs without any device allocation.
//
// Who needs this: callers that must not allocate device memory once they are running - a server that reserved
// its whole device-memory budget up front and hands every byte to its own arena, or a request path that cannot
// afford cudaMalloc/cudaFree's implicit device-wide synchronisation. They pass device buffers for the pairs and
// the results; the per-warp edge lists of the refinement live in one file-scope static device array instead of
// the context's grow-only pools (which allocate on first use and when a request outgrows them).
//
// Limits and sharing: the array is GSJ_NOALLOC_SCRATCH_BYTES (32 MiB) on every GPU that loads the library, held
// until the process exits. A call needs 2 x cap x 36 bytes per warp, cap = the larger of the two layers' largest
// geometry edge count rounded up to 8; calls whose one-warp slab does not fit are rejected with GSJ_ERR_ARG.
// Every call on a device uses the same array: calls that overlap on the GPU (other streams, other contexts on
// the device, other host threads) race on it and must be serialised by the caller. The first call on a device
// looks the array's device address up (cudaGetSymbolAddress). The address is kept for the life of the process: a
// host application that resets a device (cudaDeviceReset) must not call this entry point on that device afterwards.
// Every call synchronises the context's stream (the status word comes back to the host), so no call can be captured
// into a CUDA graph.
#include <mutex>
#include "engine.h"

namespace gsj {

__device__ bool refine_pair(const DLayer& P, const DLayer& R, uint32_t a, uint32_t b, const RefineArgs& rp, EList LA, EList LB, int cap,
                            int lane, uint8_t& o_flag, double& o_area, double4& o_ev, uint32_t& o_evb);

constexpr size_t NOALLOC_HEAD = 256;   // error word, then the warp slabs
static __device__ __align__(256) unsigned char g_noalloc_scratch[GSJ_NOALLOC_SCRATCH_BYTES];

__device__ __forceinline__ EList carve_global(unsigned char* base, int cap) {
  EList L;
  L.x0 = reinterpret_cast<double*>(base);
  L.y0 = L.x0 + cap; L.x1 = L.y0 + cap; L.y1 = L.x1 + cap;
  L.fl = reinterpret_cast<uint32_t*>(L.y1 + cap);
  return L;
}

// one warp per block; warp w uses slab w of the static array (base = its device address, passed by the host)
__global__ void __launch_bounds__(32) k_refine_static(DLayer P, DLayer R, const uint2* __restrict__ pairs, uint64_t np, RefineArgs rp,
                                                      uint8_t* flag, double* area, double4* ev, uint32_t* evb, unsigned char* base,
                                                      int cap) {
  const int lane = threadIdx.x & 31;
  int* err = reinterpret_cast<int*>(base);
  const size_t slab = 2 * (size_t)cap * (4 * sizeof(double) + sizeof(uint32_t));
  unsigned char* mine = base + NOALLOC_HEAD + (size_t)blockIdx.x * slab;
  EList LA = carve_global(mine, cap), LB = carve_global(mine + slab / 2, cap);
  for (uint64_t p = blockIdx.x; p < np; p += gridDim.x) {
    const uint2 pr = pairs[p];
    if (pr.x >= P.n || pr.y >= R.n) {   // a caller's index out of range: record it, skip the pair
      if (lane == 0) {
        atomicExch(err, 2);
        flag[p] = 0;
        if (area) area[p] = 0.0;
        if (ev) { ev[p] = make_double4(0, 0, 0, 0); evb[p] = 0u; }
      }
      continue;
    }
    uint8_t f; double ar; double4 e4; uint32_t b4;
    const bool ok = refine_pair(P, R, pr.x, pr.y, rp, LA, LB, cap, lane, f, ar, e4, b4);
    if (lane == 0) {
      if (!ok) atomicExch(err, 1);
      flag[p] = ok ? f : 0;
      if (area) area[p] = ok ? ar : 0.0;
      if (ev) { ev[p] = ok ? e4 : make_double4(0, 0, 0, 0); evb[p] = ok ? b4 : 0u; }
    }
    __syncwarp();
  }
}

RefineArgs to_args(const gsj_refine_params* p);

// device address of the static array, looked up once per device with that device current
static unsigned char* scratch_address(int device) {
  static std::mutex mu;
  static unsigned char* addr[64] = {};
  if (device < 0 || device >= 64) throw Error(GSJ_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) throw Error(GSJ_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    addr[device] = static_cast<unsigned char*>(p);
  }
  return addr[device];
}

void refine_pairs_noalloc(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint32_t* d_pairs, uint64_t np,
                          const gsj_refine_params* rpp, uint8_t* d_flag, double* d_area, double* d_ev, uint32_t* d_evb) {
  if (P->is_points || R->is_points) throw Error(GSJ_ERR_ARG, "refinement needs two polygon layers");
  if (np && (!d_pairs || !d_flag)) throw Error(GSJ_ERR_ARG, "pairs and flag buffers are required");
  if ((d_ev == nullptr) != (d_evb == nullptr)) throw Error(GSJ_ERR_ARG, "ev and evb go together");
  const uint64_t emax = std::max(P->max_geom_edges, R->max_geom_edges);
  const uint64_t cap = std::max<uint64_t>((emax + 7) & ~7ull, 8);
  const uint64_t slab = 2 * cap * (4 * sizeof(double) + sizeof(uint32_t));
  const uint64_t room = GSJ_NOALLOC_SCRATCH_BYTES - NOALLOC_HEAD;
  if (slab > room)
    throw Error(GSJ_ERR_ARG, "geometries too large for the static scratch: one warp needs " + std::to_string(slab) + " bytes, the array holds " +
                                 std::to_string(room) + " (max " + std::to_string(room / 72) + " edges per geometry)");
  unsigned char* base = scratch_address(c->device);
  cudaStream_t s = c->stream;
  GSJ_CK(cudaMemsetAsync(base, 0, sizeof(int), s));   // the error word keeps the previous call's value otherwise
  if (np) {
    const uint64_t warps = std::min<uint64_t>(std::min<uint64_t>(room / slab, (uint64_t)c->sm_count * 16), np);
    const RefineArgs rp = to_args(rpp);
    k_refine_static<<<(unsigned)warps, 32, 0, s>>>(P->d, R->d, reinterpret_cast<const uint2*>(d_pairs), np, rp, d_flag, d_area,
                                                   reinterpret_cast<double4*>(d_ev), d_evb, base, (int)cap);
    GSJ_CK(cudaGetLastError());
  }
  int herr = 0;
  GSJ_CK(cudaMemcpyAsync(&herr, base, sizeof(int), cudaMemcpyDeviceToHost, s));
  GSJ_CK(cudaStreamSynchronize(s));
  if (herr == 2) throw Error(GSJ_ERR_ARG, "a pair index is out of range for its layer");
  if (herr) throw Error(GSJ_ERR_CUDA, "a pair's edge list exceeded the static scratch slab");
}

}  // namespace gsj

extern "C" int gsj_refine_pairs_noalloc(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint32_t* d_pairs, uint64_t np,
                                        const gsj_refine_params* rp, uint8_t* d_flag, double* d_area, double* d_ev, uint32_t* d_evb) {
  if (!c || !P || !R) return GSJ_ERR_ARG;
  try {
    GSJ_CK(cudaSetDevice(c->device));
    gsj::refine_pairs_noalloc(c, P, R, d_pairs, np, rp, d_flag, d_area, d_ev, d_evb);
    c->err.clear();
    return GSJ_OK;
  } catch (const gsj::Error& e) {
    c->err = e.what();
    return e.code;
  }
}
