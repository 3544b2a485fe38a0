// Candidate search: LBVH traversal, one thread per probe box, probes taken in Morton order so the lanes of a warp
// walk neighbouring parts of the tree (the reference's k_traverse, engine/engine.cuh:233-259, runs a count pass
// and a write pass; here one pass appends with one atomic per warp step).
#include "engine.h"

namespace gsj {

constexpr int TRAV_STACK = 96;   // > tree depth (unique 64-bit keys bound the depth by 64)

__device__ __forceinline__ bool box_hit(const float4& c, const float4& b) {
  return !(c.x > b.z || c.z < b.x || c.y > b.w || c.w < b.y);
}

__global__ void __launch_bounds__(128) k_traverse(const float4* __restrict__ qbb, const uint32_t* __restrict__ qorder, uint32_t q0, uint32_t nq,
                                                  DBvh T, int upper, uint2* __restrict__ out, unsigned long long cap,
                                                  unsigned long long* counter, int* err, unsigned long long* visits) {
  const int lane = threadIdx.x & 31;
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < nq;
  uint32_t qi = 0;
  float4 b = make_float4(0, 0, 0, 0);
  int stack[TRAV_STACK];
  int sp = 0;
  if (active) {
    qi = qorder ? qorder[q0 + t] : q0 + t;
    b = qbb[qi];
    stack[sp++] = 0;
  }
  const unsigned lt = (1u << lane) - 1;
  unsigned long long nvis = 0;
  for (;;) {
    bool work = sp > 0;
    if (!__any_sync(0xffffffffu, work)) break;
    uint32_t h0 = 0, h1 = 0; int nh = 0;
    if (work) {
      int node = stack[--sp];
      nvis++;
      const BNode nd = T.nodes[node];
      bool hl = box_hit(nd.lb, b), hr = box_hit(nd.rb, b);
      if (hr) {
        if (nd.r < 0) { uint32_t id = (uint32_t)~nd.r; if (!upper || id >= qi) { h0 = id; nh = 1; } }
        else if (sp < TRAV_STACK) stack[sp++] = nd.r; else *err = 1;
      }
      if (hl) {
        if (nd.l < 0) { uint32_t id = (uint32_t)~nd.l; if (!upper || id >= qi) { if (nh) h1 = id; else h0 = id; nh++; } }
        else if (sp < TRAV_STACK) stack[sp++] = nd.l; else *err = 1;
      }
    }
    // warp-aggregated append: one atomic per warp step
    unsigned m1 = __ballot_sync(0xffffffffu, nh >= 1), m2 = __ballot_sync(0xffffffffu, nh >= 2);
    int tot = __popc(m1) + __popc(m2);
    if (tot) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(counter, (unsigned long long)tot);
      base = __shfl_sync(0xffffffffu, base, 0);
      unsigned long long pos = base + __popc(m1 & lt) + __popc(m2 & lt);
      if (nh >= 1 && pos < cap) out[pos] = make_uint2(qi, h0);
      if (nh >= 2 && pos + 1 < cap) out[pos + 1] = make_uint2(qi, h1);
    }
  }
  for (int o = 16; o > 0; o >>= 1) nvis += __shfl_xor_sync(0xffffffffu, nvis, o);
  if (lane == 0 && nvis) atomicAdd(visits, nvis);
}

uint64_t traverse(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper, uint2* out,
                  uint64_t cap) {
  if (nq == 0) return 0;
  unsigned long long* ctr = c->counters.as<unsigned long long>(8);
  int* err = reinterpret_cast<int*>(ctr + 1);
  GSJ_CK(cudaMemsetAsync(ctr, 0, 24, c->stream));
  k_traverse<<<grid_for(nq, 128), 128, 0, c->stream>>>(qbb, qorder, q0, nq, T, upper, out, cap, ctr, err, ctr + 2); c->launches++;
  GSJ_CK(cudaGetLastError());
  unsigned long long* h = c->h_counters.as<unsigned long long>(3);
  GSJ_CK(cudaMemcpyAsync(h, ctr, 24, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  if (reinterpret_cast<int*>(h + 1)[0]) throw Error(GSJ_ERR_CUDA, "traversal stack overflow");
  c->node_visits += h[2];
  return h[0];
}

}  // namespace gsj
