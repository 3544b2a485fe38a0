// Candidate search: LBVH traversal, QPT probe boxes per thread, probes taken in Morton order so the lanes of a warp
// walk neighbouring parts of the tree (the reference's k_traverse, engine/engine.cuh:233-259, runs a count pass
// and a write pass; here one pass appends with one atomic per warp step).
#include "engine.h"

namespace gsj {

constexpr int TRAV_STACK = 96;   // > tree depth (unique 64-bit keys bound the depth by 64)

__device__ __forceinline__ bool box_hit(const float4& c, const float4& b) {
  return !(c.x > b.z || c.z < b.x || c.y > b.w || c.w < b.y);
}

// QPT neighbouring probes per thread (adjacent in Morton order), walked in lockstep: each step issues all their node
// loads before testing any, so every lane keeps QPT independent load chains in flight (the walk is latency-bound:
// one dependent load per step otherwise).
constexpr int QPT = 4;
__global__ void __launch_bounds__(128) k_traverse(const float4* __restrict__ qbb, const uint32_t* __restrict__ qorder, uint32_t q0, uint32_t nq,
                                                  DBvh T, int upper, uint2* __restrict__ out, unsigned long long cap,
                                                  unsigned long long* counter, int* err, unsigned long long* visits) {
  const int lane = threadIdx.x & 31;
  const uint32_t t0 = (blockIdx.x * blockDim.x + threadIdx.x) * QPT;
  uint32_t qi[QPT];
  float4 b[QPT];
  int stack[QPT][TRAV_STACK];
  int sp[QPT], node[QPT];   // node: the next internal node to visit (register); only a second hit child is pushed
#pragma unroll
  for (int k = 0; k < QPT; k++) {
    const uint32_t t = t0 + k;
    sp[k] = 0; node[k] = -1; qi[k] = 0; b[k] = make_float4(0, 0, 0, 0);
    if (t < nq) {
      qi[k] = qorder ? qorder[q0 + t] : q0 + t;
      b[k] = qbb[qi[k]];
      node[k] = 0;
    }
  }
  const unsigned lt = (1u << lane) - 1;
  unsigned long long nvis = 0;
  for (;;) {
    bool any = false;
#pragma unroll
    for (int k = 0; k < QPT; k++) {
      if (node[k] < 0 && sp[k] > 0) node[k] = stack[k][--sp[k]];
      any = any || node[k] >= 0;
    }
    if (!__any_sync(0xffffffffu, any)) break;
    float4 lb[QPT], rb[QPT];
    int4 ch[QPT];
#pragma unroll
    for (int k = 0; k < QPT; k++)   // both loads first
      if (node[k] >= 0) {
        const BNode* np_ = T.nodes + node[k];
        lb[k] = __ldg(&np_->lb); rb[k] = __ldg(&np_->rb);
        ch[k] = __ldg(reinterpret_cast<const int4*>(&np_->l));
      }
    uint32_t hq[2 * QPT], hid[2 * QPT];
    int nh = 0;
#pragma unroll
    for (int k = 0; k < QPT; k++) {
      if (node[k] < 0) continue;
      nvis++;
      const bool hl = box_hit(lb[k], b[k]), hr = box_hit(rb[k], b[k]);
      int next = -1;
      if (hr) {
        if (ch[k].y < 0) { const uint32_t id = (uint32_t)~ch[k].y; if (!upper || id >= qi[k]) { hq[nh] = qi[k]; hid[nh] = id; nh++; } }
        else next = ch[k].y;
      }
      if (hl) {
        if (ch[k].x < 0) { const uint32_t id = (uint32_t)~ch[k].x; if (!upper || id >= qi[k]) { hq[nh] = qi[k]; hid[nh] = id; nh++; } }
        else {
          if (next >= 0) { if (sp[k] < TRAV_STACK) stack[k][sp[k]++] = next; else *err = 1; }
          next = ch[k].x;
        }
      }
      node[k] = next;
    }
    // warp-aggregated append: one atomic per warp step
    int x = nh;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const int tot = __shfl_sync(0xffffffffu, x, 31);
    if (tot) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(counter, (unsigned long long)tot);
      base = __shfl_sync(0xffffffffu, base, 0);
      const unsigned long long pos = base + (unsigned long long)(x - nh);
#pragma unroll
      for (int h = 0; h < 2 * QPT; h++)
        if (h < nh && pos + h < cap) out[pos + h] = make_uint2(hq[h], hid[h]);
    }
  }
  (void)lt;
  for (int o = 16; o > 0; o >>= 1) nvis += __shfl_xor_sync(0xffffffffu, nvis, o);
  if (lane == 0 && nvis) atomicAdd(visits, nvis);
}

uint64_t traverse(gsj_ctx* c, const float4* qbb, const uint32_t* qorder, uint32_t q0, uint32_t nq, const DBvh& T, int upper, uint2* out,
                  uint64_t cap) {
  if (nq == 0) return 0;
  unsigned long long* ctr = c->counters.as<unsigned long long>(8);
  int* err = reinterpret_cast<int*>(ctr + 1);
  GSJ_CK(cudaMemsetAsync(ctr, 0, 24, c->stream));
  k_traverse<<<grid_for((nq + QPT - 1) / QPT, 128), 128, 0, c->stream>>>(qbb, qorder, q0, nq, T, upper, out, cap, ctr, err, ctr + 2); c->launches++;
  GSJ_CK(cudaGetLastError());
  unsigned long long* h = c->h_counters.as<unsigned long long>(3);
  GSJ_CK(cudaMemcpyAsync(h, ctr, 24, cudaMemcpyDeviceToHost, c->stream));
  GSJ_CK(cudaStreamSynchronize(c->stream));
  if (reinterpret_cast<int*>(h + 1)[0]) throw Error(GSJ_ERR_CUDA, "traversal stack overflow");
  c->node_visits += h[2];
  return h[0];
}

}  // namespace gsj
