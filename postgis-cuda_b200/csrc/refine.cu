// Exact refinement of candidate pairs: ST_Intersects, intersection area (Green's theorem over the boundary
// pieces inside the other polygon, product-rule weights on shared boundaries) and DE-9IM evidence, one warp per
// pair. Restates the decisions of the reference's k_refine / edge_contrib_loc (engine/engine.cuh:333-636) with
// its lane ownership kept (lane l owns local edges l, l+32, ...; A's then B's; shfl_down tree 16..1), so the
// FP64 area and boundary-length sums have one fixed rounding order: bit-identical to the CPU oracle.
//
// Pairs whose local edge lists fit CAP run from shared memory; larger pairs are queued and re-run by
// k_refine_scratch with per-warp lists in global scratch (the same device code, so the same results).
//
// Two variants of the same pair routine (template flag F):
//  - plain (F = false): FP64 box tests, as the reference.
//  - filtered (F = true): the box rejection tests that dominate the inner loops are written as plain comparisons
//    (max(a, b) < x  <=>  a < x && b < x for finite values) instead of FP64 min/max, which on sm_100a issue on the
//    XU pipe - the pipe the plain kernel saturates (ncu: XU 77 % of peak, FP64 25 %). The same booleans, so every
//    decision and every FP64 value is unchanged. Containment probes are tested by the whole warp (crossing parity
//    is order-free).
#include "engine.h"
#include "pairkit.cuh"

namespace gsj {

constexpr int CAP = 128;                         // plain: local edges per polygon per warp in shared memory
constexpr int RB_WARPS = 4;                      // warps per block
constexpr size_t EDGE_BYTES = 4 * sizeof(double) + sizeof(uint32_t);
constexpr size_t LIST_BYTES = CAP * EDGE_BYTES;  // one list
constexpr size_t RB_SMEM = (size_t)RB_WARPS * 2 * LIST_BYTES;
constexpr int CAP_F = 128;                       // filtered: local edges per polygon per warp
constexpr size_t EDGE_BYTES_F = EDGE_BYTES;
constexpr size_t LIST_BYTES_F = CAP_F * EDGE_BYTES_F;
constexpr size_t RB_SMEM_F = (size_t)RB_WARPS * 2 * LIST_BYTES_F;

struct PairGeo { Box ov; double tol, eps_par, snap, cx, cy; };

// Candidate edge pairs of the filtered variant: every (i, j) of A's and B's local edges whose boxes come within
// 2 tol of each other - a superset of the pairs any box test of the pair routine keeps (those use tol or no pad).
// Built by one lane-balanced sweep over the na x nb grid (ballot compaction keeps (i, j) order); per-edge
// ranges: A edge i owns cp[sa[i] .. sa[i+1]), B edge j owns pj[(j ? sb[j-1] : 0) .. sb[j]) (entries in i order).
// Large grids are searched by buckets instead: NBK slabs along the overlap box's longer side, B's edges listed per
// slab (bl, boff), each lane scanning only its A edge's slabs and reporting a pair once, in the first slab both
// edges reach; the lane sorts its few candidates (at most LCAP) so the list keeps (i, j) order.
// Only the oversized pairs of the scratch kernel use the buckets: for the shared-memory bins the grid is faster.
constexpr int NBK = 16, LCAP = 32;
constexpr int GRID_MAX = 2048;   // scratch kernel: na x nb up to this: the grid sweep
// cap: entries of cp / pj; rec: a self pair's recorded contributions, one per A edge (the scratch kernel's B list)
struct FlatBuf { uint32_t* cp; uint16_t* pj; uint32_t* sa; uint32_t* sb; uint32_t* bl; uint32_t* boff; int cap, blcap; double* rec; };

__device__ __forceinline__ void warp_exscan(uint32_t* a, int n, int lane) {   // in place over a[0 .. n)
  uint32_t run = 0;
  for (int base = 0; base < n; base += 32) {
    const int t = base + lane;
    const uint32_t v = t < n ? a[t] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (t < n) a[t] = run + x - v;
    run += __shfl_sync(0xffffffffu, x, 31);
  }
  __syncwarp();
}

// Bucketed search (large grids): fills cp in (i, j) order with the per-edge counts in sa / sb and returns the
// number of candidates, or -1 when a bucket list or a lane's candidate buffer would overflow.
__device__ int bucket_candidates(const EList& LA, int na, const EList& LB, int nb, double pad, const Box& ov, const FlatBuf& fb, int lane) {
  const bool ax = (ov.x1 - ov.x0) >= (ov.y1 - ov.y0);
  const double o0 = ax ? ov.x0 : ov.y0, len = ax ? ov.x1 - ov.x0 : ov.y1 - ov.y0;
  const double inv = len > 0 ? NBK / len : 0.0;
  auto bk = [&](double v) {   // monotone in v
    const double t = (v - o0) * inv;
    return t < 1.0 ? 0 : (t >= (double)(NBK - 1) ? NBK - 1 : (int)t);
  };
  const unsigned lt = (1u << lane) - 1;
  if (lane <= NBK) fb.boff[lane] = 0;
  __syncwarp();
  for (int j = lane; j < nb; j += 32) {   // slab span of each B edge (kept in pj until the scatter)
    const double c0 = ax ? LB.x0[j] : LB.y0[j], c1 = ax ? LB.x1[j] : LB.y1[j];
    const int s0 = bk(c0 < c1 ? c0 : c1), s1 = bk(c0 < c1 ? c1 : c0);
    fb.pj[j] = (uint16_t)(s0 | (s1 << 8));
    for (int b2 = s0; b2 <= s1; b2++) atomicAdd(&fb.boff[b2], 1u);
  }
  __syncwarp();
  warp_exscan(fb.boff, NBK + 1, lane);
  if ((int)fb.boff[NBK] > fb.blcap) return -1;
  for (int b2 = 0; b2 < NBK; b2++) {   // stable lists: B edges of slab b2 in increasing j
    int run = 0;
    for (int j0 = 0; j0 < nb; j0 += 32) {
      const int j = j0 + lane;
      int s0 = 0;
      bool cov = false;
      if (j < nb) { const uint32_t sp = fb.pj[j]; s0 = (int)(sp & 0xFFu); cov = s0 <= b2 && b2 <= (int)(sp >> 8); }
      const unsigned m = __ballot_sync(0xffffffffu, cov);
      if (cov) fb.bl[fb.boff[b2] + run + __popc(m & lt)] = (uint32_t)j | ((uint32_t)s0 << 16);
      run += __popc(m);
    }
  }
  __syncwarp();
  int cnt = 0;
  for (int t0 = 0; t0 < na; t0 += 32) {
    const int i = t0 + lane;
    int ni = 0;
    uint16_t lc[LCAP];
    if (i < na) {
      const double px = LA.x0[i], py = LA.y0[i], qx = LA.x1[i], qy = LA.y1[i];
      const double ax0 = (px < qx ? px : qx) - pad, ax1 = (px < qx ? qx : px) + pad;
      const double ay0 = (py < qy ? py : qy) - pad, ay1 = (py < qy ? qy : py) + pad;
      const int s0 = bk(ax ? ax0 : ay0), s1 = bk(ax ? ax1 : ay1);
      for (int b2 = s0; b2 <= s1; b2++)
        for (uint32_t e = fb.boff[b2]; e < fb.boff[b2 + 1]; e++) {
          const uint32_t v = fb.bl[e];
          const int j = (int)(v & 0xFFFFu), sj = (int)(v >> 16);
          if ((sj > s0 ? sj : s0) != b2) continue;   // the pair belongs to the first slab both edges reach
          if (out_cmp(LB.x0[j], LB.y0[j], LB.x1[j], LB.y1[j], ax0, ay0, ax1, ay1)) continue;
          if (ni < LCAP) lc[ni] = (uint16_t)j;
          ni++;
        }
      if (ni <= LCAP)
        for (int u = 1; u < ni; u++) {
          const uint16_t v = lc[u];
          int w = u - 1;
          while (w >= 0 && lc[w] > v) { lc[w + 1] = lc[w]; w--; }
          lc[w + 1] = v;
        }
    }
    if (__any_sync(0xffffffffu, ni > LCAP)) return -1;
    int x = ni;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    const int off = cnt + x - ni;
    if (i < na) {
      fb.sa[i] = (uint32_t)ni;
      for (int k = 0; k < ni; k++) {
        if (off + k < fb.cap) fb.cp[off + k] = (uint32_t)i | ((uint32_t)lc[k] << 16);
        atomicAdd(&fb.sb[lc[k]], 1u);
      }
    }
    cnt += __shfl_sync(0xffffffffu, x, 31);
  }
  __syncwarp();
  return cnt;
}

// returns the number of candidate pairs (> fb.cap: the lists were not kept)
template <bool BUCKETS>
__device__ int flat_candidates(const EList& LA, int na, const EList& LB, int nb, double pad, const Box& ov, const FlatBuf& fb, int lane) {
  for (int t = lane; t <= na; t += 32) fb.sa[t] = 0;
  for (int t = lane; t <= nb; t += 32) fb.sb[t] = 0;
  __syncwarp();
  if (na == 0 || nb == 0) return 0;
  const unsigned lt = (1u << lane) - 1;
  const int total = na * nb;
  int cnt = -1;
  if (BUCKETS && total > GRID_MAX) {
    cnt = bucket_candidates(LA, na, LB, nb, pad, ov, fb, lane);
    if (cnt < 0) {   // overflowed: count afresh with the grid
      for (int t = lane; t <= na; t += 32) fb.sa[t] = 0;
      for (int t = lane; t <= nb; t += 32) fb.sb[t] = 0;
      __syncwarp();
    }
  }
  if (cnt < 0) {
  const int qi = 32 / nb, qj = 32 % nb;
  int i = lane / nb, j = lane % nb;
  cnt = 0;
  for (int base = 0; base < total; base += 32) {
    bool keep = false;
    if (base + lane < total) {
      const double px = LA.x0[i], py = LA.y0[i], qx = LA.x1[i], qy = LA.y1[i];
      const double ax0 = (px < qx ? px : qx) - pad, ax1 = (px < qx ? qx : px) + pad;
      const double ay0 = (py < qy ? py : qy) - pad, ay1 = (py < qy ? qy : py) + pad;
      keep = !out_cmp(LB.x0[j], LB.y0[j], LB.x1[j], LB.y1[j], ax0, ay0, ax1, ay1);
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    const int pos = cnt + __popc(m & lt);
    if (keep && pos < fb.cap) {
      fb.cp[pos] = (uint32_t)i | ((uint32_t)j << 16);
      atomicAdd(&fb.sa[i], 1u);
      atomicAdd(&fb.sb[j], 1u);
    }
    cnt += __popc(m);
    i += qi; j += qj;
    if (j >= nb) { j -= nb; i++; }
  }
  }
  if (cnt > fb.cap) return cnt;
  __syncwarp();
  warp_exscan(fb.sa, na + 1, lane);
  warp_exscan(fb.sb, nb + 1, lane);
  // stable scatter by j: entries of one B edge keep their (increasing i) order
  for (int base = 0; base < cnt; base += 32) {
    const int e = base + lane;
    const bool v = e < cnt;
    const uint32_t jj = v ? (fb.cp[e] >> 16) : 0xFFFFFu;
    const unsigned peers = __match_any_sync(0xffffffffu, jj);
    if (v) fb.pj[fb.sb[jj] + __popc(peers & lt)] = (uint16_t)e;
    __syncwarp();
    if (v && (peers & lt) == 0) fb.sb[jj] += __popc(peers);
    __syncwarp();
  }
  return cnt;
}

// Candidate edge pairs of the shared-memory kernel as bit masks: row i holds the B edges j whose boxes come within
// 2 tol of A edge i (the flat lists' test and set), column j the A edges i. A row visits its j, a column its i, in
// increasing order by walking set bits, which is the order of the flat lists; the masks never overflow (up to
// CAP_F edges per side) and cost no counting, scans or scatter. Word-major: word w of row i at rm[w * CAP_F + i].
constexpr int MASK_WORDS = CAP_F / 32;
struct MaskBuf { uint32_t* rm; uint32_t* cm; };
constexpr size_t MASK_BYTES = 2 * (size_t)MASK_WORDS * CAP_F * sizeof(uint32_t);

// one stage of the in-register 32 x 32 bit transpose: lanes l and l ^ s swap the off-diagonal s x s blocks
__device__ __forceinline__ uint32_t transpose_stage(uint32_t x, int s, uint32_t m, int lane) {
  const uint32_t p = __shfl_xor_sync(0xffffffffu, x, s);
  return (lane & s) ? ((x & ~m) | ((p >> s) & m)) : ((x & m) | ((p << s) & ~m));
}
// lane l holds row l of a 32 x 32 bit matrix (bit j = M[l][j]); returns column l (bit i = M[i][l])
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, int lane) {
  x = transpose_stage(x, 16, 0x0000FFFFu, lane);
  x = transpose_stage(x, 8, 0x00FF00FFu, lane);
  x = transpose_stage(x, 4, 0x0F0F0F0Fu, lane);
  x = transpose_stage(x, 2, 0x33333333u, lane);
  return transpose_stage(x, 1, 0x55555555u, lane);
}

// lane i (per 32 A edges) keeps its padded box in registers and tests every B edge j, read once for the whole warp
// (a shared-memory broadcast); each 32 x 32 block of rows is transposed into columns by shuffles (COLS; the self
// bin reads rows only). STRIDE: rows per mask word plane (the bin's list capacity).
template <int STRIDE = CAP_F, bool COLS = true>
__device__ void mask_candidates(const EList& LA, int na, const EList& LB, int nb, double pad, const MaskBuf& mb, int lane) {
  const int nbw = (nb + 31) >> 5;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  for (int ic = 0; ic < na; ic += 32) {
    const int i = ic + lane;
    double ax0 = inf, ay0 = inf, ax1 = -inf, ay1 = -inf;   // lanes past the end keep an empty box: no bits
    if (i < na) {
      const double px = LA.x0[i], py = LA.y0[i], qx = LA.x1[i], qy = LA.y1[i];
      ax0 = (px < qx ? px : qx) - pad; ax1 = (px < qx ? qx : px) + pad;
      ay0 = (py < qy ? py : qy) - pad; ay1 = (py < qy ? qy : py) + pad;
    }
    for (int w = 0; w < nbw; w++) {
      const int j0 = w << 5, j1 = min(nb, j0 + 32);
      uint32_t bits = 0;
      for (int j = j0; j < j1; j++)
        bits |= (out_cmp(LB.x0[j], LB.y0[j], LB.x1[j], LB.y1[j], ax0, ay0, ax1, ay1) ? 0u : 1u) << (j - j0);
      if (i < na) mb.rm[w * STRIDE + i] = bits;
      if constexpr (COLS) {
        const uint32_t col = warp_transpose32(bits, lane);
        if (j0 + lane < nb) mb.cm[(ic >> 5) * STRIDE + j0 + lane] = col;
      }
    }
  }
  __syncwarp();
}

// Green's-theorem contribution of edge p->q within the other polygon + relate lengths (engine.cuh:416-515).
// each_k(visit) calls visit(k) for the other polygon's local edges k in increasing order: all of them, or only
// those of a candidate list that holds every k passing the box test below (the same visits, the same results).
template <bool F, bool S32, class EachK>
__device__ double edge_contrib_k(double px, double py, double qx, double qy, const EList& L, int cnt, bool in_c, const PairGeo& G, bool real,
                                 double* l_in, double* l_on, uint32_t* bits, uint32_t cut, EachK&& each_k) {
  const double dx = qx - px, dy = qy - py;
  const double len2 = dx * dx + dy * dy;
  if (len2 == 0) return 0.0;
  const double tol = G.tol;
  const double tol2len2 = tol * tol * len2, eps2 = G.eps_par * G.eps_par;
  double ts[MAXS]; int ns = 0;
  double ol0[MAXO], ol1[MAXO]; bool osame[MAXO]; int oidx[MAXO]; int no = 0;
  ts[ns++] = 0; ts[ns++] = 1;
  const double bx0 = fmin(px, qx) - tol, bx1 = fmax(px, qx) + tol, by0 = fmin(py, qy) - tol, by1 = fmax(py, qy) + tol;
  const double snap2 = G.snap * G.snap;
  auto visit = [&](int k) {
    const double ex0 = L.x0[k], ey0 = L.y0[k], ex1 = L.x1[k], ey1 = L.y1[k];
    if (F ? out_cmp(ex0, ey0, ex1, ey1, bx0, by0, bx1, by1)
          : (fmax(ex0, ex1) < bx0 || fmin(ex0, ex1) > bx1 || fmax(ey0, ey1) < by0 || fmin(ey0, ey1) > by1)) return false;
    const uint32_t efl = L.fl[k];
    const double fx = ex1 - ex0, fy = ey1 - ey0;
    const double r = dx * fy - dy * fx;
    const double flen2 = fx * fx + fy * fy;
    const double c0 = orient(px, py, qx, qy, ex0, ey0), c1 = orient(px, py, qx, qy, ex1, ey1);
    bool col = (c0 * c0 <= snap2 * len2 || ((efl & 2u) && c0 * c0 <= tol2len2)) && (c1 * c1 <= snap2 * len2 || ((efl & 4u) && c1 * c1 <= tol2len2));
    if (!col && flen2 > 0) {
      const double g0 = orient(ex0, ey0, ex1, ey1, px, py), g1 = orient(ex0, ey0, ex1, ey1, qx, qy), tf = tol * tol * flen2;
      col = (g0 * g0 <= snap2 * flen2 || ((cut & 2u) && g0 * g0 <= tf)) && (g1 * g1 <= snap2 * flen2 || ((cut & 4u) && g1 * g1 <= tf));
    }
    if (col) {
      double tc = (ex0 - px) * dx + (ey0 - py) * dy, te = (ex1 - px) * dx + (ey1 - py) * dy;
      if (F) {   // n / len2 is n for n = +-0 and exactly 1 for n = len2 (> 0): a coincident edge's ends need no division
        tc = tc == 0.0 ? tc : (tc == len2 ? 1.0 : tc / len2);
        te = te == 0.0 ? te : (te == len2 ? 1.0 : te / len2);
      } else {
        tc = tc / len2; te = te / len2;
      }
      const double lo = fmax((double)0, fmin(tc, te)), hi = fmin((double)1, fmax(tc, te));
      if (hi > lo) {
        if (lo > 0 && ns < MAXS) ts[ns++] = lo;
        if (hi < 1 && ns < MAXS) ts[ns++] = hi;
        if (no < MAXO) { ol0[no] = lo; ol1[no] = hi; osame[no] = (dx * fx + dy * fy) > 0; oidx[no] = k; no++; }
      }
    } else if (r * r > eps2 * len2 * flen2) {
      const double wx = ex0 - px, wy = ey0 - py;
      const double tn = wx * fy - wy * fx;
      if (r > 0 ? (tn <= 0 || tn >= r) : (tn >= 0 || tn <= r)) return false;
      const double t = tn / r, u = (wx * dy - wy * dx) / r;
      const double du = tol / (flen2 > 0 ? sqrt(flen2) : (double)1);
      if (u >= -du && u <= 1 + du && ns < MAXS) ts[ns++] = t;
    }
    return false;
  };
  each_k(visit);
  for (int a = 1; a < ns; a++) { double v = ts[a]; int b = a - 1; while (b >= 0 && ts[b] > v) { ts[b + 1] = ts[b]; b--; } ts[b + 1] = v; }
  double acc = 0.0;
  for (int k = 0; k + 1 < ns; k++) {
    const double t0 = ts[k], t1 = ts[k + 1];
    if (!(t1 > t0)) continue;
    const double tm = (double)0.5 * (t0 + t1);
    const double mx = px + dx * tm, my = py + dy * tm;
    const bool in_ov = mx >= G.ov.x0 && mx <= G.ov.x1 && my >= G.ov.y0 && my <= G.ov.y1;
    int net = 0, first = -1, net_real = 0, n_real = 0;
    for (int o = 0; o < no; o++)
      if (tm > ol0[o] && tm < ol1[o]) {
        const int sgn = osame[o] ? 1 : -1;
        net += sgn; if (first < 0) first = o;
        if (!(L.fl[oidx[o]] & 1u)) { net_real += sgn; n_real++; }
      }
    // the inside test of the midpoint, evaluated once and only where a branch below reads it
    const bool lens = l_in && real;
    const bool need = first < 0 || (net != 1 && net != -1) || (lens && net_real == 0 && !(n_real == 0 && (net == 1 || net == -1)));
    const int vin = (need && in_ov && inside_from_c<F, S32>(L, cnt, G.cx, G.cy, in_c, mx, my)) ? 1 : 0;
    if (lens) {
      const double seg = sqrt(len2) * (t1 - t0);
      if (net_real != 0) { *l_on += seg; *bits |= (net_real > 0 ? REL_COIN_SAME : REL_COIN_OPP) | REL_TOUCH; }
      else if (n_real == 0 && (net == 1 || net == -1)) *l_in += 0.5 * seg;
      else if (vin) *l_in += seg;
    }
    double w;
    if (first < 0) w = vin ? 1.0 : 0.0;
    else if (net == 1 || net == -1) w = 0.5;
    else if (net == 0) w = vin ? 1.0 : 0.0;
    else {
      const int fo = oidx[first];
      const bool sb = left_of(L.x0[fo], L.y0[fo], L.x1[fo], L.y1[fo], mx, my);
      const bool m_left = osame[first] ? sb : !sb;
      int other = m_left ? vin - net : vin + net;
      other = other < 0 ? 0 : (other > 1 ? 1 : other);
      w = 0.5 * (vin + other);
    }
    if (w != 0.0) {
      const double ax = px + dx * t0 - G.cx, ay = py + dy * t0 - G.cy, bx = px + dx * t1 - G.cx, by = py + dy * t1 - G.cy;
      acc += w * (double)(ax * by - ay * bx);
    }
  }
  return acc;
}

template <bool F>
__device__ __forceinline__ double edge_contrib(double px, double py, double qx, double qy, const EList& L, int cnt, bool in_c, const PairGeo& G,
                                               bool real, double* l_in, double* l_on, uint32_t* bits, uint32_t cut) {
  return edge_contrib_k<F, false>(px, py, qx, qy, L, cnt, in_c, G, real, l_in, l_on, bits, cut, [&](auto&& visit) {
    for (int k = 0; k < cnt; k++) visit(k);
  });
}

__device__ __forceinline__ double pair_snap(double2 oa, double2 ea) {   // engine.cuh:524-527
  double m = fmax(fmax(fabs(oa.x), fabs(oa.x + ea.x)), fmax(fabs(oa.y), fabs(oa.y + ea.y)));
  return 0.5 * (nextafter(m, INFINITY) - m);
}

// One pair, whole warp. Returns false when a local list exceeded cap (nothing written).
// MASK (the filtered shared-memory kernel): candidate edge pairs as bit masks (mb).
// FLAT (the filtered scratch kernel): candidate lists in global scratch; a pair whose list would exceed fb->cap is
// handed back (false) and runs with the full sweeps.
// SELF (> 0, filtered shared-memory bin only): the pair is a geometry with itself in one layer; the caller passes
// one list of SELF edges as both LA and LB. B's gather and B's contribution pass would repeat A's exactly (the same
// edges in the same frame, the same candidates in the same order, so the same values): A's pass runs once and each
// lane adds its recorded values a second time, in the same order, which is the sum the two passes make.
template <bool F, bool FLAT = false, bool BUCKETS = false, bool MASK = false, bool S32 = false, int SELF = 0>
__device__ bool refine_pair_t(const DLayer& P, const DLayer& R, uint32_t a, uint32_t b, const RefineArgs& rp, EList LA, EList LB, int cap,
                              int lane, uint8_t& o_flag, double& o_area, double4& o_ev, uint32_t& o_evb, const FlatBuf* fb = nullptr,
                              const MaskBuf* mb = nullptr, unsigned long long* ep = nullptr) {
  const double2 oa = P.origin[a], ob = R.origin[b], ea = P.ext[a], eb = R.ext[b];
  const double sx = ob.x - oa.x, sy = ob.y - oa.y;
  const double pad = 4.0 * fmax(rp.tol_abs, (double)rp.tol_rel * fmax(fmax(ea.x, ea.y), fmax(eb.x, eb.y)));
  PairGeo G;
  G.ov = Box{fmax(0.0, sx) - pad, fmax(0.0, sy) - pad, fmin(ea.x, sx + eb.x) + pad, fmin(ea.y, sy + eb.y) + pad};
  const Frame A = frame_of(P, a, oa.x, oa.y), B = frame_of(R, b, oa.x, oa.y);
  G.tol = fmax(rp.tol_abs, (double)rp.tol_rel * fmax(G.ov.x1 - G.ov.x0, G.ov.y1 - G.ov.y0));
  G.eps_par = rp.eps_par;
  G.snap = rp.snap_half_ulp ? pair_snap(oa, ea) : 0.0;
  G.cx = (double)(G.ov.x0 + 0.381966 * (G.ov.x1 - G.ov.x0));
  G.cy = (double)(G.ov.y0 + 0.414213 * (G.ov.y1 - G.ov.y0));
  int na = 0, nb = 0;
  bool inB_c = false, inA_c = false;
  for (int side = 0; side < (SELF ? 1 : 2); side++) {   // one inlined copy of the gather
    bool in = false;
    // MASK: the containment parity of the probe point c is taken in the gather's pass over each polygon's edges
    const int n = collect<F, MASK, S32>(side ? B : A, G.ov, side ? LB : LA, cap, lane, G.cx, G.cy, &in);
    if (side) { nb = n; inB_c = in; } else { na = n; inA_c = in; }
  }
  if constexpr (SELF > 0) { nb = na; inB_c = inA_c; }
  if (na > cap || nb > cap) return false;
  __syncwarp();
  constexpr int MW = SELF ? SELF / 32 : MASK_WORDS, MS = SELF ? SELF : CAP_F;   // mask words per row, row stride
  int ncp = -1;   // candidate edge pairs (FLAT); -1: sweep every edge pair
  if constexpr (MASK) {
    mask_candidates<MS, SELF == 0>(LA, na, LB, nb, 2.0 * G.tol, *mb, lane);
  } else if constexpr (FLAT) {
    ncp = flat_candidates<BUCKETS>(LA, na, LB, nb, 2.0 * G.tol, G.ov, *fb, lane);
    if (ncp > fb->cap) return false;
  }
  // boundary contact
  bool hit = false, hit_any = false;
  auto seg_loop = [&](int i) {
    const double px0 = LA.x0[i], py0 = LA.y0[i], px1 = LA.x1[i], py1 = LA.y1[i];
    const uint32_t fa = LA.fl[i];
    const double ax0 = fmin(px0, px1), ax1 = fmax(px0, px1), ay0 = fmin(py0, py1), ay1 = fmax(py0, py1);
    auto test = [&](int j) {
      const double qx0 = LB.x0[j], qy0 = LB.y0[j], qx1 = LB.x1[j], qy1 = LB.y1[j];
      if (F ? out_cmp(qx0, qy0, qx1, qy1, ax0, ay0, ax1, ay1)
            : (fmax(qx0, qx1) < ax0 || fmin(qx0, qx1) > ax1 || fmax(qy0, qy1) < ay0 || fmin(qy0, qy1) > ay1)) return false;
      if (seg_isect(px0, py0, px1, py1, qx0, qy0, qx1, qy1)) {
        hit_any = true;
        if (!((fa | LB.fl[j]) & 1u)) { hit = true; return true; }
      }
      return false;
    };
    for (int j = 0; j < nb; j++) if (test(j)) break;
  };
  if constexpr (MASK) {
    // each lane walks its A edge's candidates, one per round; the warp stops at the first real contact
    const int nbw = (nb + 31) >> 5;
    for (int ic = 0; ic < na && !hit; ic += 32) {
      const int i = ic + lane;
      uint32_t w[MW];
      #pragma unroll
      for (int q = 0; q < MW; q++) w[q] = (i < na && q < nbw) ? mb->rm[q * MS + i] : 0u;
      double px0 = 0, py0 = 0, px1 = 0, py1 = 0;
      uint32_t fa = 0;
      if (i < na) { px0 = LA.x0[i]; py0 = LA.y0[i]; px1 = LA.x1[i]; py1 = LA.y1[i]; fa = LA.fl[i]; }
      const double ax0 = px0 < px1 ? px0 : px1, ax1 = px0 < px1 ? px1 : px0, ay0 = py0 < py1 ? py0 : py1, ay1 = py0 < py1 ? py1 : py0;
      for (;;) {
        int j = -1;
        #pragma unroll
        for (int q = 0; q < MW; q++)
          if (j < 0 && w[q]) { j = (q << 5) + __ffs(w[q]) - 1; w[q] &= w[q] - 1; }
        if (!__any_sync(0xffffffffu, j >= 0)) break;
        if (j >= 0) {
          const double qx0 = LB.x0[j], qy0 = LB.y0[j], qx1 = LB.x1[j], qy1 = LB.y1[j];
          if (!out_cmp(qx0, qy0, qx1, qy1, ax0, ay0, ax1, ay1) &&
              (S32 ? seg_isect32(px0, py0, px1, py1, qx0, qy0, qx1, qy1) : seg_isect(px0, py0, px1, py1, qx0, qy0, qx1, qy1))) {
            hit_any = true;
            if (!((fa | LB.fl[j]) & 1u)) hit = true;
          }
        }
        if (__any_sync(0xffffffffu, hit)) { hit = true; break; }
      }
    }
  } else if constexpr (FLAT) {
    // one candidate per lane; the warp stops at the first real contact (hit_any is then implied)
    for (int base = 0; base < ncp; base += 32) {
      const int e = base + lane;
      if (e < ncp) {
        const uint32_t c = fb->cp[e];
        const int i = (int)(c & 0xFFFFu), j = (int)(c >> 16);
        const double px0 = LA.x0[i], py0 = LA.y0[i], px1 = LA.x1[i], py1 = LA.y1[i];
        const double qx0 = LB.x0[j], qy0 = LB.y0[j], qx1 = LB.x1[j], qy1 = LB.y1[j];
        const double ax0 = px0 < px1 ? px0 : px1, ax1 = px0 < px1 ? px1 : px0, ay0 = py0 < py1 ? py0 : py1, ay1 = py0 < py1 ? py1 : py0;
        if (!out_cmp(qx0, qy0, qx1, qy1, ax0, ay0, ax1, ay1) && seg_isect(px0, py0, px1, py1, qx0, qy0, qx1, qy1)) {
          hit_any = true;
          if (!((LA.fl[i] | LB.fl[j]) & 1u)) hit = true;
        }
      }
      if (__any_sync(0xffffffffu, hit)) { hit = true; break; }
    }
  } else {
    for (int i = lane; i < na && !hit; i += 32) seg_loop(i);
  }
  hit = __any_sync(0xffffffffu, hit);
  hit_any = __any_sync(0xffffffffu, hit_any || hit);
  const bool rtouch = hit;
  if (!MASK && (!hit || rp.want_area || rp.want_relate))
    for (int side = 0; side < 2; side++) {
      const bool in = pip_full_warp(side ? A : B, G.cx, G.cy, lane);
      if (side) inA_c = in; else inB_c = in;
    }
  bool contain_any = false;
  if (!hit) {
    // no real boundary contact: intersects iff a real-edge vertex of one lies inside the other (engine.cuh:577-594)
    bool h = false, ha = false;
    if constexpr (F) {
      // one probe at a time, the warp splitting the other polygon's edges (crossing parity is order-free)
      for (int side = 0; side < 2 && !h; side++) {
        const Frame& S = side ? B : A;
        const DLayer& SL = side ? R : P;
        const EList& LO = side ? LA : LB;
        const int no_ = side ? na : nb;
        const bool inc = side ? inA_c : inB_c;
        for (uint32_t r = S.r0; r < S.r1 && !h; r++) {
          double x, y; const bool real = probe_vertex(S, r, x, y);
          if (!real) S.v(SL.rvo[r], x, y);
          if (x >= G.ov.x0 && x <= G.ov.x1 && y >= G.ov.y0 && y <= G.ov.y1 && inside_from_c_warp<S32>(LO, no_, G.cx, G.cy, inc, x, y, lane)) {
            ha = true; h = real;
          }
        }
      }
      hit = h;
      contain_any = ha;
    } else {
      for (uint32_t r = A.r0 + lane; r < A.r1 && !h; r += 32) {
        double x, y; const bool real = probe_vertex(A, r, x, y);
        if (!real) A.v(P.rvo[r], x, y);
        if (x >= G.ov.x0 && x <= G.ov.x1 && y >= G.ov.y0 && y <= G.ov.y1 && inside_from_c<F>(LB, nb, G.cx, G.cy, inB_c, x, y)) { ha = true; h = real; }
      }
      for (uint32_t r = B.r0 + lane; r < B.r1 && !h; r += 32) {
        double x, y; const bool real = probe_vertex(B, r, x, y);
        if (!real) B.v(R.rvo[r], x, y);
        if (x >= G.ov.x0 && x <= G.ov.x1 && y >= G.ov.y0 && y <= G.ov.y1 && inside_from_c<F>(LA, na, G.cx, G.cy, inA_c, x, y)) { ha = true; h = real; }
      }
      hit = __any_sync(0xffffffffu, h);
      contain_any = __any_sync(0xffffffffu, ha);
    }
  }
  double ar = 0.0; double4 e4 = make_double4(0, 0, 0, 0); uint32_t eb4 = 0;
  if ((hit || hit_any || contain_any) && (rp.want_area || rp.want_relate)) {
    double s2 = 0.0, ai = 0, ao = 0, bi = 0, bo = 0;
    uint32_t bits = rtouch ? REL_TOUCH : 0;
    const bool rel = rp.want_relate != 0;
    if constexpr (MASK && SELF > 0) {   // A's pass once, then each lane's recorded values added again in order
      const int nbw = (nb + 31) >> 5;
      double rec[MW];
      double lin = 0.0, lon = 0.0;
      int k = 0;
      for (int i = lane; i < na; i += 32, k++) {
        const uint32_t f = LA.fl[i];
        rec[k] = edge_contrib_k<F, S32>(LA.x0[i], LA.y0[i], LA.x1[i], LA.y1[i], LB, nb, inB_c, G, !(f & 1u), rel ? &lin : nullptr, &lon, &bits, f,
                                   [&](auto&& visit) {
                                     for (int q = 0; q < nbw; q++)
                                       for (uint32_t m = mb->rm[q * MS + i]; m; m &= m - 1) visit((q << 5) + __ffs(m) - 1);
                                   });
        s2 += rec[k];
      }
      for (int q = 0; q < k; q++) s2 += rec[q];
      ai = bi = lin; ao = bo = lon;
    } else if constexpr (MASK) {   // visit only each edge's candidates, in increasing order, by walking the set bits
      const int nbw = (nb + 31) >> 5, naw = (na + 31) >> 5;
      for (int pass = 0; pass < 2; pass++) {
        const EList& LS = pass ? LB : LA;
        const EList& LO = pass ? LA : LB;
        const int nself = pass ? nb : na, nother = pass ? na : nb, nw = pass ? naw : nbw;
        const uint32_t* mrow = pass ? mb->cm : mb->rm;
        const bool inc = pass ? inA_c : inB_c;
        double lin = 0.0, lon = 0.0;   // this pass's lengths (each starts from 0, so the sums are the same)
        for (int i = lane; i < nself; i += 32) {
          const uint32_t f = LS.fl[i];
          s2 += edge_contrib_k<F, S32>(LS.x0[i], LS.y0[i], LS.x1[i], LS.y1[i], LO, nother, inc, G, !(f & 1u), rel ? &lin : nullptr, &lon, &bits, f,
                                  [&](auto&& visit) {
                                    for (int q = 0; q < nw; q++)
                                      for (uint32_t m = mrow[q * CAP_F + i]; m; m &= m - 1) visit((q << 5) + __ffs(m) - 1);
                                  });
        }
        if (pass) { bi = lin; bo = lon; } else { ai = lin; ao = lon; }
      }
    } else if constexpr (FLAT && SELF > 0) {   // the self pair's A pass, recorded per edge, then added again in order
      const uint32_t* cp = fb->cp;
      double lin = 0.0, lon = 0.0;
      for (int i = lane; i < na; i += 32) {
        const uint32_t f = LA.fl[i];
        const int r0 = (int)fb->sa[i], r1 = (int)fb->sa[i + 1];
        const double v = edge_contrib_k<F, S32>(LA.x0[i], LA.y0[i], LA.x1[i], LA.y1[i], LB, nb, inB_c, G, !(f & 1u), rel ? &lin : nullptr, &lon, &bits, f,
                                           [&](auto&& visit) {
                                             for (int e = r0; e < r1; e++) visit((int)(cp[e] >> 16));
                                           });
        fb->rec[i] = v;
        s2 += v;
      }
      for (int i = lane; i < na; i += 32) s2 += fb->rec[i];
      ai = bi = lin; ao = bo = lon;
    } else if constexpr (FLAT) {   // visit only each edge's candidates, in the same increasing order; one call site for both passes
      const uint32_t* cp = fb->cp;
      const uint16_t* pj = fb->pj;
      for (int pass = 0; pass < 2; pass++) {
        const EList& LS = pass ? LB : LA;
        const EList& LO = pass ? LA : LB;
        const int nself = pass ? nb : na, nother = pass ? na : nb;
        const bool inc = pass ? inA_c : inB_c;
        double lin = 0.0, lon = 0.0;   // this pass's lengths (each starts from 0, so the sums are the same)
        for (int i = lane; i < nself; i += 32) {
          const uint32_t f = LS.fl[i];
          const int r0 = pass ? (i ? (int)fb->sb[i - 1] : 0) : (int)fb->sa[i];
          const int r1 = pass ? (int)fb->sb[i] : (int)fb->sa[i + 1];
          s2 += edge_contrib_k<F, S32>(LS.x0[i], LS.y0[i], LS.x1[i], LS.y1[i], LO, nother, inc, G, !(f & 1u), rel ? &lin : nullptr, &lon, &bits, f,
                                  [&](auto&& visit) {
                                    for (int e = r0; e < r1; e++) visit(pass ? (int)(cp[pj[e]] & 0xFFFFu) : (int)(cp[e] >> 16));
                                  });
        }
        if (pass) { bi = lin; bo = lon; } else { ai = lin; ao = lon; }
      }
    } else {
      for (int i = lane; i < na; i += 32) {
        const uint32_t f = LA.fl[i];
        s2 += edge_contrib<F>(LA.x0[i], LA.y0[i], LA.x1[i], LA.y1[i], LB, nb, inB_c, G, !(f & 1u), rel ? &ai : nullptr, &ao, &bits, f);
      }
      for (int i = lane; i < nb; i += 32) {
        const uint32_t f = LB.fl[i];
        s2 += edge_contrib<F>(LB.x0[i], LB.y0[i], LB.x1[i], LB.y1[i], LA, na, inA_c, G, !(f & 1u), rel ? &bi : nullptr, &bo, &bits, f);
      }
    }
    s2 = warp_sum(s2); ai = warp_sum(ai); ao = warp_sum(ao); bi = warp_sum(bi); bo = warp_sum(bo);
    ar = 0.5 * s2;
    e4 = make_double4(ai, ao, bi, bo);
    eb4 = __reduce_or_sync(0xffffffffu, bits);
  } else if (rtouch) eb4 = REL_TOUCH;
  const bool ev_any = e4.x != 0 || e4.y != 0 || e4.z != 0 || e4.w != 0;
  o_flag = hit ? 1 : ((ar != 0.0 || ev_any) ? 2 : 0);
  o_area = ar; o_ev = e4; o_evb = eb4;
  if (ep && lane == 0) *ep += (unsigned long long)na * (unsigned long long)nb;   // local edge pairs: the refinement's work unit
  return true;
}

// the plain routine, callable from other translation units (the allocation-free entry point)
__device__ bool refine_pair(const DLayer& P, const DLayer& R, uint32_t a, uint32_t b, const RefineArgs& rp, EList LA, EList LB, int cap, int lane,
                            uint8_t& o_flag, double& o_area, double4& o_ev, uint32_t& o_evb) {
  return refine_pair_t<false>(P, R, a, b, rp, LA, LB, cap, lane, o_flag, o_area, o_ev, o_evb);
}

template <bool F> struct Cfg;
template <> struct Cfg<false> { static constexpr int cap = CAP; static constexpr size_t list = LIST_BYTES, smem = RB_SMEM, edge = EDGE_BYTES; static constexpr int minb = 3; };
template <> struct Cfg<true> { static constexpr int cap = CAP_F; static constexpr size_t list = LIST_BYTES_F, smem = RB_SMEM_F + RB_WARPS * MASK_BYTES, edge = EDGE_BYTES_F; static constexpr int minb = 4; };

template <bool F>
__device__ __forceinline__ EList carve_t(unsigned char* base, int cap) { return F ? carve_f(base, cap) : carve(base, cap); }

// S32 (filtered only): the contact test's and the gather's orientation signs through the certified FP32 filter
template <bool F, bool S32 = false>
__global__ void __launch_bounds__(RB_WARPS * 32, Cfg<F>::minb) k_refine(DLayer P, DLayer R, const uint2* __restrict__ pairs, uint64_t np,
                                                                        RefineArgs rp, uint8_t* flag, double* area, double4* ev, uint32_t* evb,
                                                                        uint32_t* heavy, unsigned long long* nheavy, unsigned long long* next,
                                                                        unsigned long long* epairs, int run, int runs, int bin_cap,
                                                                        int skip_self) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned long long s_ep[RB_WARPS];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane == 0) s_ep[wib] = 0;
  __syncwarp();
  EList LA = carve_t<F>(smem + (size_t)wib * 2 * Cfg<F>::list, Cfg<F>::cap);
  EList LB = carve_t<F>(smem + (size_t)wib * 2 * Cfg<F>::list + Cfg<F>::list, Cfg<F>::cap);
  MaskBuf mbuf{nullptr, nullptr};
  if constexpr (F) {   // after the lists of all warps: row masks, then column masks
    unsigned char* mbase = smem + (size_t)RB_WARPS * 2 * Cfg<F>::list + (size_t)wib * MASK_BYTES;
    mbuf.rm = reinterpret_cast<uint32_t*>(mbase);
    mbuf.cm = mbuf.rm + MASK_WORDS * CAP_F;
  }
  auto one = [&](uint64_t p) {
    const uint2 pr = pairs[p];
    if (skip_self && pr.x == pr.y) return;   // a geometry with itself: the self bin's
    uint8_t f; double ar; double4 e4; uint32_t b4;
    const bool ok = refine_pair_t<F, false, false, F, S32>(P, R, pr.x, pr.y, rp, LA, LB, bin_cap, lane, f, ar, e4, b4, nullptr, &mbuf, &s_ep[wib]);
    if (lane == 0) {
      if (!ok) { heavy[atomicAdd(nheavy, 1ull)] = (uint32_t)p; flag[p] = 0; }
      else {
        flag[p] = f;
        if (area) area[p] = ar;
        if (ev) { ev[p] = e4; evb[p] = b4; }
      }
    }
    __syncwarp();
  };
  if constexpr (F) {
    // warps take runs of `run` consecutive pairs (shared probe geometry) from a counter, at most `runs` runs each:
    // the grid is sized to cover every pair that way, and bounded block lifetimes let the kernels of other
    // streams (higher-priority requests) take SMs as blocks retire
    for (int k = 0; k < runs; k++) {
      unsigned long long p0 = 0;
      if (lane == 0) p0 = atomicAdd(next, (unsigned long long)run);
      p0 = __shfl_sync(0xffffffffu, p0, 0);
      if (p0 >= np) break;
      const uint64_t p1 = p0 + run < np ? p0 + run : np;
      for (uint64_t p = p0; p < p1; p++) one(p);
    }
  } else {
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t p = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw) one(p);
  }
  __syncwarp();
  if (lane == 0 && s_ep[wib]) atomicAdd(epairs, s_ep[wib]);
}

// Self bin (filtered variants, a layer joined with itself): the pairs of a geometry with itself, 24 % of a parcel
// self-join's pairs and the costliest (every edge is local). One list of up to 192 edges per warp (a multiple of 32
// for the row masks; the largest that keeps 4 blocks of 4 warps per SM: 256 with 3 blocks measured 5 % slower),
// row masks only, A's gather and contribution pass only (refine_pair_t SELF).
constexpr int CAP_SELF = 192;
constexpr size_t SELF_LIST = (size_t)CAP_SELF * EDGE_BYTES_F;
constexpr size_t SELF_MASK = (size_t)(CAP_SELF / 32) * CAP_SELF * sizeof(uint32_t);
constexpr size_t SELF_SMEM = (size_t)RB_WARPS * (SELF_LIST + SELF_MASK);
constexpr int SELF_MINB = 4;   // blocks per SM: 4 x 46 KB of shared memory

// positions of the self pairs (a == b) among the candidate pairs, warp-aggregated (order free: outputs go by position)
__global__ void k_self_index(const uint2* __restrict__ pairs, uint64_t np, uint32_t* sidx, unsigned long long* nself) {
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < np; base += stride) {   // warp-uniform
    const uint64_t p = base + lane;
    bool is = false;
    if (p < np) { const uint2 pr = pairs[p]; is = pr.x == pr.y; }
    const unsigned m = __ballot_sync(0xffffffffu, is);
    unsigned long long at = 0;
    if (lane == 0 && m) at = atomicAdd(nself, (unsigned long long)__popc(m));
    at = __shfl_sync(0xffffffffu, at, 0);
    if (is) sidx[at + __popc(m & ((1u << lane) - 1))] = (uint32_t)p;
  }
}

template <bool S32>
__global__ void __launch_bounds__(RB_WARPS * 32, SELF_MINB) k_refine_self(DLayer P, const uint2* __restrict__ pairs, const uint32_t* __restrict__ sidx,
                                                                          const unsigned long long* nself, RefineArgs rp, uint8_t* flag, double* area,
                                                                          double4* ev, uint32_t* evb, uint32_t* heavy, unsigned long long* nheavy,
                                                                          unsigned long long* next, unsigned long long* epairs, int run, int runs,
                                                                          int self_cap) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ unsigned long long s_ep[RB_WARPS];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (lane == 0) s_ep[wib] = 0;
  __syncwarp();
  const EList L = carve_f(smem + (size_t)wib * SELF_LIST, CAP_SELF);
  MaskBuf mbuf;
  mbuf.rm = reinterpret_cast<uint32_t*>(smem + (size_t)RB_WARPS * SELF_LIST + (size_t)wib * SELF_MASK);
  mbuf.cm = nullptr;
  const uint64_t n = *nself;   // written by k_self_index, launched before this kernel
  for (int k = 0; k < runs; k++) {
    unsigned long long h0 = 0;
    if (lane == 0) h0 = atomicAdd(next, (unsigned long long)run);
    h0 = __shfl_sync(0xffffffffu, h0, 0);
    if (h0 >= n) break;
    const uint64_t h1 = h0 + run < n ? h0 + run : n;
    for (uint64_t h = h0; h < h1; h++) {
      const uint32_t p = sidx[h];
      const uint2 pr = pairs[p];
      uint8_t f; double ar; double4 e4; uint32_t b4;
      const bool ok = refine_pair_t<true, false, false, true, S32, CAP_SELF>(P, P, pr.x, pr.y, rp, L, L, self_cap, lane, f, ar, e4, b4, nullptr, &mbuf,
                                                                            &s_ep[wib]);
      if (lane == 0) {
        if (!ok) { heavy[atomicAdd(nheavy, 1ull)] = p; flag[p] = 0; }
        else {
          flag[p] = f;
          if (area) area[p] = ar;
          if (ev) { ev[p] = e4; evb[p] = b4; }
        }
      }
      __syncwarp();
    }
  }
  __syncwarp();
  if (lane == 0 && s_ep[wib]) atomicAdd(epairs, s_ep[wib]);
}

// oversized pairs: the same pair routine with per-warp edge lists in global scratch. The filtered variant also
// keeps its candidate list there (cph entries); a pair with more candidates runs the full sweeps instead.
template <bool F>
__host__ __device__ constexpr size_t scratch_per_warp(int cap, int cph) {
  return ((2 * (size_t)cap * Cfg<F>::edge + (F ? (size_t)cph * 6 + 2 * ((size_t)cap + 1) * 4 + ((size_t)(2 * cap + 64) + NBK + 1) * 4 : 0)) + 15) &
         ~(size_t)15;
}
template <bool F>
__global__ void __launch_bounds__(128) k_refine_scratch(DLayer P, DLayer R, const uint2* __restrict__ pairs, const uint32_t* __restrict__ heavy,
                                                       const unsigned long long* nheavy, RefineArgs rp, uint8_t* flag, double* area, double4* ev, uint32_t* evb,
                                                       unsigned char* scratch, int cap, int cph, int* err, unsigned long long* epairs,
                                                       unsigned long long* next, int same_layer) {
  const int lane = threadIdx.x & 31;
  const uint64_t nh = *nheavy;   // written by the shared-memory bin launched before this kernel on the same stream
  if (nh == 0) return;
  unsigned long long ep = 0;
  const uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned char* base = scratch + w * scratch_per_warp<F>(cap, cph);
  EList LA = carve_t<F>(base, cap), LB = carve_t<F>(base + (size_t)cap * Cfg<F>::edge, cap);
  FlatBuf fb;
  if constexpr (F) {   // cp (u32), sa, sb (u32), pj (u16) after the lists
    fb.cp = reinterpret_cast<uint32_t*>(base + 2 * (size_t)cap * Cfg<F>::edge);
    fb.sa = fb.cp + cph;
    fb.sb = fb.sa + (cap + 1);
    fb.bl = fb.sb + (cap + 1);
    fb.boff = fb.bl + (2 * cap + 64);
    fb.pj = reinterpret_cast<uint16_t*>(fb.boff + (NBK + 1));
    fb.cap = cph;
    fb.blcap = 2 * cap + 64;
    fb.rec = LB.x0;   // cap doubles, unused by a self pair's single list
  }
  (void)nw;
  for (;;) {   // one listed pair at a time from a counter: their costs vary widely
    unsigned long long h = 0;
    if (lane == 0) h = atomicAdd(next, 1ull);
    h = __shfl_sync(0xffffffffu, h, 0);
    if (h >= nh) break;
    const uint32_t p = heavy[h];
    const uint2 pr = pairs[p];
    uint8_t f; double ar; double4 e4; uint32_t b4;
    bool ok;
    if constexpr (F) {   // candidate entries pack both edge indices in 16 bits each
      if (same_layer && pr.x == pr.y)   // a geometry with itself: one list, one contribution pass (B's list records it)
        ok = cap <= 0xFFFF && refine_pair_t<F, true, true, false, false, 1>(P, P, pr.x, pr.y, rp, LA, LA, cap, lane, f, ar, e4, b4, &fb, nullptr, &ep);
      else
        ok = cap <= 0xFFFF && refine_pair_t<F, true, true>(P, R, pr.x, pr.y, rp, LA, LB, cap, lane, f, ar, e4, b4, &fb, nullptr, &ep);
      if (!ok) ok = refine_pair_t<F, false>(P, R, pr.x, pr.y, rp, LA, LB, cap, lane, f, ar, e4, b4, nullptr, nullptr, &ep);
    } else {
      ok = refine_pair_t<F, false>(P, R, pr.x, pr.y, rp, LA, LB, cap, lane, f, ar, e4, b4, nullptr, nullptr, &ep);
    }
    if (lane == 0) {
      if (!ok) *err = 1;
      else {
        flag[p] = f;
        if (area) area[p] = ar;
        if (ev) { ev[p] = e4; evb[p] = b4; }
      }
    }
    __syncwarp();
  }
  if (lane == 0 && ep) atomicAdd(epairs, ep);
}

// Scratch-bin layout for a layer pair: list capacity (rounded to 8 edges, which keeps every double array of the slab
// 8-byte aligned), candidate entries (indices stay below 2^16) and bytes per warp.
struct ScratchGeom { int cap, cph; size_t per; };
template <bool F>
static ScratchGeom scratch_geom(const gsj_layer* P, const gsj_layer* R) {
  ScratchGeom g;
  g.cap = (int)((std::max<uint32_t>(std::max(P->max_geom_edges, R->max_geom_edges), 1u) + 7u) & ~7u);
  g.cph = std::min(8 * g.cap, 1 << 16);
  g.per = scratch_per_warp<F>(g.cap, g.cph);
  return g;
}

// One refinement = one graph launch between the counters' reset and their copy to pinned host memory: the
// shared-memory bin (pairs whose local lists fit bin_cap), then the scratch bin (the pairs the first bin listed as
// oversized; it reads their count on the device, so no host round trip separates the bins); then one stream sync.
// The executable graph is built once per context and variant and re-parameterised per call.
template <bool F, bool S32 = false>
static void refine_t(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint2* pairs, uint64_t np, const RefineArgs& rp, uint8_t* flag,
                     double* area, double4* ev, uint32_t* evb) {
  cudaStream_t s = c->stream;
  const int bit = S32 ? 4 : (F ? 2 : 1);
  if (!(c->refine_attr & bit)) {
    GSJ_CK(cudaFuncSetAttribute(k_refine<F, S32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg<F>::smem));
    c->refine_attr |= bit;
  }
  const RefineShape& sh = c->shape;
  unsigned long long* ctr = c->counters.as<unsigned long long>(8);
  int* err = reinterpret_cast<int*>(ctr + 1);
  uint32_t* heavy = c->heavy.as<uint32_t>(np);
  const int bin_cap = std::min(sh.bin_cap, Cfg<F>::cap), run = sh.run, runs = sh.runs;
  int blocks;
  if constexpr (F) {
    // enough warps to cover every pair with `runs` fetches each, spread over all SMs; more than one wave of blocks
    // is rounded up to whole waves, so the last wave's blocks share the remaining pairs (the counter hands them out)
    // instead of leaving part of the GPU idle while a partial wave runs
    const uint64_t per_block = (uint64_t)RB_WARPS * runs * run, wave = (uint64_t)c->sm_count * Cfg<F>::minb;
    uint64_t cover = (np + per_block - 1) / per_block;
    if (cover > wave) cover = (cover + wave - 1) / wave * wave;
    const uint64_t spread = std::min<uint64_t>((np + (uint64_t)RB_WARPS * run - 1) / ((uint64_t)RB_WARPS * run), wave);
    blocks = (int)std::min<uint64_t>(std::max<uint64_t>(cover, spread), 1u << 30);
  } else {
    blocks = (int)std::min<uint64_t>((np + RB_WARPS - 1) / RB_WARPS, (uint64_t)c->sm_count * 8);
  }
  // a pair can only be oversized when one of its polygons has more edges than the bin holds
  const bool scr = std::max(P->max_geom_edges, R->max_geom_edges) > (uint32_t)bin_cap;
  const ScratchGeom sg = scratch_geom<F>(P, R);
  int sblocks = 0;
  unsigned char* sbuf = nullptr;
  if (scr) {   // warps: the shape's share of every SM, at most one per pair and at most 1 GiB of lists
    uint64_t nwarps = std::min<uint64_t>((uint64_t)c->sm_count * sh.scratch_wpsm, std::max<uint64_t>(1, (1ull << 30) / sg.per));
    nwarps = std::min<uint64_t>(nwarps, np);
    nwarps = (nwarps + 3) / 4 * 4;
    sblocks = (int)(nwarps / 4);
    sbuf = c->scratch.as<unsigned char>(sg.per * nwarps);
  }
  // self bin: a layer joined with itself (filtered variants); its pairs of a geometry with itself go to
  // k_refine_self, the others stay in the shared-memory bin, and the two run side by side
  const bool self = F && P == R;
  int iblocks = 1, fblocks = 1;
  uint32_t* sidx = nullptr;
  const int self_cap = std::min(sh.bin_cap + sh.bin_cap / 2, CAP_SELF);   // 1.5 x the shape's shared-memory bin threshold
  if (self) {
    const int sbit = S32 ? 16 : 8;
    if (!(c->refine_attr & sbit)) {
      GSJ_CK(cudaFuncSetAttribute(k_refine_self<S32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SELF_SMEM));
      c->refine_attr |= sbit;
    }
    sidx = c->selfidx.as<uint32_t>(np);
    iblocks = (int)std::min<uint64_t>((np + 255) / 256, (uint64_t)c->sm_count * 8);
    // at most one self pair per probe geometry: cover that many with `runs` fetches per warp, whole waves
    const uint64_t ub = std::min<uint64_t>(np, P->d.n), per_block = (uint64_t)RB_WARPS * runs * run, wave = (uint64_t)c->sm_count * SELF_MINB;
    uint64_t cover = (ub + per_block - 1) / per_block;
    if (cover > wave) cover = (cover + wave - 1) / wave * wave;
    const uint64_t spread = std::min<uint64_t>((ub + (uint64_t)RB_WARPS * run - 1) / ((uint64_t)RB_WARPS * run), wave);
    fblocks = (int)std::min<uint64_t>(std::max<uint64_t>(cover, spread), 1u << 30);
  }
  unsigned long long* h = c->h_refine.as<unsigned long long>(4);
  // counters: [0] oversized pairs, [1] error word, [2] pair counter, [3] local edge pairs, [4] scratch pair counter,
  // [5] self pairs, [6] self pair counter
  auto a_main = kernel_args(k_refine<F, S32>, P->d, R->d, pairs, np, rp, flag, area, ev, evb, heavy, ctr, ctr + 2, ctr + 3, run, runs, bin_cap,
                            self ? 1 : 0);
  auto a_scr = kernel_args(k_refine_scratch<F>, P->d, R->d, pairs, heavy, ctr, rp, flag, area, ev, evb, sbuf, sg.cap, sg.cph, err, ctr + 3,
                           ctr + 4, P == R ? 1 : 0);
  auto a_idx = kernel_args(k_self_index, pairs, np, sidx, ctr + 5);
  auto a_self = kernel_args(k_refine_self<S32>, P->d, pairs, sidx, ctr + 5, rp, flag, area, ev, evb, heavy, ctr, ctr + 6, ctr + 3, run, runs, self_cap);
  cudaKernelNodeParams km{}, ks{}, ki{}, kf{};
  km.func = (void*)k_refine<F, S32>;
  km.gridDim = dim3(blocks);
  km.blockDim = dim3(RB_WARPS * 32);
  km.sharedMemBytes = (unsigned)Cfg<F>::smem;
  km.kernelParams = a_main.ptr;
  ks.func = (void*)k_refine_scratch<F>;
  ks.gridDim = dim3(std::max(sblocks, 1));
  ks.blockDim = dim3(128);
  ks.kernelParams = a_scr.ptr;
  ki.func = (void*)k_self_index;
  ki.gridDim = dim3(iblocks);
  ki.blockDim = dim3(256);
  ki.kernelParams = a_idx.ptr;
  kf.func = (void*)k_refine_self<S32>;
  kf.gridDim = dim3(fblocks);
  kf.blockDim = dim3(RB_WARPS * 32);
  kf.sharedMemBytes = (unsigned)SELF_SMEM;
  kf.kernelParams = a_self.ptr;
  RefineGraph& g = c->rgraph[((S32 ? 2 : (F ? 1 : 0)) * 2 + (scr ? 1 : 0)) * 2 + (self ? 1 : 0)];
  if (!g.exec) {   // the graph is kept with its executable: the node handles used for the updates belong to it
    if (!g.graph) {
      GSJ_CK(cudaGraphCreate(&g.graph, 0));
      // shared-memory bin || (self index -> self bin), then the scratch bin after both
      GSJ_CK(cudaGraphAddKernelNode(&g.n_main, g.graph, nullptr, 0, &km));
      std::vector<cudaGraphNode_t> before{g.n_main};
      if (self) {
        GSJ_CK(cudaGraphAddKernelNode(&g.n_idx, g.graph, nullptr, 0, &ki));
        GSJ_CK(cudaGraphAddKernelNode(&g.n_self, g.graph, &g.n_idx, 1, &kf));
        before.push_back(g.n_self);
      }
      if (scr) GSJ_CK(cudaGraphAddKernelNode(&g.n_scr, g.graph, before.data(), before.size(), &ks));
    }
    GSJ_CK(cudaGraphInstantiate(&g.exec, g.graph, 0));
  } else {
    GSJ_CK(cudaGraphExecKernelNodeSetParams(g.exec, g.n_main, &km));
    if (self) {
      GSJ_CK(cudaGraphExecKernelNodeSetParams(g.exec, g.n_idx, &ki));
      GSJ_CK(cudaGraphExecKernelNodeSetParams(g.exec, g.n_self, &kf));
    }
    if (scr) GSJ_CK(cudaGraphExecKernelNodeSetParams(g.exec, g.n_scr, &ks));
  }
  GSJ_CK(cudaMemsetAsync(ctr, 0, 7 * sizeof(unsigned long long), s));
  GSJ_CK(cudaGraphLaunch(g.exec, s));
  c->launches += 1 + (scr ? 1 : 0) + (self ? 2 : 0);
  GSJ_CK(cudaMemcpyAsync(h, ctr, 32, cudaMemcpyDeviceToHost, s));
  c->refine_pending = true;
}

void refine_enqueue(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint2* pairs, uint64_t np, const RefineArgs& rp, int mode,
                    uint8_t* flag, double* area, double4* ev, uint32_t* evb) {
  if (!np) return;
  if (mode == GSJ_REFINE_FILTERED_FP32) refine_t<true, true>(c, P, R, pairs, np, rp, flag, area, ev, evb);
  else if (mode == GSJ_REFINE_FILTERED) refine_t<true>(c, P, R, pairs, np, rp, flag, area, ev, evb);
  else refine_t<false>(c, P, R, pairs, np, rp, flag, area, ev, evb);
}

uint64_t refine_result(gsj_ctx* c) {
  if (!c->refine_pending) return 0;
  c->refine_pending = false;
  const unsigned long long* h = c->h_refine.as<unsigned long long>(4);
  if (reinterpret_cast<const int*>(h + 1)[0]) throw Error(GSJ_ERR_CUDA, "oversized pair exceeded the scratch edge capacity");
  c->edge_pairs += h[3];
  return h[0];
}

uint64_t refine(gsj_ctx* c, const gsj_layer* P, const gsj_layer* R, const uint2* pairs, uint64_t np, const RefineArgs& rp, int mode,
                uint8_t* flag, double* area, double4* ev, uint32_t* evb) {
  refine_enqueue(c, P, R, pairs, np, rp, mode, flag, area, ev, evb);
  GSJ_CK(cudaStreamSynchronize(c->stream));
  return refine_result(c);
}

}  // namespace gsj
