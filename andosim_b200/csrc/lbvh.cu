// lbvh.cu -- linear BVH broad phase (replaces Collision::build_*_bvh and
// broad_phase_triangles / broad_phase_edges, collision.cpp:65-276).
//
// Boxes are FP32, built from the FP32-rounded positions exactly as the
// reference's Real=float AABBs are (collision.cpp:48-62), optionally inflated
// by `pad`. The candidate predicate is the reference's inclusive overlap test
// (collision.h:37-41) with a +-1e-4 point box, the incident-face exclusion
// (collision.cpp:221) and, for edges, e1 < e2 and no shared vertex
// (collision.cpp:259-266). Any correct hierarchy returns exactly the set of
// primitive pairs whose boxes pass that test, so the result equals the
// brute-force query bit for bit once sorted.
//
// Pipeline: primitive boxes -> scene bounds -> 30-bit Morton codes of box
// centres (index appended, so keys are unique) -> radix sort -> Karras
// hierarchy (one thread per internal node) -> bottom-up refit in shared
// memory (cut subtrees, then the nodes above the cut) -> one thread per query with an explicit stack; hits are compacted
// with a warp ballot (one atomic per warp) and the pair list is then sorted so
// its order does not depend on scheduling.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>

#include "lbvh.cuh"
#include "narrow.cuh"

namespace ando {

namespace {

constexpr int TPB = 256;
inline int nblk(long long n) { return int((n + TPB - 1) / TPB); }

using Box = LbvhBox;

__device__ inline float3 xf(const double* x, int i) { return make_float3(float(x[3 * i]), float(x[3 * i + 1]), float(x[3 * i + 2])); }

__device__ inline void grow(Box& b, float3 q) {
  b.lo[0] = fminf(b.lo[0], q.x); b.lo[1] = fminf(b.lo[1], q.y); b.lo[2] = fminf(b.lo[2], q.z);
  b.hi[0] = fmaxf(b.hi[0], q.x); b.hi[1] = fmaxf(b.hi[1], q.y); b.hi[2] = fmaxf(b.hi[2], q.z);
}

// Box of primitive i at positions x, or swept over x -> x1 when x1 is given.
__device__ inline Box prim_box(const double* x, const double* x1, const int* prims, int arity, int i, float pad) {
  float3 p = xf(x, prims[arity * i]);
  Box b; b.lo[0] = b.hi[0] = p.x; b.lo[1] = b.hi[1] = p.y; b.lo[2] = b.hi[2] = p.z;
  for (int k = 1; k < arity; ++k) grow(b, xf(x, prims[arity * i + k]));
  if (x1) for (int k = 0; k < arity; ++k) grow(b, xf(x1, prims[arity * i + k]));
  if (pad > 0.f) for (int k = 0; k < 3; ++k) { b.lo[k] -= pad; b.hi[k] += pad; }
  return b;
}

__global__ void k_prim_boxes(const double* x, const double* x1, const int* prims, int arity, int n, float pad, Box* boxes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  boxes[i] = prim_box(x, x1, prims, arity, i, pad);
}

// Scene bounds as min/max over box centres (block reduction + float atomics
// on the ordered-int encoding, exact for min/max).
__device__ inline int f2ord(float f) { int i = __float_as_int(f); return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ inline float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_bounds_init(int* b) {
  if (threadIdx.x < 3) { b[threadIdx.x] = 0x7fffffff; b[3 + threadIdx.x] = (int)0x80000000; }
}
__global__ void k_bounds(const Box* boxes, int n, int* bounds) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (i < n) for (int k = 0; k < 3; ++k) { float c = 0.5f * (boxes[i].lo[k] + boxes[i].hi[k]); lo[k] = c; hi[k] = c; }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) for (int k = 0; k < 3; ++k) { atomicMin(&bounds[k], f2ord(lo[k])); atomicMax(&bounds[3 + k], f2ord(hi[k])); }
}

__device__ inline unsigned expand10(unsigned v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(const Box* boxes, int n, const int* bounds, unsigned long long* keys, int* vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned m = 0;
  unsigned q[3];
  for (int k = 0; k < 3; ++k) {
    float lo = ord2f(bounds[k]), hi = ord2f(bounds[3 + k]);
    float c = 0.5f * (boxes[i].lo[k] + boxes[i].hi[k]);
    float t = hi > lo ? (c - lo) / (hi - lo) : 0.5f;
    t = fminf(fmaxf(t, 0.f), 1.f);
    q[k] = min(1023u, (unsigned)(t * 1024.f));
  }
  m = (expand10(q[0]) << 2) | (expand10(q[1]) << 1) | expand10(q[2]);
  keys[i] = ((unsigned long long)m << 32) | (unsigned)i;
  vals[i] = i;
}

__device__ inline int delta(const unsigned long long* k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return __clzll(k[i] ^ k[j]);
}

// Karras 2012: internal node i covers a key range found from the common
// prefix lengths of its neighbours. Nodes [0, n-1) are internal, leaves are
// encoded as n-1 + sorted position.
// topo[i] = {first leaf, last leaf of the left child, last leaf, parent} in
// sorted leaf positions (parent -1 at the root); the parent component is
// written by the parent's thread.
__global__ void k_karras(const unsigned long long* keys, int n, int* parent, LbvhInner* inner, int4* topo) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = delta(keys, n, i, j);
  int s = 0;
  int t = l;
  do {
    t = (t + 1) >> 1;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  int gamma = i + s * d + min(d, 0);
  int lo = min(i, j), hi = max(i, j);
  int lc = (lo == gamma) ? (n - 1 + gamma) : gamma;
  int rc = (hi == gamma + 1) ? (n - 1 + gamma + 1) : gamma + 1;
  inner[i].lc = lc; inner[i].rc = rc;
  inner[i].lmax = gamma; inner[i].rmax = hi;  // leaf ranges [lo, gamma] and [gamma + 1, hi]
  parent[lc] = i; parent[rc] = i;
  int* tw = reinterpret_cast<int*>(topo);
  tw[4 * i] = lo; tw[4 * i + 1] = gamma; tw[4 * i + 2] = hi;
  if (i == 0) tw[3] = -1;
  if (lc < n - 1) tw[4 * lc + 3] = i;
  if (rc < n - 1) tw[4 * rc + 3] = i;
}

__global__ void k_rank(const int* order, int n, int* rank) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) rank[order[p]] = p;
}

// Per sorted leaf position: {primitive, its vertices (-1 past the arity)},
// so a query's leaf test is one 16-byte load.
__global__ void k_leafv(const int* order, const int* prims, int arity, int n, int4* leafv) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int prim = order[p];
  const int* v = prims + (long long)arity * prim;
  leafv[p] = make_int4(prim, v[0], arity > 1 ? v[1] : -1, arity > 2 ? v[2] : -1);
}

// Build time: 1 for the internal nodes at even depth, the nodes of the
// four-wide hierarchy (the root is node 0 at depth 0). Karras depth is at most
// about 64 with unique 64-bit keys; the climb is bounded at 256 regardless.
__global__ void k_wide_flags(const int4* topo, int n, int* wflag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = 0, p = topo[i].w;
  while (p >= 0 && d < 256) { ++d; p = topo[p].w; }
  wflag[i] = (d & 1) == 0;
}

__device__ inline Box ld_box_volatile(const Box* b) {
  const volatile float* v = reinterpret_cast<const volatile float*>(b);
  Box r;
  for (int k = 0; k < 3; ++k) { r.lo[k] = v[k]; r.hi[k] = v[3 + k]; }
  return r;
}

__device__ inline Box ld_box_cg(const Box* b) {
  const float* v = reinterpret_cast<const float*>(b);
  Box r;
  for (int k = 0; k < 3; ++k) { r.lo[k] = __ldcg(v + k); r.hi[k] = __ldcg(v + 3 + k); }
  return r;
}

__device__ inline Box unite(const Box& a, const Box& b) {
  Box u;
  for (int k = 0; k < 3; ++k) { u.lo[k] = fminf(a.lo[k], b.lo[k]); u.hi[k] = fmaxf(a.hi[k], b.hi[k]); }
  return u;
}

// Tiled bottom-up refit in two launches over a cut of the hierarchy made at
// build time. Below the cut: every subtree of at most RF_CUT leaves whose
// parent has more ("cut subtree"). Above it: the top nodes (more than RF_CUT
// leaves), numbered compactly.
//
// k_refit_cut: one CTA per cut subtree (grid-stride over the cut list). With
// Karras numbering a node covering leaves [lo, hi] has its index in [lo, hi],
// so every node of a subtree over [c0, c1] has a shared-memory slot (index -
// c0): the subtree's topology is staged once, each node is finished in shared
// memory by the second of its children to arrive (block-scope arrival
// counters), and the subtree's node boxes and child records are written in
// one pass afterwards; thread 0 puts the subtree's root box into its parent's
// record. The leaf boxes are computed from the positions here.
//
// k_refit_top: one CTA finishes the top nodes the same way in shared memory,
// reading the cut subtrees' boxes from nodes[], and writes them in one pass.
//
// When the top has more nodes than one CTA holds (or than the caller's
// capacity, Lbvh::top_cap), thread 0 of each cut subtree carries on through
// the top nodes with global arrival counters (acquire/release atomics; the
// second arrival zeroes the counter for the next refit) and k_refit_top does
// nothing. Min/max are exact, so every box has the same bits in any arrival
// order.
constexpr int RF_TPB = 512, RF_CUT = 1024;
struct RefitSmem { Box leaf[RF_CUT]; Box node[RF_CUT]; int4 topo[RF_CUT]; int arr[RF_CUT]; };
constexpr int TOP_TPB = 1024, TOP_MAX = 4096;
// top node: {node index, parent's top number (-1 at the root), left, right};
// a child is its top number (>= 0) or -(1 + its nodes[] index) below the cut
struct TopSmem { int4 rec[TOP_MAX]; Box box[TOP_MAX]; int arr[TOP_MAX]; };

__device__ inline bool is_top(const int4& t) { return t.z - t.x + 1 > RF_CUT; }

// Build time: 1 for the top nodes (exclusive-scanned into their numbers).
__global__ void k_top_flags(const int4* topo, int n, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n - 1) flag[i] = is_top(topo[i]) ? 1 : 0;
}

// Build time: the top records and the cut list (entries 2k, 2k+1: the
// below-cut children of top node k as leaf ranges, {-1, -1} for a top child).
__global__ void k_top_records(const int4* topo, const LbvhInner* inner, const int* topnum, int n, int4* rec, int2* cuts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int4 t = topo[i];
  if (!is_top(t)) return;
  const int k = topnum[i];
  const int lc = inner[i].lc, rc = inner[i].rc;
  const bool ltop = lc < n - 1 && is_top(topo[lc]), rtop = rc < n - 1 && is_top(topo[rc]);
  rec[k] = make_int4(i, t.w >= 0 ? topnum[t.w] : -1, ltop ? topnum[lc] : -(1 + lc), rtop ? topnum[rc] : -(1 + rc));
  cuts[2 * k] = ltop ? make_int2(-1, -1) : make_int2(t.x, t.y);
  cuts[2 * k + 1] = rtop ? make_int2(-1, -1) : make_int2(t.y + 1, t.z);
}

// Build time: meta = {top nodes, cut entries}; with no top node the whole
// hierarchy is one cut subtree.
__global__ void k_top_count(const int* flag, const int* topnum, int n, int* meta, int2* cuts) {
  const int m = n > 1 ? topnum[n - 2] + flag[n - 2] : 0;
  meta[0] = m;
  meta[1] = m > 0 ? 2 * m : 1;
  if (m == 0) cuts[0] = make_int2(0, n - 1);
}

// A node's final box into its four-wide slot (ws = 4 * node + slot; the
// slot's six floats start on an 8-byte boundary).
__device__ inline void store_slot(LbvhWide* wide, int ws, const Box& b) {
  float2* d = reinterpret_cast<float2*>(&wide[ws >> 2].box[ws & 3][0]);
  d[0] = make_float2(b.lo[0], b.lo[1]);
  d[1] = make_float2(b.lo[2], b.hi[0]);
  d[2] = make_float2(b.hi[1], b.hi[2]);
}

// The climbs below touch shared memory only (their block-scope fences then
// have no global store to wait for); each kernel writes its boxes to global
// memory in one pass after the climb.
__global__ void __launch_bounds__(RF_TPB) k_refit_cut(const double* x, const double* x1, const int* prims, int arity, float pad,
                                                      const int* order, int n, const int* parent, const int4* topo, const int2* cuts,
                                                      const int* meta, int top_cap, Box* nodes, int* arrive, const int* wslot, LbvhWide* wide) {
  extern __shared__ __align__(16) unsigned char rf_raw[];
  RefitSmem& S = *reinterpret_cast<RefitSmem*>(rf_raw);
  const int ncut = meta[1];
  const bool top_global = meta[0] > top_cap;
  for (int cb = blockIdx.x; cb < ncut; cb += gridDim.x) {
    const int2 cut = cuts[cb];
    if (cut.x < 0) continue;  // uniform over the CTA
    const int c0 = cut.x, c1 = cut.y;
    __syncthreads();  // the previous subtree's shared memory is no longer read
    for (int t = threadIdx.x; t <= c1 - c0; t += RF_TPB) {
      S.arr[t] = 0;
      const int q = c0 + t;
      if (q < n - 1) S.topo[t] = topo[q];
      S.leaf[t] = prim_box(x, x1, prims, arity, order[q], pad);
    }
    __syncthreads();
    const int4 outside = make_int4(-1, 0, 0, -1);  // fails the inside test
    for (int t = threadIdx.x; t <= c1 - c0; t += RF_TPB) {
      const int i = c0 + t;
      Box box = S.leaf[t];
      int chi = i;  // last leaf under the current node
      int p = n > 1 ? parent[n - 1 + i] : -1;
      int4 tp = p >= c0 && p <= c1 ? S.topo[p - c0] : outside;
      while (p >= 0 && tp.x >= c0 && tp.z <= c1) {  // p's leaves all in this subtree
        const int plo = tp.x, pl = tp.y, phi = tp.z, pp = tp.w;
        const bool from_left = chi == pl;
        // the sibling covers [sl, sh]: a leaf when sl == sh, else internal node sidx
        const int sl = from_left ? pl + 1 : plo, sh = from_left ? phi : pl, sidx = from_left ? pl + 1 : pl;
        __threadfence_block();
        if (atomicAdd(&S.arr[p - c0], 1) == 0) break;
        __threadfence_block();
        box = unite(box, sl == sh ? ld_box_volatile(&S.leaf[sl - c0]) : ld_box_volatile(&S.node[sidx - c0]));
        S.node[p - c0] = box;
        chi = phi;
        p = pp;
        tp = p >= c0 && p <= c1 ? S.topo[p - c0] : outside;
      }
    }
    __syncthreads();
    // write-out: the boxes of the subtree's leaves and internal nodes, each
    // also into its four-wide slot
    for (int t = threadIdx.x; t <= c1 - c0; t += RF_TPB) {
      const int q = c0 + t;
      nodes[n - 1 + q] = S.leaf[t];
      const int wl = wslot[n - 1 + q];
      if (wl >= 0) store_slot(wide, wl, S.leaf[t]);
      if (q < n - 1) {
        const int4 tq = S.topo[t];
        if (tq.x >= c0 && tq.z <= c1) {
          nodes[q] = S.node[t];
          const int wn = wslot[q];
          if (wn >= 0) store_slot(wide, wn, S.node[t]);
        }
      }
    }
    // with more top nodes than k_refit_top holds, thread 0 carries on from
    // the subtree's root (index c0 or c1, or the leaf) through the top nodes;
    // that needs every thread's nodes[] published first
    if (top_global) {
      __threadfence();
      __syncthreads();
    }
    if (top_global && threadIdx.x == 0) {
      int root = -1;  // internal root index, -1: a single leaf
      if (c1 > c0) root = (S.topo[0].x == c0 && S.topo[0].z == c1) ? c0 : c1;
      Box box = root < 0 ? S.leaf[0] : S.node[root - c0];
      int p = root < 0 ? (n > 1 ? parent[n - 1 + c0] : -1) : S.topo[root - c0].w;
      int chi = c1;
      if (p >= 0) {
        while (p >= 0) {
          const int4 tp = __ldg(topo + p);
          const bool from_left = chi == tp.y;
          int prior;
          asm volatile("atom.add.acq_rel.gpu.s32 %0, [%1], 1;" : "=r"(prior) : "l"(arrive + p) : "memory");
          if (prior == 0) break;
          arrive[p] = 0;
          const int sl = from_left ? tp.y + 1 : tp.x, sh = from_left ? tp.z : tp.y, sidx = from_left ? tp.y + 1 : tp.y;
          box = unite(box, ld_box_cg(nodes + (sl == sh ? n - 1 + sl : sidx)));
          nodes[p] = box;
          const int wp = wslot[p];
          if (wp >= 0) store_slot(wide, wp, box);
          chi = tp.z;
          p = tp.w;
        }
      }
    }
  }
}

__global__ void __launch_bounds__(TOP_TPB) k_refit_top(const int* meta, int top_cap, const int4* rec, Box* nodes, const int* wslot, LbvhWide* wide) {
  extern __shared__ __align__(16) unsigned char rt_raw[];
  TopSmem& S = *reinterpret_cast<TopSmem*>(rt_raw);
  const int m = meta[0];
  if (m <= 0 || m > top_cap) return;
  for (int k = threadIdx.x; k < m; k += TOP_TPB) {
    const int4 r = rec[k];
    S.rec[k] = r;
    S.arr[k] = (r.z < 0) + (r.w < 0);  // below-cut children have arrived already
  }
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += TOP_TPB) {
    int4 r = S.rec[k];
    if (r.z >= 0 || r.w >= 0) continue;  // starts only where both children are below the cut
    int cur = k;
    Box box = unite(ld_box_cg(nodes + (-r.z - 1)), ld_box_cg(nodes + (-r.w - 1)));
    while (true) {
      S.box[cur] = box;
      const int pc = r.y;
      if (pc < 0) break;
      const int4 pr = S.rec[pc];
      const bool from_left = pr.z == cur;
      __threadfence_block();
      if (atomicAdd(&S.arr[pc], 1) == 0) break;
      __threadfence_block();
      const int sib = from_left ? pr.w : pr.z;
      box = unite(box, sib >= 0 ? ld_box_volatile(&S.box[sib]) : ld_box_cg(nodes + (-sib - 1)));
      cur = pc;
      r = pr;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < m; k += TOP_TPB) {
    const int4 r = S.rec[k];
    nodes[r.x] = S.box[k];
    const int ws = wslot[r.x];
    if (ws >= 0) store_slot(wide, ws, S.box[k]);
  }
}

// Build time: the topology of each four-wide node (children, leaf bounds,
// empty slots) and the slot of every binary node whose box a four-wide node
// keeps: a leaf child of a four-wide node, or a child of a folded node. The
// caller sets wslot to -1 first (the root and the folded nodes keep it).
__global__ void k_wide_topo(const LbvhInner* inner, const int* wflag, const int* widx, int n, LbvhWide* wide, int* wslot) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1 || !wflag[i]) return;
  const int leaf0 = n - 1, w = widx[i];
  LbvhWide& W = wide[w];
  const LbvhInner r = inner[i];
  auto enc = [&](int c) { return c >= leaf0 ? -(c - leaf0) - 1 : widx[c]; };
  for (int sd = 0; sd < 2; ++sd) {
    const int c = sd ? r.rc : r.lc;
    const int k = 2 * sd;
    if (c >= leaf0) {
      W.child[k] = enc(c); W.cmax[k] = sd ? r.rmax : r.lmax; wslot[c] = 4 * w + k;
      for (int e = 0; e < 3; ++e) { W.box[k + 1][e] = FLT_MAX; W.box[k + 1][3 + e] = -FLT_MAX; }
      W.child[k + 1] = 0; W.cmax[k + 1] = INT_MIN;
    } else {
      const LbvhInner g = inner[c];
      W.child[k] = enc(g.lc); W.cmax[k] = g.lmax; wslot[g.lc] = 4 * w + k;
      W.child[k + 1] = enc(g.rc); W.cmax[k + 1] = g.rmax; wslot[g.rc] = 4 * w + k + 1;
    }
  }
}

__device__ inline bool overlap(const Box& a, const Box& b) {
  return a.lo[0] <= b.hi[0] && a.hi[0] >= b.lo[0] && a.lo[1] <= b.hi[1] && a.hi[1] >= b.lo[1] && a.lo[2] <= b.hi[2] && a.hi[2] >= b.lo[2];
}

// Warp-ballot append: one atomic per warp per round of hits.
__device__ inline void emit(bool hit, int q, int prim, int2* out, int* count, int cap) {
  unsigned mask = __ballot_sync(0xffffffffu, hit);
  if (!mask) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (hit) {
    int slot = base + __popc(mask & ((1u << lane) - 1u));
    if (slot < cap) out[slot] = make_int2(q, prim);
  }
}

// One thread per query. kind 0: query = vertex (point box +-1e-4 inflated by
// pad), prims = triangles, skip incident triangles. kind 1: query = edge,
// prims = edges, keep e1 < e2 without shared vertex. kind 2: query = edge,
// prims = triangles, skip triangles that hold either end of the edge.
__global__ void k_query(const double* x, const double* x1, const int* qprims, const int* qorder, int kind, int nq, float pad, int n,
                        const int4* leafv, const int* rank, const LbvhWide* wide, const Box* nodes, int2* out, int* count, int cap) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < nq;
  const int q = active && qorder ? qorder[t] : t;
  Box qb;
  int qa = -1, qc = -1;
  if (active) {
    if (kind == 0) {
      float3 p = xf(x, q);
      float e = 1e-4f;
      qb.lo[0] = p.x - e; qb.lo[1] = p.y - e; qb.lo[2] = p.z - e;
      qb.hi[0] = p.x + e; qb.hi[1] = p.y + e; qb.hi[2] = p.z + e;
      if (x1) {
        float3 p1 = xf(x1, q);
        qb.lo[0] = fminf(qb.lo[0], p1.x - e); qb.lo[1] = fminf(qb.lo[1], p1.y - e); qb.lo[2] = fminf(qb.lo[2], p1.z - e);
        qb.hi[0] = fmaxf(qb.hi[0], p1.x + e); qb.hi[1] = fmaxf(qb.hi[1], p1.y + e); qb.hi[2] = fmaxf(qb.hi[2], p1.z + e);
      }
      if (pad > 0.f) for (int k = 0; k < 3; ++k) { qb.lo[k] -= pad; qb.hi[k] += pad; }
    } else {
      qa = qprims[2 * q]; qc = qprims[2 * q + 1];
      float3 a = xf(x, qa), b = xf(x, qc);
      qb.lo[0] = fminf(a.x, b.x); qb.lo[1] = fminf(a.y, b.y); qb.lo[2] = fminf(a.z, b.z);
      qb.hi[0] = fmaxf(a.x, b.x); qb.hi[1] = fmaxf(a.y, b.y); qb.hi[2] = fmaxf(a.z, b.z);
      if (x1) { grow(qb, xf(x1, qa)); grow(qb, xf(x1, qc)); }
      if (pad > 0.f) for (int k = 0; k < 3; ++k) { qb.lo[k] -= pad; qb.hi[k] += pad; }
    }
  }
  // Depth-first traversal of the four-wide hierarchy: each step loads one
  // 128-byte node and tests its (up to) four child boxes; an overlapping leaf
  // child is reported at once, the first overlapping internal child is entered
  // and the others go on the stack. The binary hierarchy is at most 64 levels
  // deep with unique 64-bit keys, the four-wide one half that, so three
  // pushes per level fit 96 slots; an overflow would be reported through
  // count[1] instead of dropping candidates silently.
  //
  // The edge-edge query is a self query: each pair is found from the edge
  // that comes first in the tree's sorted leaf order (children whose leaves
  // all come before the query's own position are skipped) and reported with
  // the lower edge index first, which is the set the q < prim rule of a full
  // query gives.
  constexpr int STACK = 96;
  int stack[STACK];
  int sp = 0;
  const int qpos = active && kind == 1 ? rank[q] : -1;
  const bool single = active && n == 1;  // one primitive: the root (node 0) is its leaf
  int node = active && n > 1 ? 0 : -1;
  auto accept = [&](int pos) {
    const int4 lv = leafv[pos];
    bool hit;
    if (kind == 0) hit = lv.y != q && lv.z != q && lv.w != q;
    else if (kind == 2) hit = lv.y != qa && lv.y != qc && lv.z != qa && lv.z != qc && lv.w != qa && lv.w != qc;
    else hit = pos > qpos && lv.y != qa && lv.y != qc && lv.z != qa && lv.z != qc;
    return hit ? lv.x : -1;
  };
  auto emit_pair = [&](int prim) {  // (lower, higher) edge index for the self query
    const bool hit = prim >= 0;
    const int a = kind == 1 && hit ? min(q, prim) : q, b = kind == 1 && hit ? max(q, prim) : prim;
    emit(hit, a, b, out, count, cap);
  };
  if (__any_sync(0xffffffffu, single)) {
    int prim = single && overlap(qb, nodes[0]) ? accept(0) : -1;
    emit_pair(prim);
  }
  while (__any_sync(0xffffffffu, node >= 0)) {
    int h[4] = {-1, -1, -1, -1};
    if (node >= 0) {
      const float4* r = reinterpret_cast<const float4*>(wide + node);
      const float4 f0 = __ldg(r), f1 = __ldg(r + 1), f2 = __ldg(r + 2), f3 = __ldg(r + 3), f4 = __ldg(r + 4), f5 = __ldg(r + 5);
      const int4 ch = __ldg(reinterpret_cast<const int4*>(r) + 6), cm = __ldg(reinterpret_cast<const int4*>(r) + 7);
      int next = -1;
      auto slot = [&](float lox, float loy, float loz, float hix, float hiy, float hiz, int c, int m, int& hk) {
        if (!(m > qpos && qb.lo[0] <= hix && qb.hi[0] >= lox && qb.lo[1] <= hiy && qb.hi[1] >= loy && qb.lo[2] <= hiz && qb.hi[2] >= loz))
          return;
        if (c < 0) hk = accept(-c - 1);
        else if (next < 0) next = c;
        else if (sp < STACK) stack[sp++] = c;
        else atomicAdd(count + 1, 1);
      };
      slot(f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, ch.x, cm.x, h[0]);
      slot(f1.z, f1.w, f2.x, f2.y, f2.z, f2.w, ch.y, cm.y, h[1]);
      slot(f3.x, f3.y, f3.z, f3.w, f4.x, f4.y, ch.z, cm.z, h[2]);
      slot(f4.z, f4.w, f5.x, f5.y, f5.z, f5.w, ch.w, cm.w, h[3]);
      node = next >= 0 ? next : (sp > 0 ? stack[--sp] : -1);
    }
    emit_pair(h[0]);
    emit_pair(h[1]);
    emit_pair(h[2]);
    emit_pair(h[3]);
  }
}

// The four vertices of candidate pair (q, prim): kind 0 vertex q against
// triangle prim; kind 1 edge q against edge prim.
__device__ inline void pair_ids(int kind, int2 pr, const int* prims, const int* qprims, int id[4]) {
  if (kind == 0) { id[0] = pr.x; id[1] = prims[3 * pr.y]; id[2] = prims[3 * pr.y + 1]; id[3] = prims[3 * pr.y + 2]; }
  else { id[0] = qprims[2 * pr.x]; id[1] = qprims[2 * pr.x + 1]; id[2] = prims[2 * pr.y]; id[3] = prims[2 * pr.y + 1]; }
}

// Narrow phase over the candidate list of the last traversal. The count
// stays on the device (count[0]); a list that overflowed its capacity sets
// *overflow instead of being used, so the caller grows it and runs again.
constexpr int NARROW_GRID = 148 * 8;

// candidates whose FP64 distance at x is below gap -> surv (count[2])
__global__ void k_pairs_gap(const int2* cand, const int* count, int cap, int kind, const int* prims, const int* qprims, const double* x,
                            double gap, int2* surv, int* scount) {
  const int n = min(count[0], cap);
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    bool keep = false;
    int2 pr = make_int2(0, 0);
    if (i < n) {
      pr = cand[i];
      int id[4];
      pair_ids(kind, pr, prims, qprims, id);
      keep = pair_gap(kind, id, x) < gap;
    }
    emit(keep, pr.x, pr.y, surv, scount, cap);
  }
}

// min over the candidates of the conservative time of impact along ext. With
// `pad` > 0 the traversal ran on boxes inflated by pad (so that the list also
// holds every pair that can come within the contact distance at any position
// on the way): only the pairs whose boxes overlap without the pad, built and
// compared exactly as an unpadded traversal does, bound the step.
__global__ void k_pairs_toi(const int2* cand, const int* count, int cap, int kind, const int* prims, const int* qprims, const double* x,
                            const double* x1, const double* ext, float pad, double eta_min, double near, unsigned long long* toi,
                            int* overflow) {
  if (count[0] > cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(overflow, count[0]);  // the capacity that is needed
    return;
  }
  const int n = count[0];
  double t = 1.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 pr = cand[i];
    if (pad > 0.f) {
      Box qb;
      if (kind == 0) {
        const float3 p = xf(x, pr.x), p1 = xf(x1, pr.x);
        const float e = 1e-4f;
        qb.lo[0] = fminf(p.x - e, p1.x - e); qb.lo[1] = fminf(p.y - e, p1.y - e); qb.lo[2] = fminf(p.z - e, p1.z - e);
        qb.hi[0] = fmaxf(p.x + e, p1.x + e); qb.hi[1] = fmaxf(p.y + e, p1.y + e); qb.hi[2] = fmaxf(p.z + e, p1.z + e);
      } else {
        qb = prim_box(x, x1, qprims, 2, pr.x, 0.f);
      }
      if (!overlap(qb, prim_box(x, x1, prims, kind == 0 ? 3 : 2, pr.y, 0.f))) continue;
    }
    int id[4];
    pair_ids(kind, pr, prims, qprims, id);
    t = fmin(t, pair_toi(kind, id, x, ext, eta_min, near));
  }
  t = warp_min(t);
  if ((threadIdx.x & 31) == 0 && t < 1.0) atomic_min_pos(toi, t);
}

// Exact segment-triangle crossing test in FP64: the segment's ends lie
// strictly on opposite sides of the triangle's plane and the crossing point
// has barycentric coordinates in [0, 1]. Every product, sum and quotient is
// rounded on its own (no fused multiply-add), in the order written, so the
// test takes the same decision as the same formula in plain IEEE double
// arithmetic on the host.
__device__ inline bool segment_crosses_triangle(const double* x, int p, int q, int a, int b, int c) {
  auto mul = [](double u, double v) { return __dmul_rn(u, v); };
  auto add = [](double u, double v) { return __dadd_rn(u, v); };
  auto sub = [](double u, double v) { return __dsub_rn(u, v); };
  double A[3], u[3], w[3], P[3], Q[3];
  for (int k = 0; k < 3; ++k) {
    A[k] = x[3 * a + k];
    u[k] = sub(x[3 * b + k], A[k]);
    w[k] = sub(x[3 * c + k], A[k]);
    P[k] = x[3 * p + k];
    Q[k] = x[3 * q + k];
  }
  const double n0 = sub(mul(u[1], w[2]), mul(u[2], w[1]));
  const double n1 = sub(mul(u[2], w[0]), mul(u[0], w[2]));
  const double n2 = sub(mul(u[0], w[1]), mul(u[1], w[0]));
  const double s0 = add(add(mul(n0, sub(P[0], A[0])), mul(n1, sub(P[1], A[1]))), mul(n2, sub(P[2], A[2])));
  const double s1 = add(add(mul(n0, sub(Q[0], A[0])), mul(n1, sub(Q[1], A[1]))), mul(n2, sub(Q[2], A[2])));
  if (!((s0 > 0.0 && s1 < 0.0) || (s0 < 0.0 && s1 > 0.0))) return false;
  const double t = __ddiv_rn(s0, sub(s0, s1));
  double X[3];
  for (int k = 0; k < 3; ++k) X[k] = sub(add(P[k], mul(t, sub(Q[k], P[k]))), A[k]);
  auto dot3 = [&](const double* e, const double* f) { return add(add(mul(e[0], f[0]), mul(e[1], f[1])), mul(e[2], f[2])); };
  const double uu = dot3(u, u), uw = dot3(u, w), ww = dot3(w, w), xu = dot3(X, u), xw = dot3(X, w);
  const double den = sub(mul(uu, ww), mul(uw, uw));
  if (!(fabs(den) > 0.0)) return false;
  const double bv = __ddiv_rn(sub(mul(ww, xu), mul(uw, xw)), den);
  const double bw = __ddiv_rn(sub(mul(uu, xw), mul(uw, xu)), den);
  return bv >= 0.0 && bw >= 0.0 && add(bv, bw) <= 1.0;
}

// Crossings among the (edge, triangle) candidates of a kind-2 traversal,
// summed into *crossings; nothing when the list overflowed its capacity (the
// caller reads count[0], grows the list and runs again).
__global__ void k_pairs_cross(const int2* cand, const int* count, int cap, const int* tris, const int* edges, const double* x,
                              unsigned long long* crossings) {
  if (count[0] > cap) return;
  const int n = count[0];
  unsigned long long mine = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int2 pr = cand[i];
    mine += segment_crosses_triangle(x, edges[2 * pr.x], edges[2 * pr.x + 1], tris[3 * pr.y], tris[3 * pr.y + 1], tris[3 * pr.y + 2]);
  }
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(crossings, mine);
}

__global__ void k_pair_keys(const int2* pairs, int n, unsigned long long* keys) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = ((unsigned long long)(unsigned)pairs[i].x << 32) | (unsigned)pairs[i].y;
}

}  // namespace

cudaError_t Lbvh::reserve_prims(int n) {
  cudaError_t e;
  size_t N = n > 0 ? n : 1;
  if ((e = boxes.reserve(N))) return e;
  if ((e = keys.reserve(N))) return e;
  if ((e = keys_sorted.reserve(N))) return e;
  if ((e = idx.reserve(N))) return e;
  if ((e = order.reserve(N))) return e;
  if ((e = parent.reserve(2 * N))) return e;
  if ((e = nodes.reserve(2 * N))) return e;
  if ((e = inner.reserve(N))) return e;
  if ((e = wide.reserve(N))) return e;
  if ((e = wflag.reserve(N))) return e;
  if ((e = widx.reserve(N))) return e;
  if ((e = wslot.reserve(2 * N))) return e;
  if ((e = rank.reserve(N))) return e;
  if ((e = arrive.reserve(N))) return e;
  if ((e = topo.reserve(N))) return e;
  if ((e = leafv.reserve(N))) return e;
  if ((e = topflag.reserve(N))) return e;
  if ((e = topnum.reserve(N))) return e;
  if ((e = toprec.reserve(N))) return e;
  if ((e = cuts.reserve(2 * N))) return e;
  if ((e = meta.reserve(2))) return e;
  if ((e = bounds.reserve(6))) return e;
  return cudaSuccess;
}

// Build the hierarchy over `n` primitives of `arity` vertex indices each.
cudaError_t Lbvh::build(const double* x, const double* x1, const int* prims_, int arity_, int n_, float pad, DevBuf<unsigned char>& tmp, cudaStream_t s) {
  n = n_;
  prims = prims_;
  arity = arity_;
  cudaError_t e = reserve_prims(n);
  if (e) return e;
  if (n == 0) return cudaSuccess;
  k_prim_boxes<<<nblk(n), TPB, 0, s>>>(x, x1, prims, arity, n, pad, boxes.p);
  k_bounds_init<<<1, 32, 0, s>>>(bounds.p);
  k_bounds<<<nblk(n), TPB, 0, s>>>(boxes.p, n, bounds.p);
  k_morton<<<nblk(n), TPB, 0, s>>>(boxes.p, n, bounds.p, keys.p, idx.p);
  size_t bytes = 0;
  if ((e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.p, keys_sorted.p, idx.p, order.p, n, 0, 64, s))) return e;
  if ((e = tmp.reserve(bytes))) return e;
  if ((e = cub::DeviceRadixSort::SortPairs(tmp.p, bytes, keys.p, keys_sorted.p, idx.p, order.p, n, 0, 64, s))) return e;
  k_rank<<<nblk(n), TPB, 0, s>>>(order.p, n, rank.p);
  k_leafv<<<nblk(n), TPB, 0, s>>>(order.p, prims, arity, n, leafv.p);
  if (n > 1) {
    if ((e = cudaMemsetAsync(parent.p, 0xff, sizeof(int) * (2 * n - 1), s))) return e;
    k_karras<<<nblk(n - 1), TPB, 0, s>>>(keys_sorted.p, n, parent.p, inner.p, topo.p);
    if ((e = cudaMemsetAsync(arrive.p, 0, sizeof(int) * n, s))) return e;
    k_top_flags<<<nblk(n - 1), TPB, 0, s>>>(topo.p, n, topflag.p);
    size_t sb = 0;
    if ((e = cub::DeviceScan::ExclusiveSum(nullptr, sb, topflag.p, topnum.p, n - 1, s))) return e;
    if ((e = tmp.reserve(sb))) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp.p, sb, topflag.p, topnum.p, n - 1, s))) return e;
    k_top_records<<<nblk(n - 1), TPB, 0, s>>>(topo.p, inner.p, topnum.p, n, toprec.p, cuts.p);
    k_wide_flags<<<nblk(n - 1), TPB, 0, s>>>(topo.p, n, wflag.p);
    sb = 0;
    if ((e = cub::DeviceScan::ExclusiveSum(nullptr, sb, wflag.p, widx.p, n - 1, s))) return e;
    if ((e = tmp.reserve(sb))) return e;
    if ((e = cub::DeviceScan::ExclusiveSum(tmp.p, sb, wflag.p, widx.p, n - 1, s))) return e;
    if ((e = cudaMemsetAsync(wslot.p, 0xff, sizeof(int) * (2 * n - 1), s))) return e;
    k_wide_topo<<<nblk(n - 1), TPB, 0, s>>>(inner.p, wflag.p, widx.p, n, wide.p, wslot.p);
    launches += 4;
  } else {
    if ((e = cudaMemsetAsync(wslot.p, 0xff, sizeof(int), s))) return e;  // the single leaf is the root
  }
  k_top_count<<<1, 1, 0, s>>>(topflag.p, topnum.p, n, meta.p, cuts.p);
  if ((e = launch_refit(x, x1, pad, s))) return e;
  launches += (n > 1 ? 10 : 8) + (n > RF_CUT ? 1 : 0);
  return cudaGetLastError();
}

// Update the boxes of the last build for new positions (same primitives):
// primitive boxes, then the bottom-up node boxes over the existing topology.
// The candidate set of a query does not depend on the topology, only the
// traversal cost does, so the Morton order of an earlier build stays valid.
cudaError_t Lbvh::refit(const double* x, const double* x1, float pad, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = launch_refit(x, x1, pad, s);
  launches += n > RF_CUT ? 2 : 1;
  return e;
}

// The global arrival counters are zero between refits: the build zeroes them
// and every refit leaves them zero (each node's second arrival resets it).
cudaError_t Lbvh::launch_refit(const double* x, const double* x1, float pad, cudaStream_t s) {
  static_assert(sizeof(RefitSmem) <= 227 * 1024 && sizeof(TopSmem) <= 227 * 1024, "refit tile exceeds shared memory");
  cudaError_t e = cudaFuncSetAttribute(k_refit_cut, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(RefitSmem)));
  if (!e) e = cudaFuncSetAttribute(k_refit_top, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(TopSmem)));
  if (e) return e;
  // SMs of the device (contexts of a batch step on host threads: the
  // function-local static is initialised once, thread-safely; 148 if the
  // query fails)
  static const int sms = [] {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
      cudaGetLastError();
      return 148;
    }
    return n;
  }();
  // grid-stride over the cut list (its length stays on the device): about
  // three subtrees per SM resident at once
  const int grid = std::max(1, std::min(3 * sms, 2 * ((n + 255) / 256)));
  const int cap = top_cap < 0 || top_cap > TOP_MAX ? TOP_MAX : top_cap;
  k_refit_cut<<<grid, RF_TPB, sizeof(RefitSmem), s>>>(x, x1, prims, arity, pad, order.p, n, parent.p, topo.p, cuts.p, meta.p, cap,
                                                      nodes.p, arrive.p, wslot.p, wide.p);
  if (n > RF_CUT) k_refit_top<<<1, TOP_TPB, sizeof(TopSmem), s>>>(meta.p, cap, toprec.p, nodes.p, wslot.p, wide.p);
  return cudaGetLastError();
}

cudaError_t Lbvh::update(const double* x, const double* x1, const int* prims_, int arity_, int n_, float pad, long long epoch_,
                         DevBuf<unsigned char>& tmp, cudaStream_t s) {
  if (epoch_ == epoch && n_ == n && prims_ == prims && arity_ == arity && n > 0) return refit(x, x1, pad, s);
  epoch = epoch_;
  return build(x, x1, prims_, arity_, n_, pad, tmp, s);
}

namespace {
// Sorted box-candidate pairs of a query (capacity grown as needed).
cudaError_t run_query(Lbvh& B, const double* x, const double* x1, int kind, const int* qprims, int nq, float pad, DevBuf<int2>& out,
                      DevBuf<int2>& scratch, DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1, DevBuf<int>& counter,
                      DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s) {
  cudaError_t e;
  *npairs = 0;
  if (B.n == 0 || nq == 0) return cudaSuccess;
  if ((e = counter.reserve(3))) return e;
  if (scratch.n < 1024) if ((e = scratch.reserve(1024))) return e;
  for (int attempt = 0; attempt < 2; ++attempt) {
    int cap = int(scratch.n);
    if ((e = cudaMemsetAsync(counter.p, 0, 3 * sizeof(int), s))) return e;
    k_query<<<nblk(nq), TPB, 0, s>>>(x, x1, qprims, B.qorder, kind, nq, pad, B.n, B.leafv.p, B.rank.p, B.wide.p, B.nodes.p,
                                     scratch.p, counter.p, cap);
    B.launches += 1;
    int cnt2[2] = {0, 0};
    if ((e = cudaMemcpyAsync(cnt2, counter.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    if (cnt2[1]) return cudaErrorLaunchOutOfResources;  // traversal stack overflow (cannot happen with unique keys)
    int cnt = cnt2[0];
    if (cnt < 0 || cnt > (1 << 26)) return cudaErrorMemoryAllocation;  // > 64M candidate pairs: refuse instead of exhausting memory
    if (cnt <= cap) { *npairs = cnt; break; }
    if ((e = scratch.reserve(size_t(cnt) + size_t(cnt) / 4))) return e;
  }
  int m = *npairs;
  if (m == 0) return cudaSuccess;
  if ((e = k0.reserve(m))) return e;
  if ((e = k1.reserve(m))) return e;
  if ((e = out.reserve(m))) return e;
  k_pair_keys<<<nblk(m), TPB, 0, s>>>(scratch.p, m, k0.p);
  B.launches += 1;
  size_t bytes = 0;
  if ((e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0.p, k1.p, scratch.p, out.p, m, 0, 64, s))) return e;
  if ((e = tmp.reserve(bytes))) return e;
  if ((e = cub::DeviceRadixSort::SortPairs(tmp.p, bytes, k0.p, k1.p, scratch.p, out.p, m, 0, 64, s))) return e;
  return cudaGetLastError();
}
}  // namespace

// Query the hierarchy; returns the sorted (query, primitive) pairs in `out`
// (capacity grown as needed) and their number in *npairs.
cudaError_t Lbvh::query(const double* x, const double* x1, int kind, const int* qprims, int nq, float pad, DevBuf<int2>& out,
                        DevBuf<int2>& scratch, DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1,
                        DevBuf<int>& counter, DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s) {
  return run_query(*this, x, x1, kind, qprims, nq, pad, out, scratch, k0, k1, counter, tmp, npairs, s);
}

cudaError_t Lbvh::contacts_launch(const double* x, int kind, const int* qprims, int nq, float pad, double gap, DevBuf<int2>& scratch,
                                  DevBuf<int>& counter, cudaStream_t s) {
  cudaError_t e;
  if ((e = counter.reserve(3))) return e;
  if ((e = cudaMemsetAsync(counter.p, 0, 3 * sizeof(int), s))) return e;
  if (n == 0 || nq == 0) return cudaSuccess;
  if (scratch.n < 1024) if ((e = scratch.reserve(1024))) return e;
  if ((e = surv.reserve(scratch.n))) return e;
  const int cap = int(scratch.n);
  k_query<<<nblk(nq), TPB, 0, s>>>(x, nullptr, qprims, qorder, kind, nq, pad, n, leafv.p, rank.p, wide.p, nodes.p, scratch.p, counter.p, cap);
  k_pairs_gap<<<NARROW_GRID, TPB, 0, s>>>(scratch.p, counter.p, cap, kind, prims, qprims, x, gap, surv.p, counter.p + 2);
  launches += 2;
  return cudaGetLastError();
}

cudaError_t Lbvh::contacts_finish(const int count[3], DevBuf<int2>& out, DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1,
                                  DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s) {
  cudaError_t e;
  *npairs = 0;
  if (count[1]) return cudaErrorLaunchOutOfResources;  // traversal stack overflow (cannot happen with unique keys)
  const int m = count[2];
  if (m < 0 || m > int(surv.n)) return cudaErrorInvalidValue;
  if (m == 0) return cudaSuccess;
  if ((e = k0.reserve(m))) return e;
  if ((e = k1.reserve(m))) return e;
  if ((e = out.reserve(m))) return e;
  k_pair_keys<<<nblk(m), TPB, 0, s>>>(surv.p, m, k0.p);
  launches += 1;
  size_t bytes = 0;
  if ((e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, k0.p, k1.p, surv.p, out.p, m, 0, 64, s))) return e;
  if ((e = tmp.reserve(bytes))) return e;
  if ((e = cub::DeviceRadixSort::SortPairs(tmp.p, bytes, k0.p, k1.p, surv.p, out.p, m, 0, 64, s))) return e;
  *npairs = m;
  return cudaGetLastError();
}

cudaError_t Lbvh::query_toi(const double* x, const double* x1, const double* ext, int kind, const int* qprims, int nq, float pad,
                            double eta_min, double near, unsigned long long* toi, DevBuf<int2>& scratch, DevBuf<int>& counter,
                            int* overflow, cudaStream_t s) {
  if (n == 0 || nq == 0) return cudaSuccess;
  cudaError_t e;
  if ((e = counter.reserve(3))) return e;
  if (scratch.n < 1024) if ((e = scratch.reserve(1024))) return e;
  const int cap = int(scratch.n);
  if ((e = cudaMemsetAsync(counter.p, 0, 3 * sizeof(int), s))) return e;
  k_query<<<nblk(nq), TPB, 0, s>>>(x, x1, qprims, qorder, kind, nq, pad, n, leafv.p, rank.p, wide.p, nodes.p, scratch.p, counter.p, cap);
  k_pairs_toi<<<NARROW_GRID, TPB, 0, s>>>(scratch.p, counter.p, cap, kind, prims, qprims, x, x1, ext, pad, eta_min, near, toi, overflow);
  launches += 2;
  return cudaGetLastError();
}

cudaError_t Lbvh::contacts_from(const double* x, int kind, const int* qprims, double gap, DevBuf<int2>& cand, DevBuf<int>& counter,
                                cudaStream_t s) {
  cudaError_t e;
  if ((e = counter.reserve(3))) return e;
  if (n == 0 || cand.n == 0) return cudaMemsetAsync(counter.p, 0, 3 * sizeof(int), s);
  if ((e = cudaMemsetAsync(counter.p + 2, 0, sizeof(int), s))) return e;
  if ((e = surv.reserve(cand.n))) return e;
  k_pairs_gap<<<NARROW_GRID, TPB, 0, s>>>(cand.p, counter.p, int(cand.n), kind, prims, qprims, x, gap, surv.p, counter.p + 2);
  launches += 1;
  return cudaGetLastError();
}

// Edge-triangle crossings at x over this triangle hierarchy (built at x):
// queries are the ne edges (their boxes inflated by pad, which only adds
// candidates for the exact test). One host round trip per attempt; the
// candidate list grows once if it overflowed.
cudaError_t Lbvh::count_crossings(const double* x, const int* edges, int ne, float pad, DevBuf<int2>& scratch, DevBuf<int>& counter,
                                  DevBuf<unsigned long long>& total, long long* crossings, cudaStream_t s) {
  cudaError_t e;
  *crossings = 0;
  if (n == 0 || ne == 0) return cudaSuccess;
  if ((e = counter.reserve(3))) return e;
  if ((e = total.reserve(1))) return e;
  if (scratch.n < 1024) if ((e = scratch.reserve(1024))) return e;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const int cap = int(scratch.n);
    if ((e = cudaMemsetAsync(counter.p, 0, 3 * sizeof(int), s))) return e;
    if ((e = cudaMemsetAsync(total.p, 0, sizeof(unsigned long long), s))) return e;
    k_query<<<nblk(ne), TPB, 0, s>>>(x, nullptr, edges, qorder, 2, ne, pad, n, leafv.p, rank.p, wide.p, nodes.p, scratch.p, counter.p, cap);
    k_pairs_cross<<<NARROW_GRID, TPB, 0, s>>>(scratch.p, counter.p, cap, prims, edges, x, total.p);
    launches += 2;
    int cnt2[2] = {0, 0};
    unsigned long long got = 0;
    if ((e = cudaMemcpyAsync(cnt2, counter.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaMemcpyAsync(&got, total.p, sizeof(got), cudaMemcpyDeviceToHost, s))) return e;
    if ((e = cudaStreamSynchronize(s))) return e;
    if (cnt2[1]) return cudaErrorLaunchOutOfResources;  // traversal stack overflow (cannot happen with unique keys)
    if (cnt2[0] < 0 || cnt2[0] > (1 << 26)) return cudaErrorMemoryAllocation;
    if (cnt2[0] <= cap) { *crossings = (long long)got; return cudaSuccess; }
    if ((e = scratch.reserve(size_t(cnt2[0]) + size_t(cnt2[0]) / 4))) return e;
  }
  return cudaErrorMemoryAllocation;
}

}  // namespace ando
