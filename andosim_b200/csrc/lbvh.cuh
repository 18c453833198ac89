// lbvh.cuh -- linear BVH over triangles or edges (definitions in lbvh.cu).
#pragma once

#include <cfloat>

#include "common.cuh"
#include "devbuf.cuh"

namespace ando {

struct LbvhBox { float lo[3], hi[3]; };
// Internal node of the binary hierarchy: its children (internal index, or
// n - 1 + sorted leaf position) and the last sorted leaf position under each.
struct alignas(16) LbvhInner { int lc, rc, lmax, rmax; };
// Four-wide node as the traversal reads it (128 bytes, one line): the binary
// hierarchy with every other level folded into its parent. Slots 2s and
// 2s + 1 hold side s of the binary node: its child when that is a leaf (slot
// 2s + 1 then empty), else the child's two children. Per slot the box
// (lo[3], hi[3]), the child (a four-wide node index >= 0, or a sorted leaf
// position p as -(p + 1)) and the last sorted leaf position under it (prunes
// the self query). An empty slot has an empty box and bound INT_MIN.
struct alignas(128) LbvhWide { float box[4][6]; int child[4], cmax[4]; };

struct Lbvh {
  int n = 0;                    // primitives
  int arity = 0;
  long long epoch = -1;         // caller's epoch of the last full build (update)
  const int* prims = nullptr;   // arity * n vertex indices (device)
  // Order in which query threads take their queries (a permutation of the
  // nq queries, device; null: identity). A spatially coherent order keeps the
  // 32 traversals of a warp on similar paths; results do not depend on it.
  const int* qorder = nullptr;
  DevBuf<LbvhBox> boxes, nodes; // primitive boxes; node boxes (internal [0,n-1), leaves [n-1, 2n-1))
  DevBuf<LbvhInner> inner;      // n-1 internal nodes: children and their last leaves (the build's topology)
  DevBuf<LbvhWide> wide;        // four-wide nodes: topology at build time, boxes by every refit
  DevBuf<int> wflag, widx;      // per internal node: 1 at even depth (a four-wide node), its four-wide index
  DevBuf<int> wslot;            // per node: 4 * four-wide index + slot where its box is kept, -1 if nowhere
  DevBuf<unsigned long long> keys, keys_sorted;
  DevBuf<int> idx, order, parent, arrive, bounds;
  DevBuf<int> rank;             // sorted leaf position of each primitive (inverse of order)
  DevBuf<int4> topo;            // per internal node: first leaf, split, last leaf, parent
  DevBuf<int4> leafv;           // per sorted leaf: primitive and its vertices (-1 past the arity)
  // refit schedule made at build time: nodes above the cut (flags, numbers,
  // records), the cut subtrees as leaf ranges, meta = {top nodes, cut entries}
  DevBuf<int> topflag, topnum, meta;
  DevBuf<int4> toprec;
  DevBuf<int2> cuts;
  DevBuf<int2> surv;            // candidates kept by the narrow phase of contacts_launch
  long long launches = 0;
  // top nodes the one-CTA refit finishes in shared memory (at most 4096;
  // negative: 4096); above that the cut kernel climbs on with global counters
  int top_cap = -1;

  cudaError_t reserve_prims(int n);
  // x1 (may be null): boxes swept from positions x to x1
  cudaError_t build(const double* x, const double* x1, const int* prims, int arity, int n, float pad, DevBuf<unsigned char>& tmp, cudaStream_t s);
  // new boxes over the last build's topology (same primitives)
  cudaError_t refit(const double* x, const double* x1, float pad, cudaStream_t s);
  cudaError_t launch_refit(const double* x, const double* x1, float pad, cudaStream_t s);
  // full build once per caller epoch, refit otherwise
  cudaError_t update(const double* x, const double* x1, const int* prims, int arity, int n, float pad, long long epoch,
                     DevBuf<unsigned char>& tmp, cudaStream_t s);
  // kind 0: vertices against triangles; kind 1: edges against edges; kind 2:
  // edges against triangles (count_crossings).
  // Sorted candidate pairs (boxes overlap) in `out`, their number in *npairs.
  cudaError_t query(const double* x, const double* x1, int kind, const int* qprims, int nq, float pad, DevBuf<int2>& out, DevBuf<int2>& scratch,
                    DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1, DevBuf<int>& counter,
                    DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s);
  // The candidates (boxes at x inflated by pad) whose FP64 distance at x is
  // below `gap`, sorted, in two halves so that several queries share one
  // host round trip: the launch (traversal and narrow phase; counter[0] = box
  // candidates, counter[1] = stack overflows, counter[2] = contacts) and,
  // once the caller has read the counter, the sort of the contacts into
  // `out`. A launch whose candidates overflowed `scratch` (counter[0] >
  // scratch.n at launch) must be grown and launched again before finishing.
  cudaError_t contacts_launch(const double* x, int kind, const int* qprims, int nq, float pad, double gap, DevBuf<int2>& scratch,
                              DevBuf<int>& counter, cudaStream_t s);
  cudaError_t contacts_finish(const int count[3], DevBuf<int2>& out, DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1,
                              DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s);
  // min over the swept-box candidates (x -> x1 = x + ext) of the pair's
  // conservative time of impact, min-reduced into *toi (IEEE bits of a
  // non-negative double) on the device, with no host round trip: the
  // candidate count stays on the device. With pad > 0 the boxes are inflated
  // by pad for the traversal (the list then also serves contacts_from at any
  // position between x and x1) and only the pairs whose boxes overlap without
  // it bound the step, so the result does not depend on the pad. When the
  // candidates overflow `scratch`, *overflow is raised to the count needed and
  // *toi is not lowered; the caller grows `scratch` and runs the pass again.
  cudaError_t query_toi(const double* x, const double* x1, const double* ext, int kind, const int* qprims, int nq, float pad,
                        double eta_min, double near, unsigned long long* toi, DevBuf<int2>& scratch, DevBuf<int>& counter, int* overflow,
                        cudaStream_t s);
  // The first half of a contact query (contacts_launch) over the candidate
  // list that a query_toi pass with the same counter left in `cand`: the
  // pairs whose FP64 distance at x is below `gap`, counter[2] = how many;
  // contacts_finish sorts them. Gives the contacts_launch result when every
  // vertex at x lies between the pass's x and x1 and its pad is at least the
  // contact query's.
  cudaError_t contacts_from(const double* x, int kind, const int* qprims, double gap, DevBuf<int2>& cand, DevBuf<int>& counter,
                            cudaStream_t s);
  // Edge-triangle crossings at x (this hierarchy is over triangles, built at
  // x): the (edge, triangle) pairs that share no vertex and where the edge's
  // segment passes through the triangle, by an exact FP64 test of every
  // candidate whose boxes (the edge's inflated by pad) overlap.
  cudaError_t count_crossings(const double* x, const int* edges, int ne, float pad, DevBuf<int2>& scratch, DevBuf<int>& counter,
                              DevBuf<unsigned long long>& total, long long* crossings, cudaStream_t s);
};

}  // namespace ando
