// lbvh.cuh -- linear BVH over triangles or edges (definitions in lbvh.cu).
#pragma once

#include <cfloat>

#include "common.cuh"
#include "devbuf.cuh"

namespace ando {

struct LbvhBox { float lo[3], hi[3]; };

struct Lbvh {
  int n = 0;                    // primitives
  int arity = 0;
  long long epoch = -1;         // caller's epoch of the last full build (update)
  const int* prims = nullptr;   // arity * n vertex indices (device)
  DevBuf<LbvhBox> boxes, nodes; // primitive boxes; node boxes (internal [0,n-1), leaves [n-1, 2n-1))
  DevBuf<unsigned long long> keys, keys_sorted;
  DevBuf<int> idx, order, left, right, parent, arrive, bounds;
  long long launches = 0;

  cudaError_t reserve_prims(int n);
  // x1 (may be null): boxes swept from positions x to x1
  cudaError_t build(const double* x, const double* x1, const int* prims, int arity, int n, float pad, DevBuf<unsigned char>& tmp, cudaStream_t s);
  // new boxes over the last build's topology (same primitives)
  cudaError_t refit(const double* x, const double* x1, float pad, cudaStream_t s);
  // full build once per caller epoch, refit otherwise
  cudaError_t update(const double* x, const double* x1, const int* prims, int arity, int n, float pad, long long epoch,
                     DevBuf<unsigned char>& tmp, cudaStream_t s);
  // kind 0: vertices against triangles; kind 1: edges against edges.
  cudaError_t query(const double* x, const double* x1, int kind, const int* qprims, int nq, float pad, DevBuf<int2>& out, DevBuf<int2>& scratch,
                    DevBuf<unsigned long long>& k0, DevBuf<unsigned long long>& k1, DevBuf<int>& counter,
                    DevBuf<unsigned char>& tmp, int* npairs, cudaStream_t s);
};

}  // namespace ando
