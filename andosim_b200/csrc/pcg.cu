// pcg.cu -- block-Jacobi preconditioned conjugate gradients as one persistent
// cooperative kernel (replaces PCGSolver::solve, pcg_solver.cpp:8-146).
//
// Same iteration as the reference: x0 = 0, r = b, block-Jacobi z = P r,
// stop when |r|_inf / |b|_inf < tol (or |r|_inf when |b|_inf < 1e-16), fail
// when |p^T A p| < 1e-16. Vectors and the BSR matrix are FP32; every dot
// product and norm is accumulated in FP64 and reduced in a fixed order, so
// results are bitwise reproducible run to run.
//
// Per iteration there are two grid barriers:
//   A: p_new = z + beta p_old (recomputed on the fly for gathered columns),
//      Ap = A p_new with one warp per block row, partial p^T Ap
//   B: x += alpha p, r -= alpha Ap, z = P r, partial r^T z and |r|_inf
// The barrier is bounded (common.cuh): on timeout the kernel reports
// PCG_TIMEOUT instead of spinning forever.
#include "kernels.cuh"

namespace ando {

namespace {

constexpr int PCG_TPB = 512;
constexpr int PCG_WARPS = PCG_TPB / 32;

__device__ inline double block_sum(double v, double* sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = l < PCG_WARPS ? sh[l] : 0.0;
    for (int o = 16; o; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (l == 0) sh[0] = r;
  }
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}
__device__ inline double block_max(double v, double* sh) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (w == 0) {
    r = l < PCG_WARPS ? sh[l] : 0.0;
    for (int o = 16; o; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    if (l == 0) sh[0] = r;
  }
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}
// Every CTA reduces the per-CTA partials in the same order -> identical scalars everywhere.
__device__ inline double grid_sum(const double* part, int n, double* sh) {
  double v = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) v += part[k];
  return block_sum(v, sh);
}
__device__ inline double grid_max(const double* part, int n, double* sh) {
  double v = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) v = fmax(v, part[k]);
  return block_max(v, sh);
}

__device__ inline void p_at(const float* z, const float* pold, float beta, bool first, int j, float& p0, float& p1, float& p2) {
  float z0 = z[3 * j], z1 = z[3 * j + 1], z2 = z[3 * j + 2];
  if (first) { p0 = z0; p1 = z1; p2 = z2; return; }
  p0 = z0 + beta * pold[3 * j]; p1 = z1 + beta * pold[3 * j + 1]; p2 = z2 + beta * pold[3 * j + 2];
}

__global__ void __launch_bounds__(PCG_TPB) k_pcg(PcgArgs a) {
  Ctrl* ctrl = a.ctrl;
  if (ctrl->converged) return;
  __shared__ double sh[PCG_WARPS + 1];
  const int V = a.V;
  const unsigned nb = gridDim.x;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  double* part_pap = a.partials;
  double* part_rz = a.partials + nb;
  double* part_rinf = a.partials + 2 * nb;

  // init: x = 0, r = b, z = P r
  double rz_loc = 0.0, binf_loc = 0.0;
  for (int i = tid; i < V; i += nthreads) {
    float r0 = a.b[3 * i], r1 = a.b[3 * i + 1], r2 = a.b[3 * i + 2];
    const float* P = a.P + 9 * (long long)i;
    float z0 = P[0] * r0 + P[1] * r1 + P[2] * r2, z1 = P[3] * r0 + P[4] * r1 + P[5] * r2, z2 = P[6] * r0 + P[7] * r1 + P[8] * r2;
    a.x[3 * i] = 0.f; a.x[3 * i + 1] = 0.f; a.x[3 * i + 2] = 0.f;
    a.r[3 * i] = r0; a.r[3 * i + 1] = r1; a.r[3 * i + 2] = r2;
    a.z[3 * i] = z0; a.z[3 * i + 1] = z1; a.z[3 * i + 2] = z2;
    rz_loc += double(r0) * z0 + double(r1) * z1 + double(r2) * z2;
    binf_loc = fmax(binf_loc, fmax(fabs(double(r0)), fmax(fabs(double(r1)), fabs(double(r2)))));
  }
  rz_loc = block_sum(rz_loc, sh);
  binf_loc = block_max(binf_loc, sh);
  if (threadIdx.x == 0) { part_rz[blockIdx.x] = rz_loc; part_rinf[blockIdx.x] = binf_loc; }
  bool ok = grid_sync(&ctrl->bar_count, &ctrl->bar_gen, &ctrl->bar_err, nb);
  int status = PCG_MAXIT, iters = 0;
  double rel = 0.0;
  if (!ok) status = PCG_TIMEOUT;
  double rz = ok ? grid_sum(part_rz, nb, sh) : 0.0;
  double binf = ok ? grid_max(part_rinf, nb, sh) : 0.0;
  if (ok) {
    rel = binf < 1e-16 ? binf : 1.0;
    if (rel < double(a.tol)) status = PCG_OK;
  }
  float* pold = a.p0;
  float* pnew = a.p1;
  float beta = 0.f;
  bool first = true;
  const int lane = threadIdx.x & 31;
  const int gwarp = tid >> 5, nwarps = nthreads >> 5;
  const int comp = lane >> 3, bi = lane & 7;
  for (int it = 0; ok && status == PCG_MAXIT && it < a.max_iters; ++it) {
    // ---- phase A: p_new, Ap = A p_new, p^T Ap
    double pap_loc = 0.0;
    for (int row = gwarp; row < V; row += nwarps) {
      float acc = 0.f;
      int s0 = a.rowptr[row], s1 = a.rowptr[row + 1];
      for (int k0 = s0; k0 < s1; k0 += 8) {
        int k = k0 + bi;
        if (comp < 3 && k < s1) {
          int col = a.cols[k];
          const float* h = a.val + 9 * (long long)k + 3 * comp;
          float q0, q1, q2; p_at(a.z, pold, beta, first, col, q0, q1, q2);
          acc += h[0] * q0 + h[1] * q1 + h[2] * q2;
        }
      }
      if (a.xbegin) {
        int e0 = a.xbegin[row], e1 = a.xend[row];
        for (int k0 = e0; k0 < e1; k0 += 8) {
          int k = k0 + bi;
          if (comp < 3 && k < e1) {
            int col = a.xcols[k];
            const float* h = a.xval + 9 * (long long)k + 3 * comp;
            float q0, q1, q2; p_at(a.z, pold, beta, first, col, q0, q1, q2);
            acc += h[0] * q0 + h[1] * q1 + h[2] * q2;
          }
        }
      }
      acc += __shfl_xor_sync(0xffffffffu, acc, 4);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      float y0 = __shfl_sync(0xffffffffu, acc, 0), y1 = __shfl_sync(0xffffffffu, acc, 8), y2 = __shfl_sync(0xffffffffu, acc, 16);
      if (lane == 0) {
        float q0, q1, q2; p_at(a.z, pold, beta, first, row, q0, q1, q2);
        pnew[3 * row] = q0; pnew[3 * row + 1] = q1; pnew[3 * row + 2] = q2;
        a.Ap[3 * row] = y0; a.Ap[3 * row + 1] = y1; a.Ap[3 * row + 2] = y2;
        pap_loc += double(q0) * y0 + double(q1) * y1 + double(q2) * y2;
      }
    }
    pap_loc = block_sum(pap_loc, sh);
    if (threadIdx.x == 0) part_pap[blockIdx.x] = pap_loc;
    ok = grid_sync(&ctrl->bar_count, &ctrl->bar_gen, &ctrl->bar_err, nb);
    if (!ok) { status = PCG_TIMEOUT; break; }
    double pap = grid_sum(part_pap, nb, sh);
    iters = it + 1;
    if (fabs(pap) < 1e-16) { status = PCG_NOT_SPD; break; }
    float alpha = float(rz / pap);
    // ---- phase B: x, r, z, r^T z, |r|_inf
    double rz_new_loc = 0.0, rinf_loc = 0.0;
    for (int i = tid; i < V; i += nthreads) {
      float p0 = pnew[3 * i], p1 = pnew[3 * i + 1], p2 = pnew[3 * i + 2];
      float q0 = a.Ap[3 * i], q1 = a.Ap[3 * i + 1], q2 = a.Ap[3 * i + 2];
      a.x[3 * i] += alpha * p0; a.x[3 * i + 1] += alpha * p1; a.x[3 * i + 2] += alpha * p2;
      float r0 = a.r[3 * i] - alpha * q0, r1 = a.r[3 * i + 1] - alpha * q1, r2 = a.r[3 * i + 2] - alpha * q2;
      a.r[3 * i] = r0; a.r[3 * i + 1] = r1; a.r[3 * i + 2] = r2;
      const float* P = a.P + 9 * (long long)i;
      float z0 = P[0] * r0 + P[1] * r1 + P[2] * r2, z1 = P[3] * r0 + P[4] * r1 + P[5] * r2, z2 = P[6] * r0 + P[7] * r1 + P[8] * r2;
      a.z[3 * i] = z0; a.z[3 * i + 1] = z1; a.z[3 * i + 2] = z2;
      rz_new_loc += double(r0) * z0 + double(r1) * z1 + double(r2) * z2;
      rinf_loc = fmax(rinf_loc, fmax(fabs(double(r0)), fmax(fabs(double(r1)), fabs(double(r2)))));
    }
    rz_new_loc = block_sum(rz_new_loc, sh);
    rinf_loc = block_max(rinf_loc, sh);
    if (threadIdx.x == 0) { part_rz[blockIdx.x] = rz_new_loc; part_rinf[blockIdx.x] = rinf_loc; }
    ok = grid_sync(&ctrl->bar_count, &ctrl->bar_gen, &ctrl->bar_err, nb);
    if (!ok) { status = PCG_TIMEOUT; break; }
    double rz_new = grid_sum(part_rz, nb, sh);
    double rinf = grid_max(part_rinf, nb, sh);
    rel = binf < 1e-16 ? rinf : rinf / binf;
    if (rel < double(a.tol)) { status = PCG_OK; break; }
    beta = float(rz_new / rz);
    rz = rz_new;
    first = false;
    float* t = pold; pold = pnew; pnew = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ctrl->pcg_iters = iters;
    ctrl->pcg_status = status;
    ctrl->pcg_converged = status == PCG_OK ? 1 : 0;
    ctrl->pcg_rel = rel;
  }
}

// ------------------------------------------------------------ scaled PCG
// CG on the block-scaled system A^ = L^-1 A L^-T (A_ii = L_i L_i^T), used by
// the CORRECTED step. With the identity as preconditioner on A^ this is the
// block-Jacobi PCG of the reference, iterate for iterate in exact arithmetic:
// x = L^-T x^, r = L r^. The stopping test is relative like the reference's
// (pcg_solver.cpp:8-75) but taken on the block-scaled residual,
// max_i |r^_i| < tol * max_i |b^_i|: on the unscaled residual a few contact or
// pin rows whose forces are orders of magnitude above the rest set the
// tolerance for every other row, and the solve stops with a direction that is
// poor everywhere else. Scaled by L^-1, rows are compared in displacement-
// like units. The learned and block-Jacobi solves stop on the same test.
//
// LEARNED: z = S r with S a symmetric positive definite block matrix on the
// static pattern (the learned approximate inverse of A^), applied as
// S_ij = coef_ij A^_ij off the diagonal plus its diagonal blocks. Phase B then
// is a second row product over A^'s values; it gathers r - alpha Ap from the
// neighbours, so
// the iteration still needs only two grid barriers (r ping-pongs between two
// buffers because neighbours read the old values). r^T z <= 0 (S lost
// definiteness) or no new best residual for `stall_window` iterations ends
// the solve with PCG_PRECOND / PCG_STALL, and the caller redoes it with
// block-Jacobi.

// Sliced-ELL layout of the static pattern (SELL-32): rows in chunks of 32,
// chunk c holding W_c = (chunk_off[c+1] - chunk_off[c]) / 32 block slots per
// row; slot k of row lane l sits at block index chunk_off[c] + 32 k + l, its
// column in sell_col (-1 pads a short row) and its 9 values at
// 9 (chunk_off[c] + 32 k) + 32 q + l, q = 0..8. One thread per block row: a
// warp's 32 rows read every value and column load as one coalesced 128-byte
// line, and 32 rows' gathers are in flight at once (sell_row_u below).

// Row stride S of the scaled PCG's vectors r, r2, z, p0, p1 and Ap: 4 (one
// float4 per row, the fourth lane unused, so a neighbour's entry is one
// 16-byte load) in the block-Jacobi solve, 3 in the learned one, where the
// larger vectors measured slower (19.5 against 18.7 us per iteration at
// C4). Each solve initialises its vectors, so the two layouts share buffers
// of 4V floats.
template <int S> __device__ inline float4 ld4(const float* v, int j) {
  if (S == 4) return reinterpret_cast<const float4*>(v)[j];
  return make_float4(v[3 * j], v[3 * j + 1], v[3 * j + 2], 0.f);
}
template <int S> __device__ inline void st4(float* v, int j, float a, float b, float c) {
  if (S == 4) reinterpret_cast<float4*>(v)[j] = make_float4(a, b, c, 0.f);
  else { v[3 * j] = a; v[3 * j + 1] = b; v[3 * j + 2] = c; }
}

template <int S> struct GatherP {  // p = z + beta p_old
  const float* z; const float* pold; float beta; bool first;
  __device__ void operator()(int j, float& q0, float& q1, float& q2) const {
    const float4 zz = ld4<S>(z, j);
    if (first) { q0 = zz.x; q1 = zz.y; q2 = zz.z; return; }
    const float4 pp = ld4<S>(pold, j);
    q0 = zz.x + beta * pp.x; q1 = zz.y + beta * pp.y; q2 = zz.z + beta * pp.z;
  }
};
struct GatherV {  // plain vector
  const float* v;
  __device__ void operator()(int j, float& q0, float& q1, float& q2) const { q0 = v[3 * j]; q1 = v[3 * j + 1]; q2 = v[3 * j + 2]; }
};
template <int S> struct GatherR {  // r - alpha Ap
  const float* r; const float* Ap; float alpha;
  __device__ void operator()(int j, float& q0, float& q1, float& q2) const {
    const float4 rr = ld4<S>(r, j), aa = ld4<S>(Ap, j);
    q0 = rr.x - alpha * aa.x; q1 = rr.y - alpha * aa.y; q2 = rr.z - alpha * aa.z;
  }
};

// Fixed-order reductions over per-slice partials. Each warp owns whole
// 32-row slices and writes one partial per slice (a xor butterfly, whose
// result is the same in every lane); after the grid barrier every CTA adds
// the partials in one order that does not depend on the launch shape:
// s_t = sum_k part[t + 1024 k] for t < 1024, then butterflies over 32 groups
// of 32. So the tuned launch shape never changes a result bit.
__device__ inline double warp_sum(double v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ inline double warp_max(double v) {
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
constexpr int RED_T = 1024;
struct RedSmem { double s[RED_T + 32]; double m[RED_T + 32]; };

// sum of part[0, n) and (with MAX) max of pm[0, n), identical in every CTA
template <bool MAX>
__device__ inline void fixed_reduce(const double* part, const double* pm, int n, RedSmem& sh, double& sum, double& mx) {
  for (int t = threadIdx.x; t < RED_T; t += blockDim.x) {
    double s = 0.0, m = 0.0;
    for (int k = t; k < n; k += RED_T) {
      s += __ldcg(part + k);  // written by other CTAs before the barrier: read from L2
      if (MAX) m = fmax(m, __ldcg(pm + k));
    }
    sh.s[t] = s;
    if (MAX) sh.m[t] = m;
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int g = w; g < 32; g += nw) {
    double v = warp_sum(sh.s[32 * g + l]);
    if (l == 0) sh.s[RED_T + g] = v;
    if (MAX) {
      double u = warp_max(sh.m[32 * g + l]);
      if (l == 0) sh.m[RED_T + g] = u;
    }
  }
  __syncthreads();
  sum = warp_sum(sh.s[RED_T + l]);
  mx = MAX ? warp_max(sh.m[RED_T + l]) : 0.0;
  __syncthreads();  // sh is reused by the next reduction
}

// a += H q for one 3x3 block (row-major, entries h(e) = h[e * stride]), with
// the FMA order written out so that every product variant rounds alike.
template <int STRIDE>
__device__ inline void block_fma(const float* h, float q0, float q1, float q2, float& a0, float& a1, float& a2) {
  a0 = __fmaf_rn(h[2 * STRIDE], q2, __fmaf_rn(h[1 * STRIDE], q1, __fmaf_rn(h[0], q0, a0)));
  a1 = __fmaf_rn(h[5 * STRIDE], q2, __fmaf_rn(h[4 * STRIDE], q1, __fmaf_rn(h[3 * STRIDE], q0, a1)));
  a2 = __fmaf_rn(h[8 * STRIDE], q2, __fmaf_rn(h[7 * STRIDE], q1, __fmaf_rn(h[6 * STRIDE], q0, a2)));
}

// One row of the SELL-32 product. U > 1 loads the column indices of U slots
// ahead of their gathers (more loads in flight per thread, more registers);
// the sum runs over k = 0, 1, ... with the same FMAs for every U.
template <int U, class Vec>
__device__ inline void sell_row_u(int row, const int* chunk_off, const int* sell_col, const float* val, const int* xbegin, const int* xend,
                                  const int* xcols, const float* xval, const Vec& vec, float& y0, float& y1, float& y2) {
  const int c = row >> 5, l = row & 31;
  const int b0 = chunk_off[c], w = (chunk_off[c + 1] - b0) >> 5;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  if (U == 1) {
    for (int k = 0; k < w; ++k) {
      const int slot = b0 + 32 * k;
      const int col = sell_col[slot + l];
      if (col < 0) continue;
      float q0, q1, q2; vec(col, q0, q1, q2);
      block_fma<32>(val + 9ll * slot + l, q0, q1, q2, a0, a1, a2);
    }
  } else {
#pragma unroll 1
    for (int k = 0; k < w; k += U) {
      int col[U];
#pragma unroll
      for (int u = 0; u < U; ++u) col[u] = k + u < w ? sell_col[b0 + 32 * (k + u) + l] : -1;
      float q[U][3];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) vec(col[u], q[u][0], q[u][1], q[u][2]);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) block_fma<32>(val + 9ll * (b0 + 32 * (k + u)) + l, q[u][0], q[u][1], q[u][2], a0, a1, a2);
    }
  }
  if (xbegin) {
    for (int e = xbegin[row]; e < xend[row]; ++e) {
      float q0, q1, q2; vec(xcols[e], q0, q1, q2);
      block_fma<1>(xval + 9ll * e, q0, q1, q2, a0, a1, a2);
    }
  }
  y0 = a0; y1 = a1; y2 = a2;
}

// One row of z = S g with S_ij = coef_ij A^_ij off the diagonal and S_ii =
// Sdiag_i: the SELL-32 product over A^'s static slots (the values phase A
// has just read) with each gathered g_j scaled by its slot's coefficient,
// the row's own slot skipped, then the diagonal block. The same FMA order
// for every U.
template <int U, class Vec>
__device__ inline void sell_row_S(int row, const int* chunk_off, const int* sell_col, const float* val, const float* coef, const float* Sdiag,
                                  const Vec& vec, float& y0, float& y1, float& y2) {
  const int c = row >> 5, l = row & 31;
  const int b0 = chunk_off[c], w = (chunk_off[c + 1] - b0) >> 5;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  if (U == 1) {
    for (int k = 0; k < w; ++k) {
      const int slot = b0 + 32 * k;
      const int col = sell_col[slot + l];
      if (col < 0 || col == row) continue;
      const float cf = coef[slot + l];
      float q0, q1, q2; vec(col, q0, q1, q2);
      block_fma<32>(val + 9ll * slot + l, cf * q0, cf * q1, cf * q2, a0, a1, a2);
    }
  } else {
#pragma unroll 1
    for (int k = 0; k < w; k += U) {
      int col[U];
      float cf[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        col[u] = k + u < w ? sell_col[b0 + 32 * (k + u) + l] : -1;
        if (col[u] == row) col[u] = -1;
        cf[u] = col[u] >= 0 ? coef[b0 + 32 * (k + u) + l] : 0.f;
      }
      float q[U][3];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) vec(col[u], q[u][0], q[u][1], q[u][2]);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (col[u] >= 0) block_fma<32>(val + 9ll * (b0 + 32 * (k + u)) + l, cf[u] * q[u][0], cf[u] * q[u][1], cf[u] * q[u][2], a0, a1, a2);
    }
  }
  float g0, g1, g2; vec(row, g0, g1, g2);
  block_fma<1>(Sdiag + 9ll * row, g0, g1, g2, a0, a1, a2);
  y0 = a0; y1 = a1; y2 = a2;
}

constexpr int SCALED_MAX_TPB = 1024;

template <bool LEARNED, int U>
__global__ void __launch_bounds__(SCALED_MAX_TPB) k_pcg_scaled(PcgScaledArgs a) {
  Ctrl* ctrl = a.ctrl;
  if (ctrl->converged) return;
  if (!LEARNED && a.fallback) {
    // every CTA reads the learned solve's status before the first grid
    // barrier; it is rewritten only after one
    const int st = ctrl->pcg_status;
    if (st == PCG_OK || st == PCG_TIMEOUT) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->fallback_ran = 1;
  }
  __shared__ RedSmem sh;
  constexpr int S = LEARNED ? 3 : 4;  // row stride of r, z, p, Ap
  const int V = a.V, ns = (V + 31) >> 5;
  const unsigned nb = gridDim.x;
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, W = (gridDim.x * blockDim.x) >> 5;
  double* part_pap = a.partials;
  double* part_rz = a.partials + ns;
  double* part_rinf = a.partials + 2 * ns;
  float* r = a.r;
  float* rn = a.r2;
  const float* zsrc = LEARNED ? a.z : a.r;
  double dummy;
  unsigned int epoch = 0;  // grid barriers passed (the launcher zeroes the arrival counter)

  // init: x^ = 0, r = b^, z = S b^, max |b^|
  for (int sl = gw; sl < ns; sl += W) {
    const int i = 32 * sl + lane;
    double rz_loc = 0.0, binf_loc = 0.0;
    if (i < V) {
      float b0 = a.bhat[3 * i], b1 = a.bhat[3 * i + 1], b2 = a.bhat[3 * i + 2];
      binf_loc = fmax(fabs(double(b0)), fmax(fabs(double(b1)), fabs(double(b2))));
      a.xh[3 * i] = 0.0; a.xh[3 * i + 1] = 0.0; a.xh[3 * i + 2] = 0.0;
      st4<S>(r, i, b0, b1, b2);
      if (LEARNED) {
        float y0, y1, y2;
        sell_row_S<U>(i, a.chunk_off, a.sell_col, a.valh, a.coef, a.Sdiag, GatherV{a.bhat}, y0, y1, y2);
        st4<S>(a.z, i, y0, y1, y2);
        rz_loc = double(b0) * y0 + double(b1) * y1 + double(b2) * y2;
      } else {
        rz_loc = double(b0) * b0 + double(b1) * b1 + double(b2) * b2;
        if (a.snap_r && a.snap_max > 0) {
          a.snap_r[3 * i] = b0; a.snap_r[3 * i + 1] = b1; a.snap_r[3 * i + 2] = b2;
          a.snap_x[3 * i] = 0.0; a.snap_x[3 * i + 1] = 0.0; a.snap_x[3 * i + 2] = 0.0;
        }
      }
    }
    rz_loc = warp_sum(rz_loc);
    binf_loc = warp_max(binf_loc);
    if (lane == 0) { part_rz[sl] = rz_loc; part_rinf[sl] = binf_loc; }
  }
  bool ok = grid_sync_ar(&ctrl->bar_arrivals, nb, epoch, &ctrl->bar_err);
  int status = PCG_MAXIT, iters = 0;
  double rel = 0.0, rz = 0.0, binf = 0.0;
  if (!ok) status = PCG_TIMEOUT;
  else fixed_reduce<true>(part_rz, part_rinf, ns, sh, rz, binf);
  if (ok) {
    rel = binf < 1e-16 ? binf : 1.0;
    if (rel < double(a.tol)) status = PCG_OK;
    else if (LEARNED && !(rz > 0.0)) status = PCG_PRECOND;
  }
  float* pold = a.p0;
  float* pnew = a.p1;
  float beta = 0.f;
  bool first = true;
  double best = rel;
  int since = 0;
  for (int it = 0; ok && status == PCG_MAXIT && it < a.max_iters; ++it) {
    // ---- phase A: p_new = z + beta p_old, Ap = A^ p_new, p^T Ap
    GatherP<S> gp{zsrc, pold, beta, first};
    for (int sl = gw; sl < ns; sl += W) {
      const int row = 32 * sl + lane;
      double pap_loc = 0.0;
      if (row < V) {
        float y0, y1, y2;
        sell_row_u<U>(row, a.chunk_off, a.sell_col, a.valh, a.xbegin, a.xend, a.xcols, a.xvalh, gp, y0, y1, y2);
        float q0, q1, q2; gp(row, q0, q1, q2);
        st4<S>(pnew, row, q0, q1, q2);
        st4<S>(a.Ap, row, y0, y1, y2);
        pap_loc = double(q0) * y0 + double(q1) * y1 + double(q2) * y2;
      }
      pap_loc = warp_sum(pap_loc);
      if (lane == 0) part_pap[sl] = pap_loc;
    }
    ok = grid_sync_ar(&ctrl->bar_arrivals, nb, epoch, &ctrl->bar_err);
    if (!ok) { status = PCG_TIMEOUT; break; }
    double pap;
    fixed_reduce<false>(part_pap, nullptr, ns, sh, pap, dummy);
    iters = it + 1;
    if (fabs(pap) < 1e-16) { status = PCG_NOT_SPD; break; }
    float alpha = float(rz / pap);
    // ---- phase B: x^ += alpha p, r -= alpha Ap, z = S r, r^T z, |L r|_inf
    if (!LEARNED) {
      // snapshot k of (r^, x^) after 2^k - 1 iterations (training probes)
      const int done = it + 1;
      const int snap = (a.snap_r && ((done & (done + 1)) == 0)) ? __ffs(done + 1) - 1 : -1;
      float* sr = (snap >= 0 && snap < a.snap_max) ? a.snap_r + 3ll * V * snap : nullptr;
      double* sx = sr ? a.snap_x + 3ll * V * snap : nullptr;
      for (int sl = gw; sl < ns; sl += W) {
        const int i = 32 * sl + lane;
        double rz_new_loc = 0.0, rinf_loc = 0.0;
        if (i < V) {
          const float4 pv = ld4<S>(pnew, i), rv = ld4<S>(r, i), av = ld4<S>(a.Ap, i);
          const float p0 = pv.x, p1 = pv.y, p2 = pv.z;
          a.xh[3 * i] += double(alpha) * p0; a.xh[3 * i + 1] += double(alpha) * p1; a.xh[3 * i + 2] += double(alpha) * p2;
          float r0 = rv.x - alpha * av.x, r1 = rv.y - alpha * av.y, r2 = rv.z - alpha * av.z;
          st4<S>(r, i, r0, r1, r2);
          if (sr) {
            sr[3 * i] = r0; sr[3 * i + 1] = r1; sr[3 * i + 2] = r2;
            sx[3 * i] = a.xh[3 * i]; sx[3 * i + 1] = a.xh[3 * i + 1]; sx[3 * i + 2] = a.xh[3 * i + 2];
          }
          rz_new_loc = double(r0) * r0 + double(r1) * r1 + double(r2) * r2;
          rinf_loc = fmax(fabs(double(r0)), fmax(fabs(double(r1)), fabs(double(r2))));
        }
        rz_new_loc = warp_sum(rz_new_loc);
        rinf_loc = warp_max(rinf_loc);
        if (lane == 0) { part_rz[sl] = rz_new_loc; part_rinf[sl] = rinf_loc; }
      }
    } else {
      GatherR<S> gr{r, a.Ap, alpha};
      for (int sl = gw; sl < ns; sl += W) {
        const int row = 32 * sl + lane;
        double rz_new_loc = 0.0, rinf_loc = 0.0;
        if (row < V) {
          float y0, y1, y2;
          sell_row_S<U>(row, a.chunk_off, a.sell_col, a.valh, a.coef, a.Sdiag, gr, y0, y1, y2);
          float r0, r1, r2; gr(row, r0, r1, r2);
          const float4 pv = ld4<S>(pnew, row);
          a.xh[3 * row] += double(alpha) * pv.x; a.xh[3 * row + 1] += double(alpha) * pv.y;
          a.xh[3 * row + 2] += double(alpha) * pv.z;
          st4<S>(rn, row, r0, r1, r2);
          st4<S>(a.z, row, y0, y1, y2);
          rz_new_loc = double(r0) * y0 + double(r1) * y1 + double(r2) * y2;
          rinf_loc = fmax(fabs(double(r0)), fmax(fabs(double(r1)), fabs(double(r2))));
        }
        rz_new_loc = warp_sum(rz_new_loc);
        rinf_loc = warp_max(rinf_loc);
        if (lane == 0) { part_rz[sl] = rz_new_loc; part_rinf[sl] = rinf_loc; }
      }
    }
    ok = grid_sync_ar(&ctrl->bar_arrivals, nb, epoch, &ctrl->bar_err);
    if (!ok) { status = PCG_TIMEOUT; break; }
    double rz_new, rinf;
    fixed_reduce<true>(part_rz, part_rinf, ns, sh, rz_new, rinf);
    rel = binf < 1e-16 ? rinf : rinf / binf;
    if (LEARNED) { float* t = r; r = rn; rn = t; }
    if (rel < double(a.tol)) { status = PCG_OK; break; }
    if (LEARNED) {
      if (!(rz_new > 0.0)) { status = PCG_PRECOND; break; }
      if (rel < best) { best = rel; since = 0; }
      else if (++since >= a.stall_window) { status = PCG_STALL; break; }
    }
    beta = float(rz_new / rz);
    rz = rz_new;
    first = false;
    float* t = pold; pold = pnew; pnew = t;
  }
  // d = L^-T x^ (every x^ write precedes the last grid barrier); x^ is FP64:
  // rounding it to FP32 would cost up to cond(L_i) x 6e-8 of d_i at stiff vertices
  if (ok) {
    for (int sl = gw; sl < ns; sl += W) {
      const int i = 32 * sl + lane;
      if (i >= V) continue;
      const double* q = a.Linv + 6 * (long long)i;
      double x0 = a.xh[3 * i], x1 = a.xh[3 * i + 1], x2 = a.xh[3 * i + 2];
      a.d[3 * i] = float(q[0] * x0 + q[1] * x1 + q[3] * x2);
      a.d[3 * i + 1] = float(q[2] * x1 + q[4] * x2);
      a.d[3 * i + 2] = float(q[5] * x2);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (LEARNED) ctrl->learned_iters = iters;
    ctrl->pcg_iters = iters;
    ctrl->pcg_status = status;
    ctrl->pcg_converged = status == PCG_OK ? 1 : 0;
    ctrl->pcg_rel = rel;
  }
}

using ScaledKernel = void (*)(PcgScaledArgs);
ScaledKernel scaled_kernel(bool learned, int unroll) {
  if (learned) return unroll >= 2 ? k_pcg_scaled<true, 2> : k_pcg_scaled<true, 1>;
  return unroll >= 2 ? k_pcg_scaled<false, 2> : k_pcg_scaled<false, 1>;
}

}  // namespace

int pcg_grid_size(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg, PCG_TPB, 0);
  if (per_sm < 1) per_sm = 1;
  int co = sms * per_sm;
  int want = 2 * sms;
  return co < want ? co : want;
}

size_t pcg_scaled_partials(int V) { return 3ull * (size_t)((V + 31) / 32 + 1); }

// Candidate launch shapes of the scaled PCG for V rows on `device`; shape 0
// is the default. Every shape gives the same result bits.
//  - balanced: the 32-row slices spread evenly over the SMs (one or two
//    CTAs per SM, each warp one slice per pass);
//  - fixed CTA sizes of 256 and 512 threads up to the co-resident grid;
// each with one and two column slots loaded ahead per thread.
int pcg_scaled_shapes(int device, int V, bool learned, PcgShape* out, int max) {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (sms < 1) sms = 1;
  const int ns = (V + 31) / 32 > 0 ? (V + 31) / 32 : 1;
  int n = 0;
  auto occ = [&](int unroll, int tpb) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, scaled_kernel(learned, unroll), tpb, 0);
    return per;
  };
  for (int unroll = 1; unroll <= 2; ++unroll) {
    const int wps = (ns + sms - 1) / sms;  // warps needed per SM for one pass
    int k = (wps + 31) / 32;               // CTAs per SM
    int tpb = 32 * ((wps + k - 1) / k);
    while (k > 1 && occ(unroll, tpb) < k) {
      --k;
      tpb = 32 * ((wps + k - 1) / k);
      if (tpb > SCALED_MAX_TPB) { tpb = SCALED_MAX_TPB; break; }
    }
    if (tpb > SCALED_MAX_TPB) tpb = SCALED_MAX_TPB;
    int per = occ(unroll, tpb);
    if (per >= 1 && n < max) {
      int grid = (ns + tpb / 32 - 1) / (tpb / 32);
      if (grid > sms * per) grid = sms * per;
      out[n++] = PcgShape{tpb, grid, unroll};
    }
    // fewer, larger CTAs: fewer arrivals at each grid barrier and fewer
    // copies of the per-slice partials read after it; the last two
    // candidates give every warp two slices
    for (int t : {256, 512, 768, 1024}) {
      int p = occ(unroll, t);
      if (p < 1 || n >= max) continue;
      int grid = (ns + t / 32 - 1) / (t / 32);
      if (grid > sms * p) grid = sms * p;
      out[n++] = PcgShape{t, grid, unroll};
      if (t >= 768 && grid > 1 && n < max) out[n++] = PcgShape{t, (grid + 1) / 2, unroll};
    }
  }
  return n;
}

cudaError_t launch_pcg_scaled(const PcgScaledArgs& a, bool learned, const PcgShape& sh, cudaStream_t s) {
  if (sh.tpb < 32 || sh.tpb > SCALED_MAX_TPB || (sh.tpb & 31) || sh.grid < 1) return cudaErrorInvalidConfiguration;
  cudaError_t e = cudaMemsetAsync(&a.ctrl->bar_arrivals, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&a};
  return cudaLaunchCooperativeKernel((void*)scaled_kernel(learned, sh.unroll), dim3(sh.grid), dim3(sh.tpb), args, 0, s);
}

cudaError_t launch_pcg(const PcgArgs& a, int grid, cudaStream_t s) {
  int need = (a.V + PCG_TPB - 1) / PCG_TPB;  // enough CTAs for one vertex per thread
  if (need < 1) need = 1;
  if (grid > need) grid = need;
  void* args[] = {(void*)&a};
  return cudaLaunchCooperativeKernel((void*)k_pcg, dim3(grid), dim3(PCG_TPB), args, 0, s);
}

}  // namespace ando
