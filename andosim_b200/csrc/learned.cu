// learned.cu -- features, message-passing network, SPD preconditioner
// assembly, training loss and its gradient, Adam (see learned.cuh).
//
// Every reduction is in a fixed order: per-CTA partials over a fixed grid,
// summed CTA by CTA; scatters to vertices are gathers through the pattern's
// transpose slots. Forward and backward are therefore bitwise reproducible.
#include <atomic>

#include <cuda_bf16.h>

#include "learned.cuh"

namespace ando {

namespace {

using namespace net;

constexpr int TPB = 256;
constexpr int GRID = 296;          // fixed grid of the reducing kernels (2 CTAs per SM on 148 SMs)
constexpr int PART = H * 2 * H + H;  // largest per-CTA partial (update layer: 64 x 128 weights + 64 bias)
inline int nblk(long long n, int tpb = TPB) { return int((n + tpb - 1) / tpb); }

// transposed (forward) layout of the dense matrices inside NetDev::wt
constexpr int WT_IN = 0;                       // FN x H
constexpr int WT_LAYER0 = WT_IN + FN * H;
constexpr int WT_U = 0;                        // H x H
constexpr int WT_W = WT_U + H * H;             // 2H x H
constexpr int WT_LSIZE = WT_W + 2 * H * H;
constexpr int WT_SIZE = WT_LAYER0 + NL * WT_LSIZE;

__device__ inline float softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }
__device__ inline float sigm(float z) { return 1.f / (1.f + expf(-z)); }
__device__ inline float warp_sum(float v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------------ weights
__global__ void k_net_round(const float* master, float* wq, unsigned short* bf, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  __nv_bfloat16 b = __float2bfloat16_rn(master[i]);
  wq[i] = __bfloat162float(b);
  if (bf) bf[i] = __bfloat16_as_ushort(b);
}
// wt[dst + k*out + o] = wq[src + o*in + k]
__global__ void k_net_transpose(const float* wq, float* wt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= WT_SIZE) return;
  int src, in, rem;
  if (i < WT_LAYER0) { src = W_IN; in = FN; rem = i; }
  else {
    int l = (i - WT_LAYER0) / WT_LSIZE, r = (i - WT_LAYER0) % WT_LSIZE;
    if (r < WT_W) { src = LAYER0 + l * L_SIZE + L_U; in = H; rem = r; }
    else { src = LAYER0 + l * L_SIZE + L_W; in = 2 * H; rem = r - WT_W; }
  }
  int k = rem / H, o = rem % H;
  wt[i] = wq[src + o * in + k];
}

// ------------------------------------------------------------------ features
// Edge features of every static slot: the 9 entries of A^_k and its Frobenius norm.
// Rows of FES floats (16-byte aligned, the last two zero).
__global__ void k_edge_feats(int nnzb, const float* valh, float* Ef) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnzb) return;
  const float* a = valh + 9ll * k;
  float e[FES];
  float s = 0.f;
  for (int q = 0; q < 9; ++q) { e[q] = a[q]; s += a[q] * a[q]; }
  e[9] = sqrtf(s); e[10] = 0.f; e[11] = 0.f;
  float4* o = reinterpret_cast<float4*>(Ef + (long long)k * FES);
  for (int q = 0; q < FES / 4; ++q) o[q] = make_float4(e[4 * q], e[4 * q + 1], e[4 * q + 2], e[4 * q + 3]);
}
// Node features: 1, log(1 + contact blocks), static and contact coupling
// (sums of |A^_ij|_F), stiffness of the diagonal block relative to the mass
// term (log10 tr(A_ii) / (3 m / dt^2), over 4), degree / 8, pinned flag,
// largest static coupling.
__global__ void k_node_feats(LsView s, const float* Ef, float* X) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.V) return;
  float stat = 0.f, mx = 0.f, cont = 0.f;
  int deg = 0, ncont = 0;
  for (int k = s.rowptr[i]; k < s.rowptr[i + 1]; ++k) {
    if (s.cols[k] == i) continue;
    float nf = Ef[(long long)k * FES + 9];
    stat += nf; mx = fmaxf(mx, nf); ++deg;
  }
  if (s.xbegin) {
    for (int k = s.xbegin[i]; k < s.xend[i]; ++k) {
      const float* a = s.xvalh + 9ll * k;
      float t = 0.f;
      for (int q = 0; q < 9; ++q) t += a[q] * a[q];
      cont += sqrtf(t); ++ncont;
    }
  }
  bool fx = s.fixed && s.fixed[i];
  const float* l = s.Lf + 6ll * i;
  double tr = double(l[0]) * l[0] + double(l[1]) * l[1] + double(l[2]) * l[2] + double(l[3]) * l[3] + double(l[4]) * l[4] +
              double(l[5]) * l[5];
  double mref = 3.0 * s.mass[i] * s.dt2inv;
  float stiff = (fx || !(mref > 0.0) || !(tr > 0.0)) ? 0.f : float(log10(tr / mref) * 0.25);
  float* x = X + (long long)i * FN;
  x[0] = 1.f; x[1] = log1pf(float(ncont)); x[2] = stat; x[3] = cont; x[4] = stiff;
  x[5] = float(deg) * 0.125f; x[6] = fx ? 1.f : 0.f; x[7] = mx;
}

// --------------------------------------------------------------- row GEMM
// Y[r, :N] = act(X[r, :] M + bias) + R1[r, :N] + R2[r, :N], X = [X1 | X2]
// (K = K1 + K2 <= 128), M row-major [K][N], N in {64, 128}; Q gets the
// pre-activation. 64 rows per CTA (M is staged in shared memory once per 64
// rows), each thread 4 rows x N/16 outputs held in registers (N is a template
// parameter so the accumulators never spill to local memory).
template <int N>
__global__ void __launch_bounds__(TPB) k_gemm(int V, const float* X1, int ld1, int K1, const float* X2, int ld2, int K2, const float* M,
                                              const float* bias, const float* R1, int ldr1, const float* R2, int ldr2, float* Q,
                                              float* Y, int relu) {
  constexpr int ROWS = 64, PER = N / 16;
  extern __shared__ float sm[];
  const int K = K1 + K2, XS = K + 1;
  float* Ms = sm;                // K x N
  float* Xs = sm + K * N;        // ROWS x XS
  const int r0 = blockIdx.x * ROWS;
  for (int i = threadIdx.x; i < K * N; i += TPB) Ms[i] = M[i];
  for (int i = threadIdx.x; i < ROWS * K; i += TPB) {
    int r = i / K, k = i % K, row = r0 + r;
    float v = 0.f;
    if (row < V) v = k < K1 ? X1[(long long)row * ld1 + k] : X2[(long long)row * ld2 + (k - K1)];
    Xs[r * XS + k] = v;
  }
  __syncthreads();
  // 16 row groups of 4 rows x 16 column groups of PER columns
  const int r = (threadIdx.x / 16) * 4, c0 = (threadIdx.x % 16) * PER;
  float acc[4][PER];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int j = 0; j < PER; ++j) acc[a][j] = 0.f;
  for (int k = 0; k < K; ++k) {
    float xv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) xv[a] = Xs[(r + a) * XS + k];
    const float* mr = Ms + k * N + c0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      float m = mr[j];
#pragma unroll
      for (int a = 0; a < 4; ++a) acc[a][j] += xv[a] * m;
    }
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    int row = r0 + r + a;
    if (row >= V) continue;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      int c = c0 + j;
      float q = acc[a][j] + (bias ? bias[c] : 0.f);
      if (Q) Q[(long long)row * N + c] = q;
      float y = relu ? fmaxf(q, 0.f) : q;
      if (R1) y += R1[(long long)row * ldr1 + c];
      if (R2) y += R2[(long long)row * ldr2 + c];
      Y[(long long)row * N + c] = y;
    }
  }
}

// Weight gradient partials: part[g] = [dQ^T X (64 x K, row-major) ; sum dQ (64)]
// over CTA g's contiguous row range.
__global__ void __launch_bounds__(TPB) k_wgrad(int V, const float* dQ, int ldq, const float* X1, int ld1, int K1, const float* X2, int ld2,
                                               int K2, float* part) {
  __shared__ float dqs[32 * H];
  __shared__ float xs[32 * (2 * H + 1)];
  const int K = K1 + K2, XS = K + 1;
  const int rows_per = (V + gridDim.x - 1) / gridDim.x;
  const int rb = blockIdx.x * rows_per, re = min(V, rb + rows_per);
  const int o = threadIdx.x >> 2, kq = threadIdx.x & 3, kw = K / 4, kb = kq * kw;
  float acc[32], bacc = 0.f;
  for (int j = 0; j < 32; ++j) acc[j] = 0.f;
  for (int c0 = rb; c0 < re; c0 += 32) {
    __syncthreads();
    for (int i = threadIdx.x; i < 32 * H; i += TPB) {
      int r = i / H, c = i % H, row = c0 + r;
      dqs[i] = row < re ? dQ[(long long)row * ldq + c] : 0.f;
    }
    for (int i = threadIdx.x; i < 32 * K; i += TPB) {
      int r = i / K, k = i % K, row = c0 + r;
      float v = 0.f;
      if (row < re) v = k < K1 ? X1[(long long)row * ld1 + k] : X2[(long long)row * ld2 + (k - K1)];
      xs[r * XS + k] = v;
    }
    __syncthreads();
    for (int r = 0; r < 32; ++r) {
      float g = dqs[r * H + o];
      if (kq == 0) bacc += g;
      for (int j = 0; j < kw; ++j) acc[j] += g * xs[r * XS + kb + j];
    }
  }
  float* p = part + (long long)blockIdx.x * PART;
  for (int j = 0; j < kw; ++j) p[o * K + kb + j] = acc[j];
  if (kq == 0) p[H * K + o] = bacc;
}

// out[i] (+)= sum over g of part[g * PART + off + i], g in order.
__global__ void k_reduce_parts(const float* part, int G, int off, int n, float* out, int accumulate) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int g = 0; g < G; ++g) s += part[(long long)g * PART + off + i];
  out[i] = accumulate ? out[i] + s : s;
}

__global__ void k_relu_mask(long long n, const float* dh, const float* q, float* dq) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dq[i] = q[i] > 0.f ? dh[i] : 0.f;
}

// ------------------------------------------------------------ messages
// m_i = (1 / deg_i) sum_{j in N(i)} relu(u_j + E e_ij + c); one warp per row,
// lane l owns channels 2l and 2l+1. A row of at most MSG_SLOTS slots loads
// its columns with one coalesced load and then every neighbour's u at once;
// each slot's features reach all lanes as three broadcast 16-byte loads.
// Longer rows walk their slots one by one. Both paths add the same terms in
// the same order.
constexpr int MSG_SLOTS = 8;
__device__ inline void msg_term(float4 q0, float4 q1, float4 q2, const float* e0, const float* e1, float& t0, float& t1) {
  const float ef[FE] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y};
#pragma unroll
  for (int f = 0; f < FE; ++f) { t0 += e0[f] * ef[f]; t1 += e1[f] * ef[f]; }
}
__global__ void __launch_bounds__(TPB) k_msg_fwd(LsView s, const float* u, const float* Ef, const float* Ew, const float* cb, float* m) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int c0 = 2 * lane, c1 = c0 + 1;
  float e0[FE], e1[FE];
  for (int f = 0; f < FE; ++f) { e0[f] = Ew[c0 * FE + f]; e1[f] = Ew[c1 * FE + f]; }
  const float b0 = cb[c0], b1 = cb[c1];
  for (int i = gw; i < s.V; i += nw) {
    float a0 = 0.f, a1 = 0.f;
    int deg = 0;
    const int kb = s.rowptr[i], ns = s.rowptr[i + 1] - kb;
    if (ns <= MSG_SLOTS) {
      const int jl = lane < ns ? s.cols[kb + lane] : -1;
      float2 uv[MSG_SLOTS];
#pragma unroll
      for (int sl = 0; sl < MSG_SLOTS; ++sl) {
        const int j = __shfl_sync(0xffffffffu, jl, sl);
        uv[sl] = sl < ns && j != i ? *reinterpret_cast<const float2*>(u + (long long)j * H + c0) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int sl = 0; sl < MSG_SLOTS; ++sl) {
        const int j = __shfl_sync(0xffffffffu, jl, sl);
        if (sl < ns && j != i) {  // uniform over the warp
          const float4* e4 = reinterpret_cast<const float4*>(Ef + (long long)(kb + sl) * FES);
          float t0 = uv[sl].x + b0, t1 = uv[sl].y + b1;
          msg_term(e4[0], e4[1], e4[2], e0, e1, t0, t1);
          a0 += fmaxf(t0, 0.f); a1 += fmaxf(t1, 0.f);
          ++deg;
        }
      }
    } else {
      for (int k = kb; k < kb + ns; ++k) {
        int j = s.cols[k];
        if (j == i) continue;
        const float4* e4 = reinterpret_cast<const float4*>(Ef + (long long)k * FES);
        float t0 = u[(long long)j * H + c0] + b0, t1 = u[(long long)j * H + c1] + b1;
        msg_term(e4[0], e4[1], e4[2], e0, e1, t0, t1);
        a0 += fmaxf(t0, 0.f); a1 += fmaxf(t1, 0.f);
        ++deg;
      }
    }
    float inv = deg ? 1.f / float(deg) : 0.f;
    m[(long long)i * H + c0] = a0 * inv;
    m[(long long)i * H + c1] = a1 * inv;
  }
}

// The same messages at inference with one thread per row: the thread reads
// its slots' own features and its neighbours' whole u rows, and the edge
// weights and bias arrive by value as kernel parameters (constant-bank
// operands of the FMAs), so no value is replicated across lanes. Same terms,
// same order as k_msg_fwd.
struct MsgWeights { float E[H * FE]; float c[H]; };
constexpr int MSG_ROWS_TPB = 128;
__global__ void __launch_bounds__(MSG_ROWS_TPB) k_msg_rows(LsView s, const float* __restrict__ u, const float* __restrict__ Ef,
                                                           const MsgWeights P, float* __restrict__ m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.V) return;
  float acc[H];
#pragma unroll
  for (int c = 0; c < H; ++c) acc[c] = 0.f;
  int deg = 0;
  const int ke = s.rowptr[i + 1];
  for (int k = s.rowptr[i]; k < ke; ++k) {
    const int j = s.cols[k];
    if (j == i) continue;
    const float4* e4 = reinterpret_cast<const float4*>(Ef + (long long)k * FES);
    const float4 q0 = e4[0], q1 = e4[1], q2 = e4[2];
    const float ef[FE] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w, q2.x, q2.y};
    const float4* u4 = reinterpret_cast<const float4*>(u + (long long)j * H);
#pragma unroll
    for (int c4 = 0; c4 < H / 4; ++c4) {
      const float4 uv = u4[c4];
      const float ux[4] = {uv.x, uv.y, uv.z, uv.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int c = 4 * c4 + e;
        float t = ux[e] + P.c[c];
#pragma unroll
        for (int f = 0; f < FE; ++f) t += P.E[c * FE + f] * ef[f];
        acc[c] += fmaxf(t, 0.f);
      }
    }
    ++deg;
  }
  const float inv = deg ? 1.f / float(deg) : 0.f;
  float4* mo = reinterpret_cast<float4*>(m + (long long)i * H);
#pragma unroll
  for (int c4 = 0; c4 < H / 4; ++c4) mo[c4] = make_float4(acc[4 * c4] * inv, acc[4 * c4 + 1] * inv, acc[4 * c4 + 2] * inv, acc[4 * c4 + 3] * inv);
}

// Backward of k_msg_fwd. Row j gathers over its slots (j, i) the messages it
// sent to i (transpose slot (i, j) holds e_ij): du_j, and per-CTA partials of
// dE (64 x FE) and dc (64).
__global__ void __launch_bounds__(TPB) k_msg_bwd(LsView s, const float* u, const float* Ef, const float* Ew, const float* cb,
                                                 const float* dm, int lddm, float* du, float* part) {
  __shared__ float red[TPB / 32][H * (FE + 1)];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int c0 = 2 * lane, c1 = c0 + 1;
  float e0[FE], e1[FE], g0[FE], g1[FE];
  for (int f = 0; f < FE; ++f) { e0[f] = Ew[c0 * FE + f]; e1[f] = Ew[c1 * FE + f]; g0[f] = 0.f; g1[f] = 0.f; }
  const float b0 = cb[c0], b1 = cb[c1];
  float gc0 = 0.f, gc1 = 0.f;
  for (int j = gw; j < s.V; j += nw) {
    float d0 = 0.f, d1 = 0.f;
    const float uj0 = u[(long long)j * H + c0], uj1 = u[(long long)j * H + c1];
    for (int k = s.rowptr[j]; k < s.rowptr[j + 1]; ++k) {
      int i = s.cols[k];
      if (i == j) continue;
      int kT = s.slot_T[k];
      int deg = s.rowptr[i + 1] - s.rowptr[i] - 1;
      if (deg <= 0) continue;
      const float* e = Ef + (long long)kT * FES;
      float t0 = uj0 + b0, t1 = uj1 + b1;
      for (int f = 0; f < FE; ++f) { float ef = e[f]; t0 += e0[f] * ef; t1 += e1[f] * ef; }
      float inv = 1.f / float(deg);
      float m0 = t0 > 0.f ? dm[(long long)i * lddm + c0] * inv : 0.f;
      float m1 = t1 > 0.f ? dm[(long long)i * lddm + c1] * inv : 0.f;
      d0 += m0; d1 += m1;
      for (int f = 0; f < FE; ++f) { float ef = e[f]; g0[f] += m0 * ef; g1[f] += m1 * ef; }
      gc0 += m0; gc1 += m1;
    }
    du[(long long)j * H + c0] = d0;
    du[(long long)j * H + c1] = d1;
  }
  for (int f = 0; f < FE; ++f) { red[warp][c0 * FE + f] = g0[f]; red[warp][c1 * FE + f] = g1[f]; }
  red[warp][H * FE + c0] = gc0; red[warp][H * FE + c1] = gc1;
  __syncthreads();
  float* p = part + (long long)blockIdx.x * PART;
  for (int i = threadIdx.x; i < H * (FE + 1); i += TPB) {
    float v = 0.f;
    for (int w = 0; w < TPB / 32; ++w) v += red[w][i];
    p[i] = v;
  }
}

// ------------------------------------------------------------- decoder
// z_i = dv . h_i + dv0; for every slot (i, j) with j > i:
// (a, b) = De [h_i ; h_j ; e_ij] + de.
__global__ void k_dec_fwd(LsView s, const float* h, const float* Ef, const float* w, float* zv, float* ab) {
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int c0 = 2 * lane, c1 = c0 + 1;
  const float* dv = w + DV;
  const float* De0 = w + DE;
  const float* De1 = w + DE + DE_IN;
  for (int i = gw; i < s.V; i += nw) {
    float hi0 = h[(long long)i * H + c0], hi1 = h[(long long)i * H + c1];
    float z = warp_sum(dv[c0] * hi0 + dv[c1] * hi1);
    if (lane == 0) zv[i] = z + w[DV0];
    float pa = De0[c0] * hi0 + De0[c1] * hi1, pb = De1[c0] * hi0 + De1[c1] * hi1;
    for (int k = s.rowptr[i]; k < s.rowptr[i + 1]; ++k) {
      int j = s.cols[k];
      if (j <= i) continue;
      float hj0 = h[(long long)j * H + c0], hj1 = h[(long long)j * H + c1];
      float a = pa + De0[H + c0] * hj0 + De0[H + c1] * hj1;
      float b = pb + De1[H + c0] * hj0 + De1[H + c1] * hj1;
      if (lane < FE) { float ef = Ef[(long long)k * FES + lane]; a += De0[2 * H + lane] * ef; b += De1[2 * H + lane] * ef; }
      a = warp_sum(a); b = warp_sum(b);
      if (lane == 0) { ab[2ll * k] = a + w[DE0]; ab[2ll * k + 1] = b + w[DE0 + 1]; }
    }
  }
}

// S on the static pattern (see learned.cuh); one thread per row.
__global__ void k_build_S(LsView s, const float* zv, const float* ab, float* S, SPcg pcg) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.V) return;
  float D[9];
  float delta = softplus(zv[i]) + DELTA_MIN;
  for (int q = 0; q < 9; ++q) D[q] = (q % 4 == 0) ? delta : 0.f;
  int kd = -1;
  for (int k = s.rowptr[i]; k < s.rowptr[i + 1]; ++k) {
    int j = s.cols[k];
    if (j == i) { kd = k; continue; }
    const float* A = s.valh + 9ll * k;
    float c;
    if (j > i) {
      float a = ab[2ll * k], b = ab[2ll * k + 1];
      c = a * b;
      D[0] += a * a; D[4] += a * a; D[8] += a * a;
    } else {
      long long kT = s.slot_T[k];
      float a = ab[2 * kT], b = ab[2 * kT + 1];
      c = a * b;
      float b2 = b * b;
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) D[3 * r + q] += b2 * (A[3 * r] * A[3 * q] + A[3 * r + 1] * A[3 * q + 1] + A[3 * r + 2] * A[3 * q + 2]);
    }
    if (S) for (int q = 0; q < 9; ++q) S[9ll * k + q] = c * A[q];
    if (pcg.coef) {
      const int l = i & 31;
      pcg.coef[(s.sell_base[k] - l) / 9 + l] = c;  // sell_base = 9 (chunk slot) + lane
    }
  }
  if (kd >= 0 && S) for (int q = 0; q < 9; ++q) S[9ll * kd + q] = D[q];
  if (pcg.diag) for (int q = 0; q < 9; ++q) pcg.diag[9ll * i + q] = D[q];
}

// ------------------------------------------------------- training loss
// y = M v row by row (warp per row), static pattern and optional extra segment.
__global__ void k_spmv(int V, const int* rowptr, const int* cols, const float* val, const int* xbegin, const int* xend, const int* xcols,
                       const float* xval, const float* v, float* y) {
  const int lane = threadIdx.x & 31, comp = lane >> 3, bi = lane & 7;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int row = gw; row < V; row += nw) {
    float acc = 0.f;
    for (int k0 = rowptr[row]; k0 < rowptr[row + 1]; k0 += 8) {
      int k = k0 + bi;
      if (comp < 3 && k < rowptr[row + 1]) {
        int c = cols[k];
        const float* h = val + 9ll * k + 3 * comp;
        acc += h[0] * v[3 * c] + h[1] * v[3 * c + 1] + h[2] * v[3 * c + 2];
      }
    }
    if (xbegin) {
      for (int k0 = xbegin[row]; k0 < xend[row]; k0 += 8) {
        int k = k0 + bi;
        if (comp < 3 && k < xend[row]) {
          int c = xcols[k];
          const float* h = xval + 9ll * k + 3 * comp;
          acc += h[0] * v[3 * c] + h[1] * v[3 * c + 1] + h[2] * v[3 * c + 2];
        }
      }
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 4);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    float y0 = __shfl_sync(0xffffffffu, acc, 0), y1 = __shfl_sync(0xffffffffu, acc, 8), y2 = __shfl_sync(0xffffffffu, acc, 16);
    if (lane == 0) { y[3 * row] = y0; y[3 * row + 1] = y1; y[3 * row + 2] = y2; }
  }
}

// per-CTA partials of T_p = y^T w - 2 r^T y (FP64), fixed grid.
__global__ void k_loss_terms(int V, int P, const float* r, const float* y, const float* w, double* parts) {
  __shared__ double red[TPB / 32];
  for (int p = 0; p < P; ++p) {
    const float* rp = r + 3ll * V * p; const float* yp = y + 3ll * V * p; const float* wp = w + 3ll * V * p;
    double t = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < 3ll * V; e += (long long)gridDim.x * blockDim.x)
      t += double(yp[e]) * wp[e] - 2.0 * double(rp[e]) * yp[e];
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      double sacc = 0.0;
      for (int k = 0; k < TPB / 32; ++k) sacc += red[k];
      parts[(long long)blockIdx.x * P + p] = sacc;
    }
    __syncthreads();
  }
}
__global__ void k_loss_final(const double* parts, int G, int P, const double* pnorm, double* loss) {
  if (threadIdx.x || blockIdx.x) return;
  double L = 0.0;
  for (int p = 0; p < P; ++p) {
    double T = 0.0;
    for (int g = 0; g < G; ++g) T += parts[(long long)g * P + p];
    L += 1.0 + T / pnorm[p];
  }
  *loss = L / P;
}

// Gradient of the loss w.r.t. delta_i (through the softplus: dzv) and the
// edge coefficients (dab), with gy_p = 2 (w_p - r_p) / (n_p P).
__global__ void k_coef_grad(LsView s, int P, const float* r, const float* w, const double* pnorm, const float* zv, const float* ab,
                            float* dzv, float* dab) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.V) return;
  const long long n3 = 3ll * s.V;
  auto gy = [&](int p, int v, int c) { return float(2.0 * (double(w[n3 * p + 3 * v + c]) - r[n3 * p + 3 * v + c]) / (pnorm[p] * P)); };
  float gbi = 0.f;
  for (int p = 0; p < P; ++p)
    for (int c = 0; c < 3; ++c) gbi += gy(p, i, c) * r[n3 * p + 3 * i + c];
  dzv[i] = gbi * sigm(zv[i]);
  for (int k = s.rowptr[i]; k < s.rowptr[i + 1]; ++k) {
    int j = s.cols[k];
    if (j <= i) continue;
    const float* A = s.valh + 9ll * k;
    float AtA[9];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) AtA[3 * a + b] = A[a] * A[b] + A[3 + a] * A[3 + b] + A[6 + a] * A[6 + b];
    float dc = 0.f, gbb = 0.f;
    for (int p = 0; p < P; ++p) {
      float gi[3], gj[3], ri[3], rj[3];
      for (int c = 0; c < 3; ++c) { gi[c] = gy(p, i, c); gj[c] = gy(p, j, c); ri[c] = r[n3 * p + 3 * i + c]; rj[c] = r[n3 * p + 3 * j + c]; }
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          dc += gi[a] * A[3 * a + b] * rj[b] + gj[b] * A[3 * a + b] * ri[a];
          gbb += gj[a] * AtA[3 * a + b] * rj[b];
        }
    }
    float a = ab[2ll * k], b = ab[2ll * k + 1];
    dab[2ll * k] = dc * b + 2.f * a * gbi;
    dab[2ll * k + 1] = dc * a + 2.f * b * gbb;
  }
}

// Backward of k_dec_fwd: dh_r, and per-CTA partials of ddv (64), ddv0 (1),
// dDe (2 x DE_IN) and dde (2), laid out as in the parameter vector from DV.
__global__ void __launch_bounds__(TPB) k_dec_bwd(LsView s, const float* h, const float* Ef, const float* w, const float* dzv,
                                                 const float* dab, float* dh, float* part) {
  constexpr int NP = H + 1 + 2 * DE_IN + 2;
  __shared__ float red[TPB / 32][NP];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  const int c0 = 2 * lane, c1 = c0 + 1;
  const float* dv = w + DV;
  const float* De0 = w + DE;
  const float* De1 = w + DE + DE_IN;
  float gdv0 = 0.f, gdv1 = 0.f, gdv00 = 0.f;
  float gA[4] = {0.f, 0.f, 0.f, 0.f}, gB[4] = {0.f, 0.f, 0.f, 0.f};  // (h_i, h_j) x (c0, c1) for rows a and b
  float gAe = 0.f, gBe = 0.f, gde0 = 0.f, gde1 = 0.f;                  // lane < FE: edge-feature weights
  for (int r = gw; r < s.V; r += nw) {
    float hr0 = h[(long long)r * H + c0], hr1 = h[(long long)r * H + c1];
    float dz = dzv[r];
    float o0 = dz * dv[c0], o1 = dz * dv[c1];
    gdv0 += dz * hr0; gdv1 += dz * hr1;
    if (lane == 0) gdv00 += dz;
    for (int k = s.rowptr[r]; k < s.rowptr[r + 1]; ++k) {
      int j = s.cols[k];
      if (j == r) continue;
      if (j > r) {
        float da = dab[2ll * k], db = dab[2ll * k + 1];
        o0 += da * De0[c0] + db * De1[c0];
        o1 += da * De0[c1] + db * De1[c1];
        float hj0 = h[(long long)j * H + c0], hj1 = h[(long long)j * H + c1];
        gA[0] += da * hr0; gA[1] += da * hr1; gA[2] += da * hj0; gA[3] += da * hj1;
        gB[0] += db * hr0; gB[1] += db * hr1; gB[2] += db * hj0; gB[3] += db * hj1;
        if (lane < FE) { float ef = Ef[(long long)k * FES + lane]; gAe += da * ef; gBe += db * ef; }
        if (lane == 0) { gde0 += da; gde1 += db; }
      } else {
        long long kT = s.slot_T[k];
        float da = dab[2 * kT], db = dab[2 * kT + 1];
        o0 += da * De0[H + c0] + db * De1[H + c0];
        o1 += da * De0[H + c1] + db * De1[H + c1];
      }
    }
    dh[(long long)r * H + c0] = o0;
    dh[(long long)r * H + c1] = o1;
  }
  float* q = red[warp];
  // layout relative to DV: [dv 64][dv0 1][De row a DE_IN][De row b DE_IN][de 2]
  q[c0] = gdv0; q[c1] = gdv1;
  if (lane == 0) q[H] = gdv00;
  const int A0 = H + 1, B0 = H + 1 + DE_IN;
  q[A0 + c0] = gA[0]; q[A0 + c1] = gA[1]; q[A0 + H + c0] = gA[2]; q[A0 + H + c1] = gA[3];
  q[B0 + c0] = gB[0]; q[B0 + c1] = gB[1]; q[B0 + H + c0] = gB[2]; q[B0 + H + c1] = gB[3];
  if (lane < FE) { q[A0 + 2 * H + lane] = gAe; q[B0 + 2 * H + lane] = gBe; }
  if (lane == 0) { q[NP - 2] = gde0; q[NP - 1] = gde1; }
  __syncthreads();
  float* p = part + (long long)blockIdx.x * PART;
  for (int i = threadIdx.x; i < NP; i += TPB) {
    float v = 0.f;
    for (int w2 = 0; w2 < TPB / 32; ++w2) v += red[w2][i];
    p[i] = v;
  }
}

__global__ void k_adam(float* w, float* m1, float* m2, const float* g, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  if (!(fabsf(gi) < 1e30f)) gi = 0.f;  // a non-finite gradient leaves the weight unchanged
  float a = b1 * m1[i] + (1.f - b1) * gi, b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a; m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

void gemm(int V, const float* X1, int ld1, int K1, const float* X2, int ld2, int K2, const float* M, int N, const float* bias,
          const float* R1, int ldr1, const float* R2, int ldr2, float* Q, float* Y, int relu, cudaStream_t s) {
  static std::atomic<unsigned> attr{0};  // one bit per device (steps of several contexts may run on host threads)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 32 && !(attr.load() & (1u << dev))) {
    cudaFuncSetAttribute(k_gemm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_gemm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    attr.fetch_or(1u << dev);
  }
  int K = K1 + K2;
  size_t smem = sizeof(float) * (size_t(K) * N + 64 * (K + 1));
  if (N == 64) k_gemm<64><<<nblk(V, 64), TPB, smem, s>>>(V, X1, ld1, K1, X2, ld2, K2, M, bias, R1, ldr1, R2, ldr2, Q, Y, relu);
  else k_gemm<128><<<nblk(V, 64), TPB, smem, s>>>(V, X1, ld1, K1, X2, ld2, K2, M, bias, R1, ldr1, R2, ldr2, Q, Y, relu);
}
void reduce(const float* part, int off, int n, float* out, cudaStream_t s) {
  k_reduce_parts<<<nblk(n), TPB, 0, s>>>(part, GRID, off, n, out, 0);
}

}  // namespace

size_t learned_work_floats(int V, int nnzb, bool training) {
  size_t VH = size_t(V) * H;
  size_t n = size_t(V) * FN + size_t(nnzb) * FES + VH * (NL + 1) + 3 * VH * NL + VH + V + 2ull * nnzb;
  if (training) n += 7 * VH + V + 2ull * nnzb + size_t(GRID) * PART;
  return n + 4 * 64;  // every buffer starts on a 16-byte boundary (vector loads and stores)
}

void learned_work_carve(LearnedWork& w, float* base, int V, int nnzb, bool training) {
  size_t VH = size_t(V) * H;
  float* p = base;
  auto take = [&](size_t n) { float* r = p; p += (n + 3) & ~size_t(3); return r; };
  w.V = V; w.nnzb = nnzb; w.training = training; w.base = base;
  w.X = take(size_t(V) * FN); w.Ef = take(size_t(nnzb) * FES);
  for (int l = 0; l <= NL; ++l) w.h[l] = take(VH);
  for (int l = 0; l < NL; ++l) { w.u[l] = take(VH); w.m[l] = take(VH); w.q[l] = take(VH); }
  w.q0 = take(VH); w.zv = take(V); w.ab = take(2ull * nnzb);
  if (training) {
    w.dh = take(VH); w.dh2 = take(VH); w.du = take(VH); w.dhm = take(2 * VH); w.dq = take(VH);
    w.dzv = take(V); w.dab = take(2ull * nnzb); w.part = take(size_t(GRID) * PART);
  } else {
    w.dh = w.dh2 = w.du = w.dhm = w.dq = w.dzv = w.dab = w.part = nullptr;
  }
}

// B images of the hidden layers: per layer U (64 x 64) then W (64 x 128)
constexpr int BIMG_U = 0, BIMG_W = H * H, BIMG_LSIZE = BIMG_W + H * 2 * H;
constexpr size_t BIMG_OFF = (size_t(NPARAM) + WT_SIZE + 3) / 4 * 4;  // floats; 16-byte aligned
size_t net_dev_floats() { return BIMG_OFF + size_t(NL) * BIMG_LSIZE / 2; }
void net_dev_carve(NetDev& n, float* base) {
  n.wq = base; n.wt = base + NPARAM;
  n.bimg = reinterpret_cast<unsigned short*>(base + BIMG_OFF);
}

void launch_net_prepare(const float* master, NetDev n, unsigned short* bf16, cudaStream_t s) {
  k_net_round<<<nblk(NPARAM), TPB, 0, s>>>(master, n.wq, bf16, NPARAM);
  k_net_transpose<<<nblk(WT_SIZE), TPB, 0, s>>>(n.wq, n.wt);
  for (int l = 0; l < NL; ++l) {
    const float* L = n.wq + LAYER0 + l * L_SIZE;
    launch_gemm_tc_image(L + L_U, H, n.bimg + l * BIMG_LSIZE + BIMG_U, s);
    launch_gemm_tc_image(L + L_W, 2 * H, n.bimg + l * BIMG_LSIZE + BIMG_W, s);
  }
}

void learned_forward(const LsView& s, const NetDev& n, LearnedWork& w, float* S, SPcg pcg, cudaStream_t st, int* err) {
  const int V = s.V;
  if (V == 0) return;
  const float* wq = n.wq;
  k_edge_feats<<<nblk(s.nnzb), TPB, 0, st>>>(s.nnzb, s.valh, w.Ef);
  k_node_feats<<<nblk(V), TPB, 0, st>>>(s, w.Ef, w.X);
  // pre-activations (Q) are kept for the training backward only
  gemm(V, w.X, FN, FN, nullptr, 0, 0, n.wt + WT_IN, H, wq + B_IN, nullptr, 0, nullptr, 0, w.training ? w.q0 : nullptr, w.h[0], 1, st);
  const int wgrid = nblk(32ll * V);
  for (int l = 0; l < NL; ++l) {
    const float* L = wq + LAYER0 + l * L_SIZE;
    // u = U h and h' = relu(W [h ; m] + b) + h on the tensor cores
    const unsigned short* bi = n.bimg ? n.bimg + l * BIMG_LSIZE : nullptr;
    // u = U h: its own launch for the first layer, fused into the previous
    // layer's update launch (same bits) for the others when the images exist
    if (l == 0 || !bi)
      launch_gemm_tc(V, w.h[l], H, H, nullptr, 0, 0, L + L_U, bi ? bi + BIMG_U : nullptr, nullptr, nullptr, 0, nullptr, w.u[l], 0, err, st);
    if (n.host_wq && !w.training) {
      MsgWeights P;
      const float* Lh = n.host_wq + LAYER0 + l * L_SIZE;
      for (int q = 0; q < H * FE; ++q) P.E[q] = Lh[L_E + q];
      for (int q = 0; q < H; ++q) P.c[q] = Lh[L_C + q];
      k_msg_rows<<<nblk(V, MSG_ROWS_TPB), MSG_ROWS_TPB, 0, st>>>(s, w.u[l], w.Ef, P, w.m[l]);
    } else {
      k_msg_fwd<<<wgrid, TPB, 0, st>>>(s, w.u[l], w.Ef, L + L_E, L + L_C, w.m[l]);
    }
    const unsigned short* bnext = bi && l + 1 < NL ? n.bimg + (l + 1) * BIMG_LSIZE + BIMG_U : nullptr;
    launch_gemm_tc(V, w.h[l], H, H, w.m[l], H, H, L + L_W, bi ? bi + BIMG_W : nullptr, L + L_B, w.h[l], H, w.training ? w.q[l] : nullptr,
                   w.h[l + 1], 1, err, st, bnext, bnext ? w.u[l + 1] : nullptr);
  }
  k_dec_fwd<<<wgrid, TPB, 0, st>>>(s, w.h[NL], w.Ef, wq, w.zv, w.ab);
  k_build_S<<<nblk(V), TPB, 0, st>>>(s, w.zv, w.ab, S, pcg);
}

void learned_build_S(const LsView& s, const LearnedWork& w, float* S, SPcg pcg, cudaStream_t st) {
  if (s.V) k_build_S<<<nblk(s.V), TPB, 0, st>>>(s, w.zv, w.ab, S, pcg);
}

void learned_loss(const LsView& s, const NetDev& n, LearnedWork& w, float* S, const float* probes, const double* pnorm, int P,
                  float* Y, float* Wv, double* loss_parts, double* loss_out, float* grad, cudaStream_t st) {
  const int V = s.V;
  learned_forward(s, n, w, S, SPcg{}, st);
  const int wgrid = nblk(32ll * V);
  for (int p = 0; p < P; ++p) {
    k_spmv<<<wgrid, TPB, 0, st>>>(V, s.rowptr, s.cols, S, nullptr, nullptr, nullptr, nullptr, probes + 3ll * V * p, Y + 3ll * V * p);
    k_spmv<<<wgrid, TPB, 0, st>>>(V, s.rowptr, s.cols, s.valh, s.xbegin, s.xend, s.xcols, s.xvalh, Y + 3ll * V * p, Wv + 3ll * V * p);
  }
  k_loss_terms<<<GRID, TPB, 0, st>>>(V, P, probes, Y, Wv, loss_parts);
  k_loss_final<<<1, 32, 0, st>>>(loss_parts, GRID, P, pnorm, loss_out);
  if (!grad || !w.training) return;
  const float* wq = n.wq;
  k_coef_grad<<<nblk(V), TPB, 0, st>>>(s, P, probes, Wv, pnorm, w.zv, w.ab, w.dzv, w.dab);
  k_dec_bwd<<<GRID, TPB, 0, st>>>(s, w.h[NL], w.Ef, wq, w.dzv, w.dab, w.dh, w.part);
  reduce(w.part, 0, H + 1 + 2 * DE_IN + 2, grad + DV, st);
  float* dh = w.dh;
  float* dh_prev = w.dh2;
  const long long VH = (long long)V * H;
  for (int l = NL - 1; l >= 0; --l) {
    const float* L = wq + LAYER0 + l * L_SIZE;
    float* G = grad + LAYER0 + l * L_SIZE;
    k_relu_mask<<<nblk(VH), TPB, 0, st>>>(VH, dh, w.q[l], w.dq);
    k_wgrad<<<GRID, TPB, 0, st>>>(V, w.dq, H, w.h[l], H, H, w.m[l], H, H, w.part);
    reduce(w.part, 0, H * 2 * H + H, G + L_W, st);       // W then its bias (L_B follows L_W)
    gemm(V, w.dq, H, H, nullptr, 0, 0, L + L_W, 2 * H, nullptr, nullptr, 0, nullptr, 0, nullptr, w.dhm, 0, st);
    k_msg_bwd<<<GRID, TPB, 0, st>>>(s, w.u[l], w.Ef, L + L_E, L + L_C, w.dhm + H, 2 * H, w.du, w.part);
    reduce(w.part, 0, H * FE + H, G + L_E, st);          // E then c (L_C follows L_E)
    k_wgrad<<<GRID, TPB, 0, st>>>(V, w.du, H, w.h[l], H, H, nullptr, 0, 0, w.part);
    reduce(w.part, 0, H * H, G + L_U, st);
    gemm(V, w.du, H, H, nullptr, 0, 0, L + L_U, H, nullptr, dh, H, w.dhm, 2 * H, nullptr, dh_prev, 0, st);
    float* t = dh; dh = dh_prev; dh_prev = t;
  }
  k_relu_mask<<<nblk(VH), TPB, 0, st>>>(VH, dh, w.q0, w.dq);
  k_wgrad<<<GRID, TPB, 0, st>>>(V, w.dq, H, w.X, FN, FN, nullptr, 0, 0, w.part);
  reduce(w.part, 0, H * FN + H, grad + W_IN, st);        // W_in then b_in
}

void launch_adam(float* master, float* m1, float* m2, const float* grad, int n, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t s) {
  float c1 = 1.f - powf(b1, float(t)), c2 = 1.f - powf(b2, float(t));
  k_adam<<<nblk(n), TPB, 0, s>>>(master, m1, m2, grad, n, lr, b1, b2, eps, c1, c2);
}

}  // namespace ando
