// tc_gemm.cu -- dense layers of the learned preconditioner's forward pass on
// the 5th-generation tensor cores: tcgen05.mma (kind::f16, BF16 x BF16 with
// an FP32 accumulator in tensor memory), operands staged in shared memory in
// the K-major no-swizzle core-matrix layout, one elected thread issuing the
// MMAs, completion through tcgen05.commit on an mbarrier, epilogue read back
// with tcgen05.ld.
//
// The weights are BF16 values already (the network's master weights are
// rounded to BF16). The FP32 activations are split exactly into three BF16
// terms x = hi + mid + lo (8 + 8 + 8 mantissa bits); every BF16 x BF16
// product is exact in FP32, so the layer keeps FP32-level accuracy with the
// BF16 weights, and three MMAs per K step cost nothing on a layer that is
// bound by reading its FP32 inputs.
#include <atomic>

#include <cuda_bf16.h>

#include "learned.cuh"

namespace ando {

namespace {

__device__ int g_tc_err;  // timeout flag of launches given no flag of their own

constexpr int TC_M = 128;        // rows per CTA (one tensor-memory lane per row)
constexpr int TC_N = 64;         // outputs per row (the network width)
constexpr int TC_THREADS = 256;  // eight warps: warp w reads tensor-memory lanes 32 (w % 4).. and columns 32 (w / 4)..
constexpr int TC_COLS_PER_WARP = TC_N / (TC_THREADS / 128);
constexpr int TC_SPLITS = 3;

__device__ inline uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Byte offset of element (r, k) in a K-major tile with K columns and no
// swizzle: 8 x 16-byte core matrices, consecutive along K (128 bytes apart),
// 8-row groups K * 16 bytes apart.
__device__ inline int core_off(int r, int k, int K) { return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

// Shared-memory matrix descriptor (sm_100): start address, leading byte
// offset (between core matrices along K), stride byte offset (between 8-row
// groups), descriptor version 1, no swizzle.
__device__ inline uint64_t smem_desc(uint32_t addr, int K) {
  uint64_t d = uint64_t((addr >> 4) & 0x3fff);
  d |= uint64_t((128 >> 4) & 0x3fff) << 16;
  d |= uint64_t(((K * 16) >> 4) & 0x3fff) << 32;
  d |= uint64_t(1) << 46;
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4
// at bit 24.
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(TC_N >> 3) << 17) | (uint32_t(TC_M >> 4) << 24);

__device__ inline void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, int acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ inline bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the barrier's phase of the given parity (about a second
// at most).
__device__ inline bool mbar_wait_bounded(uint32_t bar, uint32_t parity = 0) {
  for (long long it = 0; it < (1ll << 22); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (it > 32) __nanosleep(128);
  }
  return false;
}

__device__ inline uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return uint32_t(__bfloat16_as_ushort(a)) | (uint32_t(__bfloat16_as_ushort(b)) << 16);
}

// Split four FP32 values exactly into three BF16 4-vectors (hi, mid, lo).
__device__ inline void split3(const float f[4], uint32_t w[3][2]) {
#pragma unroll
  for (int e = 0; e < 4; e += 2) {
    __nv_bfloat16 h0 = __float2bfloat16_rn(f[e]), h1 = __float2bfloat16_rn(f[e + 1]);
    float s0 = f[e] - __bfloat162float(h0), s1 = f[e + 1] - __bfloat162float(h1);
    __nv_bfloat16 m0 = __float2bfloat16_rn(s0), m1 = __float2bfloat16_rn(s1);
    __nv_bfloat16 l0 = __float2bfloat16_rn(s0 - __bfloat162float(m0)), l1 = __float2bfloat16_rn(s1 - __bfloat162float(m1));
    w[0][e / 2] = pack2(h0, h1); w[1][e / 2] = pack2(m0, m1); w[2][e / 2] = pack2(l0, l1);
  }
}

__device__ inline void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]),
        "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}


// B image: W (64 x K, row-major, BF16-representable) as BF16 in the shared
// memory layout of the MMA's B operand, 128 K bytes.
__global__ void k_gemm_tc_image(const float* __restrict__ W, int K, unsigned short* __restrict__ img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= TC_N * K) return;
  const int n = i / K, k = i - n * K;
  img[core_off(n, k, K) >> 1] = __bfloat16_as_ushort(__float2bfloat16_rn(W[i]));
}

constexpr int TC_AV = TC_M * 128 / 4 / TC_THREADS;  // float4 loads per thread of the A tile at K = 128

// Y[r, :64] = act(X[r, :] W^T + bias) + R1[r, :64], X = [X1 | X2] (K = K1 + K2,
// a multiple of 16, at most 128; K1 a multiple of 8; rows 16-byte aligned),
// W row-major [64][K] (BF16-representable), or its B image Bimg when not
// null; Q (may be null) gets the pre-activation. res_a: R1 is X1 itself (the
// first 64 columns), taken from the A tile in shared memory, whose three
// BF16 terms sum back to the FP32 value exactly.
__global__ void __launch_bounds__(TC_THREADS) k_gemm_tc(int V, const float* __restrict__ X1, int ld1, int K1, const float* __restrict__ X2,
                                                        int ld2, int K2, const float* __restrict__ W, const uint4* __restrict__ Bimg,
                                                        const float* __restrict__ bias, const float* __restrict__ R1, int ldr1, int res_a,
                                                        float* __restrict__ Q, float* __restrict__ Y, int relu, int* err,
                                                        const uint4* __restrict__ Bimg2, float* __restrict__ Y2) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int K = K1 + K2;
  const int tile = TC_M * K * 2;  // bytes of one BF16 split of the row tile
  unsigned char* A = sm;
  unsigned char* B = sm + TC_SPLITS * tile;
  uint64_t* bar = reinterpret_cast<uint64_t*>(B + TC_N * K * 2);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int r0 = blockIdx.x * TC_M;
  const uint32_t bar_a = smem_u32(bar);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)), "r"(TC_N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar_a), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  // B: the image (16-byte copies), or W converted here (exact in BF16)
  constexpr int TC_BV = TC_N * 128 * 2 / 16 / TC_THREADS;
  uint4 bv[TC_BV];
  const int nb16 = TC_N * K * 2 / 16;
  if (Bimg) {
#pragma unroll
    for (int j = 0; j < TC_BV; ++j) {
      const int i = tid + j * TC_THREADS;
      if (i < nb16) bv[j] = Bimg[i];
    }
  } else {
    for (int i = tid; i < TC_N * K; i += TC_THREADS) {
      const int n = i / K, k = i - n * K;
      *reinterpret_cast<__nv_bfloat16*>(B + core_off(n, k, K)) = __float2bfloat16_rn(W[i]);
    }
  }
  // A: coalesced 16-byte loads (consecutive threads take consecutive
  // 4-column groups of a row), all issued before the first is used, then
  // each split into three BF16 4-vectors
  {
    const int K4 = K >> 2, n4 = TC_M * K4;
    float4 av[TC_AV];
#pragma unroll
    for (int j = 0; j < TC_AV; ++j) {
      const int c = tid + j * TC_THREADS;
      const int r = c / K4, k = (c - r * K4) << 2, row = r0 + r;
      av[j] = make_float4(0.f, 0.f, 0.f, 0.f);
      if (c < n4 && row < V)
        av[j] = k < K1 ? *reinterpret_cast<const float4*>(X1 + (long long)row * ld1 + k)
                       : *reinterpret_cast<const float4*>(X2 + (long long)row * ld2 + (k - K1));
    }
    if (Bimg) {
#pragma unroll
      for (int j = 0; j < TC_BV; ++j) {
        const int i = tid + j * TC_THREADS;
        if (i < nb16) reinterpret_cast<uint4*>(B)[i] = bv[j];
      }
    }
#pragma unroll
    for (int j = 0; j < TC_AV; ++j) {
      const int c = tid + j * TC_THREADS;
      if (c >= n4) break;
      const int r = c / K4, k = (c - r * K4) << 2;
      const float f[4] = {av[j].x, av[j].y, av[j].z, av[j].w};
      uint32_t w[TC_SPLITS][2];
      split3(f, w);
      const int off = core_off(r, k, K);  // k % 4 == 0: 8-byte aligned inside a 16-byte core-matrix row
#pragma unroll
      for (int sp = 0; sp < TC_SPLITS; ++sp) *reinterpret_cast<uint2*>(A + sp * tile + off) = make_uint2(w[sp][0], w[sp][1]);
    }
  }
  // generic-proxy shared stores -> visible to the tensor core (async proxy)
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tslot;
  if (tid == 0) {
    int first = 1;
    for (int sp = 0; sp < TC_SPLITS; ++sp)
      for (int kk = 0; kk < K / 16; ++kk) {
        const uint64_t ad = smem_desc(smem_u32(A + sp * tile + kk * 256), K);
        const uint64_t bd = smem_desc(smem_u32(B + kk * 256), K);
        mma_f16(tmem, ad, bd, TC_IDESC, first ? 0 : 1);
        first = 0;
      }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_a) : "memory");
  }
  const bool done = mbar_wait_bounded(bar_a);
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  float hv[TC_COLS_PER_WARP];  // this thread's outputs, the input of the fused second product
#pragma unroll
  for (int c = 0; c < TC_COLS_PER_WARP; ++c) hv[c] = 0.f;
  if (done) {
    // warp w: tensor-memory lanes (rows) 32 (w % 4) + lane, columns c0 .. c0 + 31
    const int quarter = warp & 3, c0 = (warp >> 2) * TC_COLS_PER_WARP;
    float acc[TC_COLS_PER_WARP];
    const uint32_t taddr = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(c0);
#pragma unroll
    for (int c = 0; c < TC_COLS_PER_WARP; c += 16) tmem_ld16(taddr + c, acc + c);
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    const int row = r0 + quarter * 32 + (tid & 31);
    if (row < V) {
      float4* yr = reinterpret_cast<float4*>(Y + (long long)row * TC_N + c0);
      float4* qr = Q ? reinterpret_cast<float4*>(Q + (long long)row * TC_N + c0) : nullptr;
      const float4* rr = R1 && !res_a ? reinterpret_cast<const float4*>(R1 + (long long)row * ldr1 + c0) : nullptr;
      float res[TC_COLS_PER_WARP];
      if (res_a) {
        const int r = quarter * 32 + (tid & 31);
#pragma unroll
        for (int c8 = 0; c8 < TC_COLS_PER_WARP; c8 += 8) {
          const int off = core_off(r, c0 + c8, K);
          const uint4 h = *reinterpret_cast<const uint4*>(A + off), m = *reinterpret_cast<const uint4*>(A + tile + off),
                      l = *reinterpret_cast<const uint4*>(A + 2 * tile + off);
          const uint32_t hw[4] = {h.x, h.y, h.z, h.w}, mw[4] = {m.x, m.y, m.z, m.w}, lw[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int sh = (e & 1) * 16;
            const float fh = __uint_as_float(((hw[e >> 1] >> sh) & 0xffffu) << 16);
            const float fm = __uint_as_float(((mw[e >> 1] >> sh) & 0xffffu) << 16);
            const float fl = __uint_as_float(((lw[e >> 1] >> sh) & 0xffffu) << 16);
            res[c8 + e] = (fh + fm) + fl;
          }
        }
      }
#pragma unroll
      for (int c4 = 0; c4 < TC_COLS_PER_WARP / 4; ++c4) {
        float q[4], y[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          q[e] = acc[4 * c4 + e] + (bias ? bias[c0 + 4 * c4 + e] : 0.f);
          y[e] = relu ? fmaxf(q[e], 0.f) : q[e];
        }
        if (qr) qr[c4] = make_float4(q[0], q[1], q[2], q[3]);
        if (rr) {
          const float4 t = rr[c4];
          y[0] += t.x; y[1] += t.y; y[2] += t.z; y[3] += t.w;
        } else if (res_a) {
#pragma unroll
          for (int e = 0; e < 4; ++e) y[e] += res[4 * c4 + e];
        }
        yr[c4] = make_float4(y[0], y[1], y[2], y[3]);
#pragma unroll
        for (int e = 0; e < 4; ++e) hv[4 * c4 + e] = y[e];
      }
    }
  } else if (tid == 0) {
    atomicExch(err ? err : &g_tc_err, 1);
    mbar_wait_bounded(bar_a);  // give the MMAs in flight a second bound before the accumulator is freed
  }
  // Fused second product Y2 = Y U^T (U: 64 x 64, its B image Bimg2): Y's tile
  // goes back into shared memory as three BF16 terms (K = 64 layout) and one
  // more set of MMAs reuses the accumulator columns, whose loads have all
  // completed. The result is the bits a separate launch on Y gives.
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  if (Bimg2 && __syncthreads_and(done)) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    constexpr int K2 = TC_N, tile2 = TC_M * K2 * 2;
    for (int i = tid; i < TC_N * K2 * 2 / 16; i += TC_THREADS) reinterpret_cast<uint4*>(B)[i] = Bimg2[i];
    {
      const int quarter = warp & 3, c0 = (warp >> 2) * TC_COLS_PER_WARP, r = quarter * 32 + (tid & 31);
#pragma unroll
      for (int c4 = 0; c4 < TC_COLS_PER_WARP / 4; ++c4) {
        const float f[4] = {hv[4 * c4], hv[4 * c4 + 1], hv[4 * c4 + 2], hv[4 * c4 + 3]};
        uint32_t w[TC_SPLITS][2];
        split3(f, w);
        const int off = core_off(r, c0 + 4 * c4, K2);
#pragma unroll
        for (int sp = 0; sp < TC_SPLITS; ++sp) *reinterpret_cast<uint2*>(A + sp * tile2 + off) = make_uint2(w[sp][0], w[sp][1]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (tid == 0) {
      int first = 1;
      for (int sp = 0; sp < TC_SPLITS; ++sp)
        for (int kk = 0; kk < K2 / 16; ++kk) {
          const uint64_t ad = smem_desc(smem_u32(A + sp * tile2 + kk * 256), K2);
          const uint64_t bd = smem_desc(smem_u32(B + kk * 256), K2);
          mma_f16(tmem, ad, bd, TC_IDESC, first ? 0 : 1);
          first = 0;
        }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_a) : "memory");
    }
    const bool done2 = mbar_wait_bounded(bar_a, 1);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (done2) {
      const int quarter = warp & 3, c0 = (warp >> 2) * TC_COLS_PER_WARP;
      float acc[TC_COLS_PER_WARP];
      const uint32_t taddr = tmem + (uint32_t(quarter * 32) << 16) + uint32_t(c0);
#pragma unroll
      for (int c = 0; c < TC_COLS_PER_WARP; c += 16) tmem_ld16(taddr + c, acc + c);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      const int row = r0 + quarter * 32 + (tid & 31);
      if (row < V) {
        float4* ur = reinterpret_cast<float4*>(Y2 + (long long)row * TC_N + c0);
#pragma unroll
        for (int c4 = 0; c4 < TC_COLS_PER_WARP / 4; ++c4) ur[c4] = make_float4(acc[4 * c4], acc[4 * c4 + 1], acc[4 * c4 + 2], acc[4 * c4 + 3]);
      }
    } else if (tid == 0) {
      atomicExch(err ? err : &g_tc_err, 1);
      mbar_wait_bounded(bar_a, 1);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TC_N));
  }
}

}  // namespace

size_t gemm_tc_smem(int K) { return size_t(TC_SPLITS) * TC_M * K * 2 + size_t(TC_N) * K * 2 + 16; }

bool gemm_tc_supported(int K1, int K2, int N, int ldr1) {
  const int K = K1 + K2;
  return N == TC_N && K >= 16 && K <= 128 && K % 16 == 0 && K1 % 8 == 0 && (ldr1 % 4) == 0;
}
static_assert(TC_THREADS % 128 == 0 && TC_COLS_PER_WARP % 16 == 0, "epilogue: whole tensor-memory lane quarters, 16-column loads");

cudaError_t launch_gemm_tc_image(const float* W, int K, unsigned short* img, cudaStream_t s) {
  if (K < 16 || K > 128 || K % 16) return cudaErrorInvalidValue;
  k_gemm_tc_image<<<(TC_N * K + 255) / 256, 256, 0, s>>>(W, K, img);
  return cudaGetLastError();
}

cudaError_t launch_gemm_tc(int V, const float* X1, int ld1, int K1, const float* X2, int ld2, int K2, const float* W,
                           const unsigned short* Bimg, const float* bias, const float* R1, int ldr1, float* Q, float* Y, int relu, int* err,
                           cudaStream_t s, const unsigned short* Bimg2, float* Y2) {
  if (V <= 0) return cudaSuccess;
  if (!gemm_tc_supported(K1, K2, TC_N, R1 ? ldr1 : 0)) return cudaErrorInvalidValue;
  auto a16 = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  if (!a16(Y) || (Q && !a16(Q)) || (R1 && !a16(R1))) return cudaErrorInvalidValue;  // float4 epilogue
  if (!a16(X1) || (ld1 & 3) || (K2 && (!a16(X2) || (ld2 & 3)))) return cudaErrorInvalidValue;  // float4 staging
  if (Bimg && !a16(Bimg)) return cudaErrorInvalidValue;
  if (Bimg2 && (!a16(Bimg2) || !Y2 || !a16(Y2))) return cudaErrorInvalidValue;
  const int res_a = R1 && R1 == X1 && ldr1 == ld1 && K1 >= TC_N;
  static std::atomic<unsigned> attr{0};  // one bit per device (steps of several contexts may run on host threads)
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 32 && !(attr.load() & (1u << dev))) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, int(gemm_tc_smem(128)));
    if (e != cudaSuccess) return e;
    attr.fetch_or(1u << dev);
  }
  const int K = K1 + K2;
  k_gemm_tc<<<(V + TC_M - 1) / TC_M, TC_THREADS, gemm_tc_smem(K), s>>>(V, X1, ld1, K1, X2, ld2, K2, W, reinterpret_cast<const uint4*>(Bimg),
                                                                      bias, R1, ldr1, res_a, Q, Y, relu, err,
                                                                      reinterpret_cast<const uint4*>(Bimg2), Y2);
  return cudaGetLastError();
}

}  // namespace ando
