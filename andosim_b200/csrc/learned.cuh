// learned.cuh -- the learned block-sparse approximate inverse of the scaled
// Newton system (no reference counterpart: the reference's only
// preconditioner is block Jacobi, pcg_solver.cpp:77-114).
//
// The preconditioner S approximates A^-1 for the block-scaled system
// A^ = L^-1 A L^-T on the static mesh pattern and is symmetric positive
// definite by construction:
//   S = sum_i delta_i E_ii  +  sum_{edges e = (i < j)} W_e W_e^T,
//   W_e = [a_e I ; b_e A^_ij^T]   (6 x 3, rows of vertex i then vertex j)
// so S_ij = a_e b_e A^_ij, and the diagonal block of a vertex collects
// delta_i I, a_e^2 I from the edges where it is the smaller index and
// b_e^2 A^_ij^T A^_ij from those where it is the larger one. delta_i > 0 and
// (a_e, b_e) come from a mesh-graph message-passing network over per-vertex
// and per-edge features of A^ (3 layers, 64 wide, BF16 weights, FP32
// accumulation).
#pragma once

#include "common.cuh"

namespace ando {
namespace net {
constexpr int FN = 8;              // node features
constexpr int FE = 10;             // edge features (the 9 entries of A^_ij and its Frobenius norm)
constexpr int FES = 12;            // row stride of the edge features in memory (16-byte rows)
constexpr int H = 64;              // width
constexpr int NL = 3;              // message-passing layers
constexpr int DE_IN = 2 * H + FE;  // edge decoder input [h_i ; h_j ; e_ij]
// offsets into the flat parameter vector; dense weights are row-major [out][in]
constexpr int W_IN = 0;
constexpr int B_IN = W_IN + H * FN;
constexpr int LAYER0 = B_IN + H;
constexpr int L_U = 0;                   // H x H      u = U h
constexpr int L_E = L_U + H * H;         // H x FE     message edge term
constexpr int L_C = L_E + H * FE;        // H          message bias
constexpr int L_W = L_C + H;             // H x 2H     update [h ; m]
constexpr int L_B = L_W + H * 2 * H;     // H          update bias
constexpr int L_SIZE = L_B + H;
constexpr int DV = LAYER0 + NL * L_SIZE; // H          vertex decoder
constexpr int DV0 = DV + H;              // 1
constexpr int DE = DV0 + 1;              // 2 x DE_IN  edge decoder
constexpr int DE0 = DE + 2 * DE_IN;      // 2
constexpr int NPARAM = DE0 + 2;
constexpr float DELTA_MIN = 1e-4f;       // delta_i = softplus(z_i) + DELTA_MIN
}  // namespace net

// A scaled system on the static pattern plus the extra contact segment.
struct LsView {
  int V, nnzb;
  const int* rowptr; const int* cols; const int* slot_row; const int* slot_T;
  const int* sell_base;         // SELL-32 position of each static slot (writes of S in the PCG layout); may be null
  const float* valh;
  const int* xbegin; const int* xend; const int* xcols; const float* xvalh;  // null when no extra blocks
  const float* Lf;              // 6V packed Cholesky factor of the unscaled diagonal blocks
  const double* mass;           // V
  const unsigned char* fixed;   // V (may be null)
  double dt2inv;
};

// Device activations of one forward (and backward) pass.
struct LearnedWork {
  int V = 0, nnzb = 0;
  bool training = false;
  float* base = nullptr;
  float *X, *Ef;                        // V x FN, nnzb x FES
  float *h[net::NL + 1], *u[net::NL], *m[net::NL], *q[net::NL], *q0;
  float *zv, *ab;                       // V, 2 nnzb
  // backward
  float *dh, *dh2, *du, *dhm, *dq, *dzv, *dab;
  float* part;                          // per-CTA weight-gradient partials
};

size_t learned_work_floats(int V, int nnzb, bool training);
void learned_work_carve(LearnedWork& w, float* base, int V, int nnzb, bool training);

// Weights as used by the kernels: FP32 values rounded to BF16 (wq), the
// transposed dense matrices for the forward products, and BF16 storage.
struct NetDev {
  float* wq = nullptr;       // NPARAM, BF16-representable values
  float* wt = nullptr;       // transposed copies of the dense matrices (forward layout)
  unsigned short* bimg = nullptr;  // hidden layers' U and W as tensor-core B operand images (launch_gemm_tc_image)
  const float* host_wq = nullptr;  // host copy of wq (may be null): lets inference pass small weight blocks by value
};
size_t net_dev_floats();
void net_dev_carve(NetDev& n, float* base);
// Round master weights to BF16 into n.wq (and bf16 storage) and build n.wt.
void launch_net_prepare(const float* master, NetDev n, unsigned short* bf16, cudaStream_t s);

// S in the form the PCG applies it: off the diagonal S_ij = coef * A^_ij, so
// one coefficient per SELL-32 slot (at slot position chunk_off + 32 k + lane,
// like sell_col) and the 3x3 diagonal blocks (9 per vertex, row-major).
struct SPcg { float* coef = nullptr; float* diag = nullptr; };

// Inference: features, network, S (9 floats per static slot when S is not
// null; the PCG form when pcg.coef is not null). The hidden dense layers run
// on the tensor cores (tc_gemm.cu); `err` (may be null) is set when one of
// their bounded waits gives up.
void learned_forward(const LsView& s, const NetDev& n, LearnedWork& w, float* S, SPcg pcg, cudaStream_t st, int* err = nullptr);

// Tensor-core dense layer (tc_gemm.cu): Y = act(X W^T + bias) + R1 with
// X = [X1 | X2] (K = K1 + K2 in 16..128, a multiple of 16), W row-major
// [64][K] BF16-representable, 64 outputs.
// Bimg (may be null): W's B operand image from launch_gemm_tc_image (64 K
// BF16 values, 16-byte aligned), copied instead of converting W per CTA.
bool gemm_tc_supported(int K1, int K2, int N, int ldr1);
// Bimg2 (may be null): the B image of a 64 x 64 matrix U; the launch then
// also writes Y2 = Y U^T (the next layer's U product, fused).
cudaError_t launch_gemm_tc(int V, const float* X1, int ld1, int K1, const float* X2, int ld2, int K2, const float* W,
                           const unsigned short* Bimg, const float* bias, const float* R1, int ldr1, float* Q, float* Y, int relu, int* err,
                           cudaStream_t s, const unsigned short* Bimg2 = nullptr, float* Y2 = nullptr);
cudaError_t launch_gemm_tc_image(const float* W, int K, unsigned short* img, cudaStream_t s);

// S from the coefficients of the last forward (w.zv, w.ab) and the current
// A^: the network output reused while A^ changes; still SPD by construction.
void learned_build_S(const LsView& s, const LearnedWork& w, float* S, SPcg pcg, cudaStream_t st);

// Training loss of one system: P probe vectors r_p (3V each) with energy
// norms n_p = r_p^T A^-1 r_p; loss = mean_p (1 + (y^T A y - 2 r^T y) / n_p),
// y = S r_p (the relative A-norm error of one preconditioned Richardson step
// from zero). With grad != null also the gradient w.r.t. the master weights.
void learned_loss(const LsView& s, const NetDev& n, LearnedWork& w, float* S, const float* probes, const double* pnorm, int P,
                  float* Y, float* Wv, double* loss_parts, double* loss_out, float* grad, cudaStream_t st);

void launch_adam(float* master, float* m1, float* m2, const float* grad, int n, float lr, float b1, float b2, float eps, int t,
                 cudaStream_t s);

}  // namespace ando
