// noalloc.cu -- block-Jacobi PCG on a caller-owned BSR system that allocates
// no device memory: ando_pcg_solve_noalloc (include/ando_gpu.h).
//
// Who needs it: callers that cannot allocate device memory at solve time. A
// host that hands out all device memory from its own fixed arena (an
// embedding application with a hard memory budget) cannot have a library
// call cudaMalloc behind its back, and a host that interleaves solves with
// other work on a busy device cannot take the device-wide synchronisation
// that cudaFree performs. Every other entry point of this library keeps its
// buffers in the context and grows them on demand, which allocates.
//
// What it runs: the persistent cooperative PCG kernel of pcg.cu (the same
// iteration as PCGSolver::solve, pcg_solver.cpp:8-146), preceded by a kernel
// that forms the block-Jacobi inverse from the matrix's diagonal blocks
// exactly as the assembly kernel does. The kernel's per-CTA reduction
// partials and its grid-barrier control words, which the context-based path
// keeps in context buffers, live here in one file-scope static device array.
// Vectors live in the caller's work buffer.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ando_gpu.h"
#include "kernels.cuh"

namespace ando {
int set_last_error(int code, const char* msg);
}

using namespace ando;

namespace {

// Scratch layout: [Ctrl control block, padded to 256 B][3 x kMaxCtas FP64 partials].
constexpr int kCtrlBytes = 256;
constexpr int kMaxCtas = 640;
constexpr size_t kScratchBytes = 16384;
static_assert(sizeof(Ctrl) <= kCtrlBytes, "control block does not fit its slot");
static_assert(kCtrlBytes + 3ull * kMaxCtas * sizeof(double) <= kScratchBytes, "partials do not fit the scratch");

// One 16 KiB scratch per device (the array is instantiated in every device's
// copy of the module). It starts zeroed at module load; each call zeroes the
// control block again before its solve, so nothing needs zeroing by the caller.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {};
int g_grid[kMaxDevices] = {};

// Block-Jacobi inverse from the diagonal blocks, the same arithmetic as the
// assembly kernel (pcg_solver.cpp:77-114): FP64 cofactors of the FP32 block,
// identity when |det| <= 1e-16 or when the row has no diagonal block.
__global__ void k_noalloc_jacobi(int V, const int* rowptr, const int* cols, const float* val, float* P) {
  int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= V) return;
  float* out = P + 9 * (long long)row;
  int s = -1;
  for (int k = rowptr[row]; k < rowptr[row + 1]; ++k)
    if (cols[k] == row) { s = k; break; }
  if (s < 0) {
    for (int k = 0; k < 9; ++k) out[k] = (k % 4 == 0) ? 1.f : 0.f;
    return;
  }
  const float* h = val + 9 * (long long)s;
  double a0 = h[0], a1 = h[1], a2 = h[2], a3 = h[3], a4 = h[4], a5 = h[5], a6 = h[6], a7 = h[7], a8 = h[8];
  double c00 = a4 * a8 - a5 * a7, c01 = a2 * a7 - a1 * a8, c02 = a1 * a5 - a2 * a4;
  double c10 = a5 * a6 - a3 * a8, c11 = a0 * a8 - a2 * a6, c12 = a2 * a3 - a0 * a5;
  double c20 = a3 * a7 - a4 * a6, c21 = a1 * a6 - a0 * a7, c22 = a0 * a4 - a1 * a3;
  double det = a0 * c00 + a1 * c10 + a2 * c20;
  if (fabs(det) > 1e-16) {
    double inv = 1.0 / det;
    out[0] = float(c00 * inv); out[1] = float(c01 * inv); out[2] = float(c02 * inv);
    out[3] = float(c10 * inv); out[4] = float(c11 * inv); out[5] = float(c12 * inv);
    out[6] = float(c20 * inv); out[7] = float(c21 * inv); out[8] = float(c22 * inv);
  } else {
    for (int k = 0; k < 9; ++k) out[k] = (k % 4 == 0) ? 1.f : 0.f;
  }
}

// Device-side address of this device's scratch, looked up once per device
// with that device current (the host-side symbol is not a device address).
int scratch_for(int device, void** ptr, int* grid) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_last_error(ANDO_ERR_CUDA, "ando_pcg_solve_noalloc: cudaGetSymbolAddress of the scratch failed");
    }
    int g = pcg_grid_size(device);
    g_grid[device] = g < 1 ? 1 : (g > kMaxCtas ? kMaxCtas : g);
    g_scratch_ptr[device] = p;
  }
  *ptr = g_scratch_ptr[device];
  *grid = g_grid[device];
  return ANDO_OK;
}

int solve(int32_t device, cudaStream_t s, int32_t V, const int32_t* rowptr, const int32_t* cols, const float* vals,
          const float* rhs, float* x, float* work, int64_t work_floats, double tol, int32_t max_iters, int32_t* iterations,
          int32_t* pcg_status, double* rel_residual) {
  if (V < 1 || !rowptr || !cols || !vals || !rhs || !x || !work || max_iters < 0 || !(tol >= 0.0))
    return set_last_error(ANDO_ERR_INVALID, "ando_pcg_solve_noalloc: invalid argument");
  if (V > ANDO_NOALLOC_MAX_ROWS)
    return set_last_error(ANDO_ERR_CAPACITY, "ando_pcg_solve_noalloc: num_rows exceeds ANDO_NOALLOC_MAX_ROWS");
  if (work_floats < 24ll * V)
    return set_last_error(ANDO_ERR_CAPACITY, "ando_pcg_solve_noalloc: work buffer smaller than 24 * num_rows floats");
  void* scratch = nullptr;
  int grid = 1;
  int rc = scratch_for(device, &scratch, &grid);
  if (rc) return rc;
  if (kCtrlBytes + 3ull * grid * sizeof(double) > kScratchBytes)
    return set_last_error(ANDO_ERR_CAPACITY, "ando_pcg_solve_noalloc: grid needs more partials than the scratch holds");
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(scratch);
  PcgArgs a{};
  a.V = V;
  a.rowptr = rowptr; a.cols = cols; a.val = vals;
  a.xbegin = nullptr; a.xend = nullptr; a.xcols = nullptr; a.xval = nullptr;
  a.P = work;
  a.b = rhs;
  a.x = x;
  a.r = work + 9ll * V; a.z = work + 12ll * V; a.p0 = work + 15ll * V; a.p1 = work + 18ll * V; a.Ap = work + 21ll * V;
  a.partials = reinterpret_cast<double*>(static_cast<unsigned char*>(scratch) + kCtrlBytes);
  a.ctrl = ctrl;
  a.tol = float(tol);
  a.max_iters = max_iters;
  // zero the control block (barrier words, error flag, converged flag)
  cudaError_t e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), s);
  if (e == cudaSuccess) {
    k_noalloc_jacobi<<<(V + 255) / 256, 256, 0, s>>>(V, rowptr, cols, vals, work);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = launch_pcg(a, grid, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_last_error(ANDO_ERR_CUDA, cudaGetErrorString(e));
  }
  if (!iterations && !pcg_status && !rel_residual) return ANDO_OK;  // asynchronous
  Ctrl h;
  e = cudaMemcpyAsync(&h, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return set_last_error(ANDO_ERR_CUDA, cudaGetErrorString(e));
  if (iterations) *iterations = h.pcg_iters;
  if (pcg_status) *pcg_status = h.pcg_status;
  if (rel_residual) *rel_residual = h.pcg_rel;
  if (h.bar_err || h.pcg_status == PCG_TIMEOUT)
    return set_last_error(ANDO_ERR_TIMEOUT, "ando_pcg_solve_noalloc: grid barrier timed out (overlapping call on this device?)");
  return ANDO_OK;
}

}  // namespace

int32_t ando_pcg_solve_noalloc(int32_t device, void* stream, int32_t num_rows, const int32_t* rowptr, const int32_t* cols,
                               const float* vals, const float* rhs, float* x, float* work, int64_t work_floats, double tol,
                               int32_t max_iters, int32_t* iterations, int32_t* pcg_status, double* rel_residual) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1) {
    cudaGetLastError();
    return set_last_error(ANDO_ERR_NO_DEVICE, "ando_pcg_solve_noalloc: no CUDA device");
  }
  if (device < 0 || device >= count || device >= kMaxDevices)
    return set_last_error(ANDO_ERR_INVALID, "ando_pcg_solve_noalloc: device index out of range");
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != device && cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return set_last_error(ANDO_ERR_CUDA, "ando_pcg_solve_noalloc: cudaSetDevice failed");
  }
  int rc = solve(device, static_cast<cudaStream_t>(stream), num_rows, rowptr, cols, vals, rhs, x, work, work_floats, tol,
                 max_iters, iterations, pcg_status, rel_residual);
  if (prev != device) cudaSetDevice(prev);
  return rc;
}
