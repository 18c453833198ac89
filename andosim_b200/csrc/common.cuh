// common.cuh -- shared device helpers and data layout of the B200 step.
//
// Data layout in HBM (one context = one scene):
//   positions / velocities / targets        : double[3V]   (AoS xyz per vertex)
//   Newton gradient                         : double[3V]
//   PCG vectors (b, x, r, z, p ping-pong, Ap): float[3V]
//   BSR Hessian values                      : float[9*nnzb] (row-major 3x3 blocks)
//   BSR pattern                             : rowptr int[V+1], cols int[nnzb], slot_row int[nnzb]
//   block-Jacobi inverse                    : float[9V]
// The BSR pattern is static (self + mesh-edge blocks); contact blocks between
// non-adjacent vertices live in a per-step "extra" segment sorted by row.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ando {

// ----------------------------------------------------------------- vectors
struct d3 { double x, y, z; };
__host__ __device__ inline d3 mk(double a, double b, double c) { return d3{a, b, c}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator-(d3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline d3 operator/(d3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__host__ __device__ inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline double sqn(d3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__host__ __device__ inline double nrm(d3 a) { return sqrt(sqn(a)); }
__host__ __device__ inline d3 cross(d3 a, d3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__host__ __device__ inline double comp(d3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__host__ __device__ inline d3 normalized(d3 a) { double n2 = sqn(a); return n2 > 0.0 ? a / sqrt(n2) : a; }
__device__ inline d3 ld3(const double* p, int i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ inline void st3(double* p, int i, d3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

// --------------------------------------------------- cubic barrier (barrier.cpp:29-65)
__host__ __device__ inline double bar_energy(double g, double gm, double k) {
  if (gm <= 0.0 || g >= gm) return 0.0;
  double d = gm - g; if (d <= 0.0) return 0.0;
  return 0.5 * k * (1.0 / gm) * d * d * d;
}
__host__ __device__ inline double bar_grad(double g, double gm, double k) {
  if (gm <= 0.0 || g >= gm) return 0.0;
  double d = gm - g; return -1.5 * k * (1.0 / gm) * d * d;
}
__host__ __device__ inline double bar_hess(double g, double gm, double k) {
  if (gm <= 0.0 || g >= gm) return 0.0;
  double d = gm - g; return 3.0 * k * (1.0 / gm) * d;
}
__host__ __device__ inline bool in_domain(double g, double gm) { return gm > 0.0 && g <= gm; }
__host__ __device__ inline d3 normalize_or_default(d3 n, double eps) { return sqn(n) > eps * eps ? normalized(n) : mk(0.0, 1.0, 0.0); }

// CORRECTED pin stiffness: kappa = PIN_SCALE (m / dt^2 + a) with a the
// vertex's elastic diagonal coefficient; a pinned vertex then follows its
// target within about 1 % of the elastic load on it.
constexpr double PIN_SCALE = 100.0;

// -------------------------------------------------------------- parameters
struct WallDev { double n[3]; double offset, gap; int active; };

struct StepParams {
  double dt, dt2inv, contact_gap_max, wall_gap, normal_eps, barrier_tol, min_gap;
  double friction_mu, friction_eps, friction_thresh;
  int enable_friction, enable_strain, semantics;
  double strain_tau, strain_eps, svd_eps;  // already converted by to_fraction
  int num_walls;
  int first_wall;                          // index of the first active wall, -1 if none
};

// --------------------------------------------------------------- contacts
struct ContactDev {
  int type, idx[4], rigid, count;
  double gap, n[3], wp[3], wq[3], bary[3], w[4];
  // per-step constants (frozen gap, frozen normal)
  double kbar, dV, d2V, nn[3];
  int in_dom;
};

// Contact contribution entry (contact c, local i, local j), sorted by row vertex.
struct ContactEntry { int contact, li, lj, col; };

// --------------------------------------------------------- mesh on device
struct MeshDev {
  int V, T, nnzb;
  double mu, thickness, density;   // material: mu = E / (2 (1 + nu))
  const int* tris;          // 3T
  const double* rest_area;  // T
  const double* dm_inv;     // 4T (a b c d row-major)
  const double* mass;       // V
  const int* rowptr;        // V+1
  const int* cols;          // nnzb
  const int* slot_row;      // nnzb
  const int* diag_slot;     // V
  const int* face_slot;     // 9T  slot of block (a,b) of face f at f*9+a*3+b
  const int* slot_cptr;     // nnzb+1
  const int* slot_contrib;  // 9T   entries f*9+a*3+b, sorted by face within a slot
  const int* vf_ptr;        // V+1
  const int* vf;            // 3T   entries f*3+a, sorted by face within a vertex
  const double* el_a;       // nnzb elastic in-plane coefficient of the diag(a,a,b) block
  const double* el_b;       // nnzb elastic third-axis coefficient
  const double* g_elastic;  // 3V  elastic gradient on the mesh vertices (constant)
  // nnzb coefficient q of the quadratic bending Hessian q I3 per slot
  // (CORRECTED semantics, bending_stiffness > 0; null without bending)
  const double* bend_q;
  // 13 per face (R0, R1, n, a_t, W00, W01, W11) of the projected exact membrane
  // Hessian at the current positions (CORRECTED, membrane_hessian projected;
  // null otherwise): the assembly subtracts its correction of the constant
  // fixed-rotation blocks
  const double* mface;
};
constexpr int MFACE = 13;

// Strain-limit data of one face and one singular value.
struct StrainSV { double J[9]; double dV, d2V; };

// Lower-triangular 3x3 (Cholesky factor or its inverse), row-major packed.
struct Tri3 { double l00, l10, l11, l20, l21, l22; };

// -------------------------------------------------------- device control
struct Ctrl {
  unsigned long long gnorm_bits;  // max |g| as IEEE bits (non-negative doubles order as integers)
  unsigned int ls_mask;           // AND over all feasibility masks, bit j = level j feasible
  int converged;                  // gradient-norm test passed this Newton iteration
  int pcg_iters, pcg_converged, pcg_status;
  double pcg_rel;
  double alpha;
  int strain_active;
  unsigned int bar_count, bar_gen; int bar_err;
  int tc_err;                     // a tensor-core GEMM's bounded wait gave up (sticky)
  int toi_overflow;               // > 0: a time-of-impact candidate list needed this many slots; the move was not applied
  int learned_iters;              // iterations of this Newton iteration's learned solve
  int fallback_ran;               // block-Jacobi redid this Newton iteration's learned solve
  int pad_;
  unsigned long long bar_arrivals;  // grid_sync_ar: arrivals since the launcher zeroed it
};

// PCG_PRECOND: the learned preconditioner lost positive definiteness
// (r^T z <= 0); PCG_STALL: its residual stopped improving. Both hand the
// solve back to block-Jacobi.
enum PcgStatus { PCG_OK = 0, PCG_MAXIT = 1, PCG_NOT_SPD = 2, PCG_TIMEOUT = 3, PCG_SKIPPED = 4, PCG_PRECOND = 5, PCG_STALL = 6 };

// Device-side control of one step (integrator.cpp:98-121 and 152-236) when the
// whole frame runs as one CUDA graph: the beta loop, the error-reduction pass
// and the Newton loop are decided on the device between graph iterations.
struct StepCtl {
  double beta, ret, last_alpha;
  int bi, phase, newton_it, max_it;   // phase 0: beta loop, 1: error-reduction pass, 2: done
  int newton_iters, pcg_iters, pcg_max, pcg_not_converged, line_search_fail, strain_active, error;
  int iterations_run, inner_steps;    // Newton bodies and inner steps executed (launch accounting)
};

// Bounded grid barrier for cooperative launches. All CTAs of the grid must be
// co-resident (cudaLaunchCooperativeKernel guarantees it). A CTA that waits
// more than `limit` polls sets *err and every CTA leaves; callers check the
// return value and bail out uniformly.
__device__ inline bool grid_sync(unsigned int* count, unsigned int* gen, int* err, unsigned int nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = gen;
    volatile int* verr = err;
    unsigned int g = *vgen;
    __threadfence();
    unsigned int arrived = atomicAdd(count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      long long polls = 0;
      const long long limit = 1ll << 24;  // ~seconds with backoff
      while (*vgen == g) {
        if (*verr) break;
        if (++polls > limit) { atomicExch(err, 1); break; }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  volatile int* verr = err;
  return *verr == 0;
}

// Bounded grid barrier with acquire/release atomics: every CTA adds one
// arrival to a 64-bit counter that the launcher zeroed (release: the CTA's
// writes, ordered before the arrival by __syncthreads, are published) and
// polls with acquire loads until all nblocks CTAs have arrived `epoch` times.
// About half the cost of grid_sync's full fences. The polling thread hands
// its verdict to the CTA through shared memory, so the other threads leave
// the barrier without another L2 round trip. A CTA that passed a barrier
// while another CTA was giving up on it meets the error flag in the poll of
// the next barrier (every wait stays bounded), and the host reads the flag
// after the launch.
__device__ inline bool grid_sync_ar(unsigned long long* arrivals, unsigned int nblocks, unsigned int& epoch, int* err) {
  __shared__ int passed;
  __syncthreads();  // also orders the previous call's reads of `passed` before this call's write
  ++epoch;
  if (threadIdx.x == 0) {
    const unsigned long long target = (unsigned long long)epoch * nblocks;
    asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(arrivals) : "memory");
    long long polls = 0;
    int ok = 1;
    while (true) {
      unsigned long long v;
      asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(arrivals) : "memory");
      if (v >= target) break;
      if (*(volatile int*)err) { ok = 0; break; }
      if (++polls > (1ll << 24)) { atomicExch(err, 1); ok = 0; break; }
      if (polls > 1024) __nanosleep(32);
    }
    passed = ok;
  }
  __syncthreads();
  return passed != 0;
}

}  // namespace ando
