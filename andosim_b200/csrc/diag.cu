// diag.cu -- device-side diagnostics: CollisionValidator metrics over the
// context's contact list and EnergyTracker moments of its velocities.
//
// Each is a grid of per-block partials (grid-stride loops, a fixed tree
// reduction in shared memory) followed by one block that folds the partials
// in block order, so the sums are the same on every run.
#include <cfloat>

#include "diag.cuh"

namespace ando {

namespace {

constexpr int DTPB = 256;

inline int diag_blocks(long long n) {
  long long b = (n + DTPB - 1) / DTPB;
  return int(b < 1 ? 1 : (b > DIAG_MAX_BLOCKS ? DIAG_MAX_BLOCKS : b));
}

__device__ inline MetricSums metric_zero() {
  MetricSums m;
  m.min_gap = DBL_MAX; m.max_gap = -DBL_MAX; m.sum_gap = 0.0; m.max_pen = 0.0; m.sum_pen = 0.0; m.max_rv = 0.0; m.sum_rv = 0.0;
  m.n = m.n_pt = m.n_ee = m.n_wall = m.n_pen = m.n_major = m.n_tunnel = m.n_ccd = m.n_rv = 0;
  return m;
}

__device__ inline void metric_fold(MetricSums& a, const MetricSums& b) {
  a.min_gap = fmin(a.min_gap, b.min_gap); a.max_gap = fmax(a.max_gap, b.max_gap); a.sum_gap += b.sum_gap;
  a.max_pen = fmax(a.max_pen, b.max_pen); a.sum_pen += b.sum_pen; a.max_rv = fmax(a.max_rv, b.max_rv); a.sum_rv += b.sum_rv;
  a.n += b.n; a.n_pt += b.n_pt; a.n_ee += b.n_ee; a.n_wall += b.n_wall; a.n_pen += b.n_pen; a.n_major += b.n_major;
  a.n_tunnel += b.n_tunnel; a.n_ccd += b.n_ccd; a.n_rv += b.n_rv;
}

__device__ inline MomentSums moment_zero() {
  MomentSums m;
  m.ke = 0.0; m.vmax2 = 0.0;
  for (int k = 0; k < 3; ++k) { m.p[k] = 0.0; m.L[k] = 0.0; }
  return m;
}

__device__ inline void moment_fold(MomentSums& a, const MomentSums& b) {
  a.ke += b.ke; a.vmax2 = fmax(a.vmax2, b.vmax2);
  for (int k = 0; k < 3; ++k) { a.p[k] += b.p[k]; a.L[k] += b.L[k]; }
}

// Fixed-order tree reduction of one value per thread; thread 0 returns the total.
template <class T, class F>
__device__ inline T block_fold(T mine, T* sh, F fold) {
  sh[threadIdx.x] = mine;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) fold(sh[threadIdx.x], sh[threadIdx.x + w]);
    __syncthreads();
  }
  return sh[0];
}

// One contact's share of the metrics: gap statistics in single precision as
// the reference's Real (collision_validator.cpp:36-76), the CCD estimate
// (:92-100) and the relative normal velocity (:181-221).
__global__ void k_contact_metrics(const ContactDev* c, int n, const double* v, double gap_max, int ccd, MetricSums* parts) {
  __shared__ MetricSums sh[DTPB];
  MetricSums m = metric_zero();
  const float gmax = float(gap_max);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const ContactDev& C = c[i];
    const float gf = float(C.gap);
    const double g = gf;
    m.n++;
    if (C.type == 0) m.n_pt++; else if (C.type == 1) m.n_ee++; else if (C.type == 2) m.n_wall++;
    m.min_gap = fmin(m.min_gap, g); m.max_gap = fmax(m.max_gap, g); m.sum_gap += g;
    if (gf < 0.0f) {
      const float pen = -gf;
      m.n_pen++;
      m.max_pen = fmax(m.max_pen, double(pen)); m.sum_pen += double(pen);
      if (double(pen) > 0.001) m.n_major++;
      if (double(pen) > 0.1 * double(gmax)) m.n_tunnel++;
    }
    if (ccd && double(gf) < double(gmax) * 0.5) m.n_ccd++;
    if (C.type <= 2) {
      const d3 nn = mk(C.n[0], C.n[1], C.n[2]);
      d3 rel;
      if (C.type == 0) rel = ld3(v, C.idx[0]) - (ld3(v, C.idx[1]) + ld3(v, C.idx[2]) + ld3(v, C.idx[3])) * (1.0 / 3.0);
      else if (C.type == 1) rel = (ld3(v, C.idx[0]) + ld3(v, C.idx[1])) * 0.5 - (ld3(v, C.idx[2]) + ld3(v, C.idx[3])) * 0.5;
      else rel = ld3(v, C.idx[0]);
      const double rv = double(float(fabs(dot(rel, nn))));
      m.n_rv++; m.max_rv = fmax(m.max_rv, rv); m.sum_rv += rv;
    }
  }
  MetricSums t = block_fold(m, sh, metric_fold);
  if (threadIdx.x == 0) parts[blockIdx.x] = t;
}

__global__ void k_contact_metrics_final(const MetricSums* parts, int nparts, MetricSums* out) {
  __shared__ MetricSums sh[DTPB];
  MetricSums m = metric_zero();
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) metric_fold(m, parts[b]);
  MetricSums t = block_fold(m, sh, metric_fold);
  if (threadIdx.x == 0) *out = t;
}

// EnergyTracker::compute_kinetic_energy / linear / angular momentum / max
// velocity (energy_tracker.cpp:7-42) in one pass over the vertices.
__global__ void k_state_moments(int V, const double* x, const double* v, const double* mass, MomentSums* parts) {
  __shared__ MomentSums sh[DTPB];
  MomentSums m = moment_zero();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < V; i += gridDim.x * blockDim.x) {
    const d3 vi = ld3(v, i), xi = ld3(x, i);
    const double mi = mass[i], v2 = sqn(vi);
    const d3 pi = vi * mi, Li = cross(xi, pi);
    m.ke += 0.5 * mi * v2;
    m.vmax2 = fmax(m.vmax2, v2);
    m.p[0] += pi.x; m.p[1] += pi.y; m.p[2] += pi.z;
    m.L[0] += Li.x; m.L[1] += Li.y; m.L[2] += Li.z;
  }
  MomentSums t = block_fold(m, sh, moment_fold);
  if (threadIdx.x == 0) parts[blockIdx.x] = t;
}

__global__ void k_state_moments_final(const MomentSums* parts, int nparts, MomentSums* out) {
  __shared__ MomentSums sh[DTPB];
  MomentSums m = moment_zero();
  for (int b = threadIdx.x; b < nparts; b += blockDim.x) moment_fold(m, parts[b]);
  MomentSums t = block_fold(m, sh, moment_fold);
  if (threadIdx.x == 0) *out = t;
}

}  // namespace

void launch_contact_metrics(const ContactDev* contacts, int n, const double* v, double gap_max, int ccd, MetricSums* parts,
                            MetricSums* out, cudaStream_t s) {
  const int nb = diag_blocks(n);
  k_contact_metrics<<<nb, DTPB, 0, s>>>(contacts, n, v, gap_max, ccd, parts);
  k_contact_metrics_final<<<1, DTPB, 0, s>>>(parts, nb, out);
}

void launch_state_moments(int V, const double* x, const double* v, const double* mass, MomentSums* parts, MomentSums* out,
                          cudaStream_t s) {
  const int nb = diag_blocks(V);
  k_state_moments<<<nb, DTPB, 0, s>>>(V, x, v, mass, parts);
  k_state_moments_final<<<1, DTPB, 0, s>>>(parts, nb, out);
}

}  // namespace ando
