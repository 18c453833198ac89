// corrected.cu -- kernels of the CORRECTED step semantics.
//
// The CORRECTED step keeps the reference's algorithm (beta accumulation,
// Newton with a block-Jacobi PCG inner solve, cubic barriers with
// elasticity-inclusive dynamic stiffness) and fixes what the reference gets
// wrong: elasticity is evaluated on the current positions, pins attract
// (springs of the implicit solve, in k_gradient), contact and wall stiffness
// take the current gap, self contact comes from a working broad phase with
// vertex-triangle and edge-edge barriers refreshed every Newton iteration, and
// the line search bounds the step by a conservative time of impact (FP64)
// instead of 10 temporal samples.
#include <cfloat>

#include "kernels.cuh"
#include "narrow.cuh"

namespace ando {

namespace {

constexpr int TPB = 256;
inline int nblk(long long n) { return int((n + TPB - 1) / TPB); }

__device__ inline d3 bary(d3 p, d3 a, d3 b, d3 c) {
  d3 v0 = b - a, v1 = c - a, v2 = p - a;
  double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
  double den = d00 * d11 - d01 * d01, v = 0, w = 0;
  if (fabs(den) > DBL_EPSILON) { v = (d11 * d20 - d01 * d21) / den; w = (d00 * d21 - d01 * d20) / den; }
  v = fmin(fmax(v, 0.0), 1.0); w = fmin(fmax(w, 0.0), 1.0);
  if (v + w > 1.0) { double sm = v + w; if (sm > DBL_EPSILON) { v /= sm; w /= sm; } }
  return mk(1.0 - v - w, v, w);
}

// Extent of one step's motion, for its sub-step count: the largest pin move
// |target - x| and the largest free motion dt |v| (IEEE bits of non-negative
// doubles, max-reduced as integers).
__global__ void k_drive_extent(const int* pin_vertex, const double* pin_target, int num_pins, const double* x, const double* v, int V,
                               double dt, unsigned long long* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.0;
  if (k < num_pins) {
    int i = pin_vertex[k];
    double a = pin_target[3 * k] - x[3 * i], b = pin_target[3 * k + 1] - x[3 * i + 1], c = pin_target[3 * k + 2] - x[3 * i + 2];
    m = sqrt(a * a + b * b + c * c);
  }
  if (k < V) m = fmax(m, dt * sqrt(v[3 * k] * v[3 * k] + v[3 * k + 1] * v[3 * k + 1] + v[3 * k + 2] * v[3 * k + 2]));
  for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
// Sub-step pin targets: start_k = x[pin vertex] once, then target = start + f (final - start).
__global__ void k_pin_gather(const int* pin_vertex, int num_pins, const double* x, double* start) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= num_pins) return;
  int v = pin_vertex[k];
  for (int q = 0; q < 3; ++q) start[3 * k + q] = x[3 * v + q];
}
__global__ void k_pin_interp(int num_pins, const double* start, const double* fin, double f, double* target) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * num_pins) return;
  target[k] = start[k] + (fin[k] - start[k]) * f;
}

// Candidate pairs -> contacts at the current positions. Every candidate gets a
// slot; the ones outside the activation distance are marked inactive
// (type < 0) and contribute nothing.
__global__ void k_pairs_to_contacts(const int2* vt, int nvt, const int2* ee, int nee, const int* tris, const int* edges,
                                    const double* x, double gap_max, ContactDev* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nvt + nee) return;
  ContactDev C;
  C.rigid = -1; C.count = 4; C.kbar = C.dV = C.d2V = 0.0; C.in_dom = 0;
  C.nn[0] = C.nn[1] = C.nn[2] = 0.0;
  if (k < nvt) {
    int v = vt[k].x, t = vt[k].y;
    C.type = 0; C.idx[0] = v; C.idx[1] = tris[3 * t]; C.idx[2] = tris[3 * t + 1]; C.idx[3] = tris[3 * t + 2];
    d3 p = ld3(x, v), a = ld3(x, C.idx[1]), b = ld3(x, C.idx[2]), c = ld3(x, C.idx[3]);
    d3 n, wq;
    double d = pt_dist(p, a, b, c, n, wq);
    d3 bc = bary(wq, a, b, c);
    C.gap = d; C.n[0] = n.x; C.n[1] = n.y; C.n[2] = n.z;
    C.wp[0] = p.x; C.wp[1] = p.y; C.wp[2] = p.z; C.wq[0] = wq.x; C.wq[1] = wq.y; C.wq[2] = wq.z;
    C.bary[0] = bc.x; C.bary[1] = bc.y; C.bary[2] = bc.z;
    C.w[0] = 1.0; C.w[1] = -bc.x; C.w[2] = -bc.y; C.w[3] = -bc.z;
  } else {
    int e1 = ee[k - nvt].x, e2 = ee[k - nvt].y;
    C.type = 1; C.idx[0] = edges[2 * e1]; C.idx[1] = edges[2 * e1 + 1]; C.idx[2] = edges[2 * e2]; C.idx[3] = edges[2 * e2 + 1];
    double s, t; d3 wp, wq;
    double d = ee_dist(ld3(x, C.idx[0]), ld3(x, C.idx[1]), ld3(x, C.idx[2]), ld3(x, C.idx[3]), s, t, wp, wq);
    d3 n = d > 1e-10 ? (wp - wq) / d : mk(0, 0, 1);
    C.gap = d; C.n[0] = n.x; C.n[1] = n.y; C.n[2] = n.z;
    C.wp[0] = wp.x; C.wp[1] = wp.y; C.wp[2] = wp.z; C.wq[0] = wq.x; C.wq[1] = wq.y; C.wq[2] = wq.z;
    C.bary[0] = s; C.bary[1] = t; C.bary[2] = 0.0;
    C.w[0] = 1.0 - s; C.w[1] = s; C.w[2] = -(1.0 - t); C.w[3] = -t;
  }
  if (!(C.gap < gap_max)) C.type = -1 - C.type;  // outside the activation distance: inactive
  out[k] = C;
}

// ext = 1.25 d, clipped vertex by vertex to length lmax (no vertex moves
// more than lmax in one Newton iteration; a single runaway entry of d no
// longer scales the whole step down); x1 = x + ext.
__global__ void k_swept_end(int V, const double* x, const float* d, const unsigned char* fixed, double ext_scale, double lmax,
                            double* x1, double* ext) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3ll * V) return;
  long long v = i / 3;
  double a = ext_scale * double(d[3 * v]), b = ext_scale * double(d[3 * v + 1]), c = ext_scale * double(d[3 * v + 2]);
  double len = sqrt(a * a + b * b + c * c);
  double cap = len > lmax ? lmax / len : 1.0;
  double e = fixed && fixed[v] ? 0.0 : cap * (ext_scale * double(d[i]));
  ext[i] = e;
  x1[i] = x[i] + e;
}

// Exact linear time of impact of each vertex against every active wall.
__global__ void k_toi_walls(int V, const double* x, const double* ext, const WallDev* walls, int nw, unsigned long long* toi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double t = 1.0;
  if (i < V) {
    d3 xi = ld3(x, i), e = ld3(ext, i);
    for (int w = 0; w < nw; ++w) {
      if (!walls[w].active) continue;
      d3 n = normalized(mk(walls[w].n[0], walls[w].n[1], walls[w].n[2]));
      double dn = dot(n, e);
      if (!(dn < 0.0)) continue;
      double gap = dot(n, xi) - walls[w].offset;
      t = fmin(t, fmax(gap, 0.0) / (-dn));
    }
  }
  t = warp_min(t);
  if ((threadIdx.x & 31) == 0 && t < 1.0) atomic_min_pos(toi, t);
}

// Vertices against static rigid triangles (the bodies do not move during the step).
__global__ void k_toi_rigid(int V, const double* x, const double* ext, const RigidDev* bodies, int nb, unsigned long long* toi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double t = 1.0;
  if (i < V) {
    d3 p = ld3(x, i), e = ld3(ext, i);
    double l = nrm(e);
    if (l > 0.0) {
      for (int b = 0; b < nb; ++b) {
        const RigidDev& B = bodies[b];
        for (int tr = 0; tr < B.nt; ++tr) {
          d3 a = ld3(B.world, B.tris[3 * tr]), bb = ld3(B.world, B.tris[3 * tr + 1]), c = ld3(B.world, B.tris[3 * tr + 2]);
          bool overlap = true;
          for (int k = 0; k < 3; ++k) {
            double lo = fmin(comp(p, k), comp(p + e, k)) - 1e-4, hi = fmax(comp(p, k), comp(p + e, k)) + 1e-4;
            double tl = fmin(fmin(comp(a, k), comp(bb, k)), comp(c, k)), th = fmax(fmax(comp(a, k), comp(bb, k)), comp(c, k));
            if (!(lo <= th && hi >= tl)) overlap = false;
          }
          if (!overlap) continue;
          t = fmin(t, advance([&](double s) { d3 n, wq; return pt_dist(p + e * s, a, bb, c, n, wq); }, l, 0.0, 0.0));
        }
      }
    }
  }
  t = warp_min(t);
  if ((threadIdx.x & 31) == 0 && t < 1.0) atomic_min_pos(toi, t);
}

// x += alpha d for free vertices, alpha = the time of impact bound (<= 1).
// x += toi * ext / 1.25 (the clipped Newton direction times the time of impact).
__global__ void k_update_toi(int V, double* x, const double* ext, double ext_scale, const unsigned char* fixed, Ctrl* ctrl,
                             const unsigned long long* toi) {
  if (ctrl->converged || ctrl->toi_overflow) return;  // overflow: incomplete time of impact, the caller redoes the pass
  double a = fmin(1.0, __longlong_as_double((long long)*toi));
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ctrl->alpha = a;
  if (a < 1e-8 || i >= 3ll * V || (fixed && fixed[i / 3])) return;
  x[i] += a * (ext[i] / ext_scale);
}

__global__ void k_toi_reset(unsigned long long* toi) { *toi = (unsigned long long)__double_as_longlong(1.0); }

}  // namespace

void launch_drive_extent(const int* pin_vertex, const double* pin_target, int num_pins, const double* x, const double* v, int V, double dt,
                         unsigned long long* out, cudaStream_t s) {
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), s);
  int n = num_pins > V ? num_pins : V;
  if (n) k_drive_extent<<<nblk(n), TPB, 0, s>>>(pin_vertex, pin_target, num_pins, x, v, V, dt, out);
}
void launch_pin_gather(const int* pin_vertex, int num_pins, const double* x, double* start, cudaStream_t s) {
  if (num_pins) k_pin_gather<<<nblk(num_pins), TPB, 0, s>>>(pin_vertex, num_pins, x, start);
}
void launch_pin_interp(int num_pins, const double* start, const double* fin, double f, double* target, cudaStream_t s) {
  if (num_pins) k_pin_interp<<<nblk(3ll * num_pins), TPB, 0, s>>>(num_pins, start, fin, f, target);
}
void launch_pairs_to_contacts(const int2* vt, int nvt, const int2* ee, int nee, const int* tris, const int* edges, const double* x,
                              double gap_max, ContactDev* out, cudaStream_t s) {
  if (nvt + nee) k_pairs_to_contacts<<<nblk(nvt + nee), TPB, 0, s>>>(vt, nvt, ee, nee, tris, edges, x, gap_max, out);
}
void launch_swept_end(int V, const double* x, const float* d, const unsigned char* fixed, double scale, double lmax,
                      double* x1, double* ext, cudaStream_t s) {
  if (V) k_swept_end<<<nblk(3ll * V), TPB, 0, s>>>(V, x, d, fixed, scale, lmax, x1, ext);
}
void launch_toi_reset(unsigned long long* toi, cudaStream_t s) { k_toi_reset<<<1, 1, 0, s>>>(toi); }
void launch_toi_walls(int V, const double* x, const double* ext, const WallDev* walls, int nw, unsigned long long* toi, cudaStream_t s) {
  if (V && nw) k_toi_walls<<<nblk(V), TPB, 0, s>>>(V, x, ext, walls, nw, toi);
}
void launch_toi_rigid(int V, const double* x, const double* ext, const RigidDev* bodies, int nb, unsigned long long* toi, cudaStream_t s) {
  if (V && nb) k_toi_rigid<<<nblk(V), TPB, 0, s>>>(V, x, ext, bodies, nb, toi);
}
void launch_update_toi(int V, double* x, const double* ext, double scale, const unsigned char* fixed, Ctrl* ctrl,
                       const unsigned long long* toi, cudaStream_t s) {
  k_update_toi<<<nblk(V > 0 ? 3ll * V : 1), TPB, 0, s>>>(V, x, ext, scale, fixed, ctrl, toi);
}

}  // namespace ando
