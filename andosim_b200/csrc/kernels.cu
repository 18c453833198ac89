// kernels.cu -- per-element, per-vertex and per-contact kernels of the implicit step.
//
// Semantics follow the reference step (src/core/integrator.cpp and the term
// files it calls); each kernel cites the reference function it replaces.
// All reductions are deterministic: scatter targets are gathered through
// precomputed sorted lists, never accumulated with floating-point atomics.
#include <cfloat>

#include <atomic>

#include "kernels.cuh"

namespace ando {

namespace {

constexpr int TPB = 256;
inline int nblk(long long n, int tpb = TPB) { return int((n + tpb - 1) / tpb); }

__device__ inline int find_slot(const MeshDev& m, int row, int col) {
  int lo = m.rowptr[row], hi = m.rowptr[row + 1];
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    int c = m.cols[mid];
    if (c < col) lo = mid + 1; else hi = mid;
  }
  return (lo < m.rowptr[row + 1] && m.cols[lo] == col) ? lo : -1;
}

// Face Hessian coefficient c of block (a,b): the block is c*diag(1,1,0)
// (elasticity.cpp:135-181), K = k * Dm_inv^T Dm_inv.
__device__ inline double face_block_coeff(double K00, double K01, double K11, int a, int b) {
  if (a == b) return a == 0 ? (K00 + K11 + 2.0 * K01) : (a == 1 ? K00 : K11);
  int lo = a < b ? a : b, hi = a < b ? b : a;
  if (lo == 0 && hi == 1) return -K00;
  if (lo == 0 && hi == 2) return -K11;
  return -K01;
}

__device__ inline void face_K(const MeshDev& m, int f, double mu, double thickness, double& K00, double& K01, double& K11) {
  double k = m.rest_area[f] * thickness * mu;
  double a = m.dm_inv[4 * f], b = m.dm_inv[4 * f + 1], c = m.dm_inv[4 * f + 2], d = m.dm_inv[4 * f + 3];
  // Dm_inv^T Dm_inv
  K00 = k * (a * a + c * c); K01 = k * (a * b + c * d); K11 = k * (b * b + d * d);
}

// --------------------------------------------------------------- setup kernels

// Constant elastic Hessian per BSR slot: sum over contributing faces (in face
// order) of the SPD-clamped face blocks (elasticity.cpp:63-91 with
// Stiffness::enforce_spd, stiffness.cpp:236-254). A block c*diag(1,1,0)
// clamps to diag(max(c,1e-8), max(c,1e-8), 1e-8) exactly. CORRECTED
// semantics uses the isotropic c*I instead.
__global__ void k_elastic_slots(MeshDev m, double mu, double thickness, int semantics, double* el_a, double* el_b) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m.nnzb) return;
  double A = 0.0, B = 0.0;
  for (int k = m.slot_cptr[s]; k < m.slot_cptr[s + 1]; ++k) {
    int e = m.slot_contrib[k];
    int f = e / 9, a = (e % 9) / 3, b = e % 3;
    if (semantics == 0) {
      double K00, K01, K11; face_K(m, f, mu, thickness, K00, K01, K11);
      double c = face_block_coeff(K00, K01, K11, a, b);
      A += fmax(c, 1e-8); B += 1e-8;
    } else {
      // Hessian of k |F - R|^2 for a fixed frame R: 2k (G G^T)_ab I3 with
      // G = [[-1,-1],[1,0],[0,1]] Dm_inv
      double k = m.rest_area[f] * thickness * mu;
      double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
      double G[3][2] = {{-(da + dc), -(db + dd)}, {da, db}, {dc, dd}};
      double c = 2.0 * k * (G[a][0] * G[b][0] + G[a][1] * G[b][1]);
      A += c; B += c;
    }
  }
  // CORRECTED: the constant Hessian of the quadratic bending energy joins the
  // elastic blocks (and with them the elasticity-inclusive stiffnesses)
  if (semantics != 0 && m.bend_q) { A += m.bend_q[s]; B += m.bend_q[s]; }
  el_a[s] = A; el_b[s] = B;
}

// Elastic gradient on the mesh vertices (elasticity.cpp:18-61), gathered per
// vertex over its incident faces in face order.
__global__ void k_elastic_gradient(MeshDev m, const double* X, double mu, double thickness, double* g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.V) return;
  d3 acc = mk(0, 0, 0);
  for (int k = m.vf_ptr[i]; k < m.vf_ptr[i + 1]; ++k) {
    int f = m.vf[k] / 3, a = m.vf[k] % 3;
    int v0 = m.tris[3 * f], v1 = m.tris[3 * f + 1], v2 = m.tris[3 * f + 2];
    d3 e1 = ld3(X, v1) - ld3(X, v0), e2 = ld3(X, v2) - ld3(X, v0);
    d3 n = normalized(cross(e1, e2)), t1 = normalized(e1), t2 = cross(n, t1);
    double Ds00 = dot(e1, t1), Ds01 = dot(e2, t1), Ds10 = dot(e1, t2), Ds11 = dot(e2, t2);
    double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
    double F00 = Ds00 * da + Ds01 * dc, F01 = Ds00 * db + Ds01 * dd, F10 = Ds10 * da + Ds11 * dc, F11 = Ds10 * db + Ds11 * dd;
    double kf = m.rest_area[f] * thickness * mu;
    double tk = 2.0 * kf;
    double P00 = tk * (F00 - 1.0), P01 = tk * F01, P10 = tk * F10, P11 = tk * (F11 - 1.0);
    // H = P * Dm_inv^T
    double H00 = P00 * da + P01 * db, H01 = P00 * dc + P01 * dd, H10 = P10 * da + P11 * db, H11 = P10 * dc + P11 * dd;
    d3 f1 = t1 * H00 + t2 * H10, f2 = t1 * H01 + t2 * H11;
    d3 contrib = a == 0 ? -(f1 + f2) : (a == 1 ? f1 : f2);
    acc = acc + contrib;
  }
  st3(g, i, acc);
}

// ------------------------------------------------------------------ per step
__global__ void k_predict(int V, const double* x, const double* v, double dt, double* x_old, double* x_hat) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * V) return;
  x_old[i] = x[i];
  x_hat[i] = x[i] + dt * v[i];
}

// State.apply_gravity (bindings.cpp:284-300)
__global__ void k_gravity(int V, double* x, double* v, double gx, double gy, double gz, double dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  double vx = v[3 * i] + gx * dt, vy = v[3 * i + 1] + gy * dt, vz = v[3 * i + 2] + gz * dt;
  v[3 * i] = vx; v[3 * i + 1] = vy; v[3 * i + 2] = vz;
  x[3 * i] += vx * dt; x[3 * i + 1] += vy * dt; x[3 * i + 2] += vz * dt;
}

// RigidBody::world_vertices (rigid_body.cpp:93-100)
__global__ void k_rigid_world(RigidDev* bodies, int nb) {
  int b = blockIdx.y;
  if (b >= nb) return;
  RigidDev& B = bodies[b];
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B.nv) return;
  d3 l = ld3(B.local, i);
  d3 w = mk(B.pos[0] + B.R[0] * l.x + B.R[1] * l.y + B.R[2] * l.z,
            B.pos[1] + B.R[3] * l.x + B.R[4] * l.y + B.R[5] * l.z,
            B.pos[2] + B.R[6] * l.x + B.R[7] * l.y + B.R[8] * l.z);
  st3(B.world, i, w);
}

// Collision::narrow_phase_point_triangle (collision.cpp:279-386)
__device__ inline void narrow_pt(d3 p, d3 a, d3 b, d3 c, double& dist, d3& normal, d3& wq) {
  d3 ab = b - a, ac = c - a, ap = p - a;
  double d1 = dot(ab, ap), d2 = dot(ac, ap);
  auto vert = [&](d3 q) { wq = q; d3 df = p - q; dist = nrm(df); normal = dist > 1e-10 ? df / dist : mk(0, 0, 1); };
  if (d1 <= 0.0 && d2 <= 0.0) { vert(a); return; }
  d3 bp = p - b; double d3_ = dot(ab, bp), d4 = dot(ac, bp);
  if (d3_ >= 0.0 && d4 <= d3_) { vert(b); return; }
  d3 cp = p - c; double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) { vert(c); return; }
  double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) { double v = d1 / (d1 - d3_); vert(a + ab * v); return; }
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) { double w = d2 / (d2 - d6); vert(a + ac * w); return; }
  double va = d3_ * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0) { double w = (d4 - d3_) / ((d4 - d3_) + (d5 - d6)); vert(b + (c - b) * w); return; }
  double den = 1.0 / (va + vb + vc);
  double v = vb * den, w = vc * den;
  wq = a + ab * v + ac * w;
  d3 df = p - wq; dist = nrm(df);
  d3 tn = cross(ab, ac); double ta = nrm(tn);
  if (ta > 1e-10) { tn = tn / ta; if (dot(tn, df) < 0.0) tn = -tn; normal = tn; }
  else normal = dist > 1e-10 ? df / dist : mk(0, 0, 1);
}

// Collision::narrow_phase_edge_edge (collision.cpp:389-452)
__device__ inline void narrow_ee(d3 p0, d3 p1, d3 q0, d3 q1, double& dist) {
  d3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  double s, t; const double eps = 1e-10;
  d3 wp, wq;
  auto cl = [](double v) { return fmin(fmax(v, 0.0), 1.0); };
  if (a <= eps && e <= eps) { wp = p0; wq = q0; }
  else {
    if (a <= eps) { s = 0; t = cl(f / e); }
    else {
      double c = dot(d1, r);
      if (e <= eps) { t = 0; s = cl(-c / a); }
      else {
        double b = dot(d1, d2), den = a * e - b * b;
        s = den != 0.0 ? cl((b * f - c * e) / den) : 0.0;
        t = (b * s + f) / e;
        if (t < 0.0) { t = 0; s = cl(-c / a); }
        else if (t > 1.0) { t = 1; s = cl((b - c) / a); }
      }
    }
    wp = p0 + d1 * s; wq = q0 + d2 * t;
  }
  dist = nrm(wp - wq);
}

// compute_triangle_barycentric (collision.cpp:11-43)
__device__ inline d3 barycentric(d3 p, d3 a, d3 b, d3 c) {
  d3 v0 = b - a, v1 = c - a, v2 = p - a;
  double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1), d20 = dot(v2, v0), d21 = dot(v2, v1);
  double den = d00 * d11 - d01 * d01, v = 0, w = 0;
  if (fabs(den) > DBL_EPSILON) { v = (d11 * d20 - d01 * d21) / den; w = (d00 * d21 - d01 * d20) / den; }
  v = fmin(fmax(v, 0.0), 1.0); w = fmin(fmax(w, 0.0), 1.0);
  if (v + w > 1.0) { double sm = v + w; if (sm > DBL_EPSILON) { v /= sm; w /= sm; } }
  return mk(1.0 - v - w, v, w);
}

// Literal broad phase (collision.cpp:65-105,198-244): the median-split BVH
// only ever holds a primitive at a node when the mesh has exactly one
// triangle (leaves of 2..4 carry none), so vertex-triangle candidates exist
// only then; edge-edge candidates never do (the one-edge root pairs with
// itself and is dropped by e1 < e2).
__device__ inline bool literal_pt_candidate(const MeshDev& m, const double* x, int v) {
  int a = m.tris[0], b = m.tris[1], c = m.tris[2];
  if (v == a || v == b || v == c) return false;
  d3 p = ld3(x, v), A = ld3(x, a), B = ld3(x, b), C = ld3(x, c);
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) { double pa = comp(A, k), pb = comp(B, k), pc = comp(C, k); lo[k] = fmin(fmin(pa, pb), pc); hi[k] = fmax(fmax(pa, pb), pc); }
  for (int k = 0; k < 3; ++k) { double pk = comp(p, k); if (!(pk - 1e-4 <= hi[k] && pk + 1e-4 >= lo[k])) return false; }
  return true;
}

// Count contacts per detection unit. Units: [0,V) vertex-vs-triangle-0 (literal
// PT, only when T == 1), then [V + b*V + v] vertex v vs rigid body b.
__global__ void k_detect_count(MeshDev m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, int* counts) {
  long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)m.V * (1 + nb);
  if (u >= total) return;
  int cnt = 0;
  if (u < m.V) {
    int v = int(u);
    if (literal_pt && literal_pt_candidate(m, x, v)) {
      double dist; d3 n, wq;
      narrow_pt(ld3(x, v), ld3(x, m.tris[0]), ld3(x, m.tris[1]), ld3(x, m.tris[2]), dist, n, wq);
      cnt = dist < thresh ? 1 : 0;
    }
  } else {
    int b = int((u - m.V) / m.V), v = int((u - m.V) % m.V);
    const RigidDev& B = bodies[b];
    d3 p = ld3(x, v);
    for (int t = 0; t < B.nt; ++t) {
      double dist; d3 n, wq;
      narrow_pt(p, ld3(B.world, B.tris[3 * t]), ld3(B.world, B.tris[3 * t + 1]), ld3(B.world, B.tris[3 * t + 2]), dist, n, wq);
      cnt += dist < thresh ? 1 : 0;
    }
  }
  counts[u] = cnt;
}

__global__ void k_detect_write(MeshDev m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, const int* offsets, ContactDev* out) {
  long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = (long long)m.V * (1 + nb);
  if (u >= total) return;
  int o = offsets[u];
  if (u < m.V) {
    int v = int(u);
    if (!(literal_pt && literal_pt_candidate(m, x, v))) return;
    d3 p = ld3(x, v), a = ld3(x, m.tris[0]), b = ld3(x, m.tris[1]), c = ld3(x, m.tris[2]);
    double dist; d3 n, wq;
    narrow_pt(p, a, b, c, dist, n, wq);
    if (!(dist < thresh)) return;
    ContactDev C;
    C.type = 0; C.idx[0] = v; C.idx[1] = m.tris[0]; C.idx[2] = m.tris[1]; C.idx[3] = m.tris[2]; C.rigid = -1; C.count = 4;
    C.gap = dist; C.n[0] = n.x; C.n[1] = n.y; C.n[2] = n.z;
    C.wp[0] = p.x; C.wp[1] = p.y; C.wp[2] = p.z; C.wq[0] = wq.x; C.wq[1] = wq.y; C.wq[2] = wq.z;
    d3 bc = barycentric(wq, a, b, c);
    C.bary[0] = bc.x; C.bary[1] = bc.y; C.bary[2] = bc.z;
    C.w[0] = 1.0; C.w[1] = -bc.x; C.w[2] = -bc.y; C.w[3] = -bc.z;
    out[o] = C;
  } else {
    int bi = int((u - m.V) / m.V), v = int((u - m.V) % m.V);
    const RigidDev& B = bodies[bi];
    d3 p = ld3(x, v);
    for (int t = 0; t < B.nt; ++t) {
      double dist; d3 n, wq;
      narrow_pt(p, ld3(B.world, B.tris[3 * t]), ld3(B.world, B.tris[3 * t + 1]), ld3(B.world, B.tris[3 * t + 2]), dist, n, wq);
      if (!(dist < thresh)) continue;
      ContactDev C;
      C.type = 3; C.idx[0] = v; C.idx[1] = B.tris[3 * t]; C.idx[2] = B.tris[3 * t + 1]; C.idx[3] = B.tris[3 * t + 2];
      C.rigid = bi; C.count = 1; C.gap = dist; C.n[0] = n.x; C.n[1] = n.y; C.n[2] = n.z;
      C.wp[0] = p.x; C.wp[1] = p.y; C.wp[2] = p.z; C.wq[0] = wq.x; C.wq[1] = wq.y; C.wq[2] = wq.z;
      C.bary[0] = C.bary[1] = C.bary[2] = 0.0;
      C.w[0] = 1.0; C.w[1] = C.w[2] = C.w[3] = 0.0;
      out[o++] = C;
    }
  }
}

// Stiffness::compute_contact_stiffness (stiffness.cpp:53-116) against the
// constant elastic Hessian: sum_i m_i w_i^2 / dt^2 + max(0, Wn^T H_el Wn), the
// submatrix taken over the contact's valid vertices (each vertex at its last
// list position, as extract_submatrix maps it).
// `dt` divides the inertial part sum(m w^2): the time step in REFERENCE
// semantics, the current gap in CORRECTED semantics.
__device__ inline double contact_kbar(const MeshDev& m, const ContactDev& C, double dt) {
  if (dt <= 0.0) return 0.0;
  d3 n = mk(C.n[0], C.n[1], C.n[2]);
  double nn = nrm(n);
  if (nn < 1e-12) return 0.0;
  n = n / nn;
  int cnt = C.count > 1 ? C.count : 1;
  int vv[4]; double ww[4]; int nvv = 0;
  for (int i = 0; i < cnt; ++i) {
    int id = C.idx[i];
    if (id < 0 || id >= m.V) continue;
    if (C.w[i] == 0.0) continue;
    vv[nvv] = id; ww[nvv] = C.w[i]; ++nvv;
  }
  if (nvv == 0) return 0.0;
  double inertial = 0.0;
  for (int i = 0; i < nvv; ++i) inertial += m.mass[vv[i]] * ww[i] * ww[i];
  inertial /= (dt * dt);
  double nxy = n.x * n.x + n.y * n.y, nz2 = n.z * n.z;
  double el = 0.0;
  for (int i = 0; i < nvv; ++i) {
    bool last_i = true; for (int q = i + 1; q < nvv; ++q) if (vv[q] == vv[i]) last_i = false;
    if (!last_i) continue;
    for (int j = 0; j < nvv; ++j) {
      bool last_j = true; for (int q = j + 1; q < nvv; ++q) if (vv[q] == vv[j]) last_j = false;
      if (!last_j) continue;
      int s = find_slot(m, vv[i], vv[j]);
      if (s < 0) continue;
      el += ww[i] * ww[j] * (m.el_a[s] * nxy + m.el_b[s] * nz2);
    }
  }
  if (el < 0.0) el = 0.0;
  return inertial + el;
}

// Per-contact constants of a step: k_bar, the normalised frozen normal and the
// barrier derivatives at the frozen gap (barrier.cpp:67-149 reads contact.gap
// and contact.normal from detection time).
__global__ void k_contact_prep(MeshDev m, ContactDev* cs, int nc, StepParams p) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  ContactDev& C = cs[c];
  // CORRECTED: the inertial part of the stiffness is sum(m w^2) / g^2 at the
  // current gap instead of / dt^2 (the form of the reference's pin and strain
  // stiffness), so the finite cubic barrier's force grows without bound as the
  // pair closes instead of saturating at 1.5 k g_max
  C.kbar = contact_kbar(m, C, p.semantics == 1 ? fmax(fmax(C.gap, p.min_gap), 1e-12) : p.dt);
  d3 nn = normalize_or_default(mk(C.n[0], C.n[1], C.n[2]), p.normal_eps);
  C.nn[0] = nn.x; C.nn[1] = nn.y; C.nn[2] = nn.z;
  bool barrier_type = (C.type == 0 || C.type == 3 || (p.semantics == 1 && C.type == 1));
  C.in_dom = barrier_type && in_domain(C.gap, p.contact_gap_max);
  C.dV = C.in_dom ? bar_grad(C.gap, p.contact_gap_max, C.kbar) : 0.0;
  C.d2V = C.in_dom ? bar_hess(C.gap, p.contact_gap_max, C.kbar) : 0.0;
}

// Entry slots: 16 per contact, (c, i, j) at c*16 + i*4 + j. Valid barrier
// entries and (c,0,0) friction entries get key = row vertex, others key = V.
// Entry kinds (ContactEntry.col < 0 encodes "friction only").
__global__ void k_contact_entries(const ContactDev* cs, int nc, int V, int friction, int* keys, ContactEntry* ents) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)nc * 16) return;
  int c = int(e / 16), i = int((e % 16) / 4), j = int(e % 4);
  const ContactDev& C = cs[c];
  int cnt = C.count > 1 ? C.count : 1;
  bool barrier = C.in_dom && C.d2V != 0.0 && i < cnt && j < cnt && C.w[i] != 0.0 && C.w[j] != 0.0 &&
                 C.idx[i] >= 0 && C.idx[j] >= 0 && C.idx[i] < V && C.idx[j] < V;
  // a barrier gradient entry is represented by the (i,i) entry even when d2V == 0 but dV != 0
  bool grad_only = !barrier && i == j && C.in_dom && C.dV != 0.0 && i < cnt && C.w[i] != 0.0 && C.idx[i] >= 0 && C.idx[i] < V;
  bool fric = friction && C.type >= 0 && i == 0 && j == 0 && C.idx[0] >= 0 && C.idx[0] < V;
  ContactEntry E; E.contact = c; E.li = i; E.lj = j;
  if (barrier || grad_only || fric) {
    keys[e] = C.idx[i];
    E.col = (barrier || grad_only) ? C.idx[j] : -1;
    E.li = i | (fric ? 8 : 0) | (grad_only ? 16 : 0);
  } else {
    keys[e] = V; E.col = -1;
  }
  ents[e] = E;
}

__global__ void k_vertex_ranges(const int* keys, int n, int V, int* begin, int* end) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  int lo = 0, hi = n;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (keys[mid] < v) lo = mid + 1; else hi = mid; }
  int b = lo; hi = n;
  while (lo < hi) { int mid = (lo + hi) >> 1; if (keys[mid] <= v) lo = mid + 1; else hi = mid; }
  begin[v] = b; end[v] = lo;
}

// Per-vertex constants of a step: elastic gradient (REFERENCE: on the rest
// mesh, so constant) + contact barrier gradient, and the contact Hessian
// blocks that land on the diagonal. Contact terms are summed in contact order.
__global__ void k_contact_vertex(MeshDev m, const ContactDev* cs, const ContactEntry* ents, const int* begin, const int* end,
                                 StepParams p, const double* g_base, double* g_const, double* diag_const) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= m.V) return;
  d3 g = ld3(g_base, v);
  double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = begin[v]; k < end[v]; ++k) {
    ContactEntry E = ents[k];
    if (E.col < 0) continue;  // friction only
    const ContactDev& C = cs[E.contact];
    int i = E.li & 3, j = E.lj;
    d3 n = mk(C.nn[0], C.nn[1], C.nn[2]);
    if (i == j && C.dV != 0.0 && C.w[i] != 0.0) g = g + n * (C.dV * C.w[i]);
    if (E.col == v && !(E.li & 16)) {
      d3 gi = n * C.w[i], gj = n * C.w[j];
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) {
          double val = C.d2V * (comp(gi, r) * comp(gj, q));
          if (fabs(val) < p.barrier_tol) continue;
          H[r * 3 + q] += val;
        }
    }
  }
  st3(g_const, v, g);
  for (int k = 0; k < 9; ++k) diag_const[9 * v + k] = H[k];
}

__global__ void k_extra_flags(const ContactEntry* ents, const int* keys, int n, int* flags) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  ContactEntry E = ents[k];
  flags[k] = (E.col >= 0 && E.col != keys[k] && !(E.li & 16)) ? 1 : 0;
}

// ---------------------------------------------------------- Newton iteration
__global__ void k_ctrl_reset(Ctrl* c) {
  c->gnorm_bits = 0ull; c->ls_mask = (1u << 20) - 1u; c->converged = 0;
  c->pcg_iters = 0; c->pcg_converged = 0; c->pcg_status = PCG_SKIPPED; c->pcg_rel = 0.0;
  c->alpha = 0.0; c->strain_active = 0; c->bar_count = 0; c->bar_err = 0;
  c->learned_iters = 0; c->fallback_ran = 0;
}

// Thin SVD of the 3x2 deformation gradient through the eigenpairs of F^T F
// (restates the JacobiSVD call of strain_limiting.cpp:28-50: sigma sorted
// descending, U = F V / sigma).
struct Svd32 { d3 U0, U1; double s0, s1; double V00, V01, V10, V11; bool ok; };
__device__ inline Svd32 svd32(d3 c0, d3 c1) {
  Svd32 r;
  double a = dot(c0, c0), b = dot(c0, c1), d = dot(c1, c1);
  double tr = a + d, df = a - d, disc = sqrt(df * df + 4.0 * b * b);
  double l0 = 0.5 * (tr + disc), l1 = fmax(0.5 * (tr - disc), 0.0);
  double v0x, v0y;
  if (b == 0.0) { if (a >= d) { v0x = 1; v0y = 0; } else { v0x = 0; v0y = 1; } }
  else { v0x = l0 - d; v0y = b; double nr = sqrt(v0x * v0x + v0y * v0y); v0x /= nr; v0y /= nr; }
  double v1x = -v0y, v1y = v0x;
  r.s0 = sqrt(l0); r.s1 = sqrt(l1);
  r.V00 = v0x; r.V10 = v0y; r.V01 = v1x; r.V11 = v1y;
  d3 u0 = c0 * v0x + c1 * v0y, u1 = c0 * v1x + c1 * v1y;
  if (r.s0 > 0.0) u0 = u0 / r.s0;
  if (r.s1 > 1e-300) u1 = u1 / r.s1;
  else {
    d3 t = fabs(u0.x) < 0.57 ? mk(1, 0, 0) : (fabs(u0.y) < 0.57 ? mk(0, 1, 0) : mk(0, 0, 1));
    u1 = normalized(cross(u0, t));
  }
  r.U0 = u0; r.U1 = u1;
  const double thr = 1e-6;
  if (r.s0 < thr || r.s1 < thr) { r.s0 = fmax(r.s0, thr); r.s1 = fmax(r.s1, thr); }
  r.ok = isfinite(r.s0) && isfinite(r.s1);
  return r;
}


// CORRECTED elasticity: the as-rigid-as-possible membrane energy
// k |F - R|^2 per face (F = [x1 - x0, x2 - x0] Dm^-1, R = U V^T from its thin
// SVD, k = area * thickness * mu). The reference's force formula
// (elasticity.cpp:18-61) drops the rotation of its edge-aligned frame and is
// not the gradient of its own energy away from rest; this one is exact, and
// the constant Hessian 2k (G G^T) (x) I3 of k_elastic_slots is its Hessian at
// fixed R. Gathered per vertex over its incident faces in face order.
__global__ void k_arap_gradient(MeshDev m, const double* X, double mu, double thickness, double* g) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.V) return;
  d3 acc = mk(0, 0, 0);
  for (int k = m.vf_ptr[i]; k < m.vf_ptr[i + 1]; ++k) {
    int f = m.vf[k] / 3, a = m.vf[k] % 3;
    int v0 = m.tris[3 * f], v1 = m.tris[3 * f + 1], v2 = m.tris[3 * f + 2];
    d3 e1 = ld3(X, v1) - ld3(X, v0), e2 = ld3(X, v2) - ld3(X, v0);
    double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
    d3 F0 = e1 * da + e2 * dc, F1 = e1 * db + e2 * dd;
    Svd32 s = svd32(F0, F1);
    d3 R0 = s.U0 * s.V00 + s.U1 * s.V01, R1 = s.U0 * s.V10 + s.U1 * s.V11;
    double tk = 2.0 * m.rest_area[f] * thickness * mu;
    d3 P0 = (F0 - R0) * tk, P1 = (F1 - R1) * tk;
    double G0 = a == 0 ? -(da + dc) : (a == 1 ? da : dc), G1 = a == 0 ? -(db + dd) : (a == 1 ? db : dd);
    acc = acc + P0 * G0 + P1 * G1;
  }
  // quadratic bending: row i of Q x, taken as sum_j q_ij (x_j - x_i) (the
  // rows of Q sum to zero), which keeps the cancellation of a nearly flat
  // sheet away from the absolute coordinates
  if (m.bend_q) {
    const d3 xi = ld3(X, i);
    for (int k = m.rowptr[i]; k < m.rowptr[i + 1]; ++k) {
      const double q = m.bend_q[k];
      if (q != 0.0) acc = acc + (ld3(X, m.cols[k]) - xi) * q;
    }
  }
  st3(g, i, acc);
}

// Per face: the data of the projected exact membrane Hessian at X (see
// membrane_correction): R = U V^T, n = U0 x U1, a_t = 2k min(1, 2 / (s0 + s1))
// and W = V diag(c0, c1) V^T with c_i = 2k min(1, 1 / s_i), from the thin SVD
// of F = [x1 - x0, x2 - x0] Dm^-1. The Hessian of k |F - R|^2 in F has the
// eigenvalues 2k (three symmetric in-plane modes), 2k (1 - 2 / (s0 + s1))
// (the twist) and 2k (1 - 1 / s_i) (the flips n v_i^T); clamping them at zero
// leaves 2k I minus a_t on the twist and c_i on the flips.
__global__ void k_membrane_face(MeshDev m, const double* X, double mu, double thickness, double* out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.T) return;
  const int v0 = m.tris[3 * f], v1 = m.tris[3 * f + 1], v2 = m.tris[3 * f + 2];
  const d3 e1 = ld3(X, v1) - ld3(X, v0), e2 = ld3(X, v2) - ld3(X, v0);
  const double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
  const d3 F0 = e1 * da + e2 * dc, F1 = e1 * db + e2 * dd;
  const Svd32 s = svd32(F0, F1);
  const d3 R0 = s.U0 * s.V00 + s.U1 * s.V01, R1 = s.U0 * s.V10 + s.U1 * s.V11;
  const d3 n = normalized(cross(s.U0, s.U1));
  const double k2 = 2.0 * m.rest_area[f] * thickness * mu;
  const double at = k2 * fmin(1.0, 2.0 / (s.s0 + s.s1));
  const double c0 = k2 * fmin(1.0, 1.0 / s.s0), c1 = k2 * fmin(1.0, 1.0 / s.s1);
  double* q = out + (long long)MFACE * f;
  q[0] = R0.x; q[1] = R0.y; q[2] = R0.z; q[3] = R1.x; q[4] = R1.y; q[5] = R1.z;
  q[6] = n.x; q[7] = n.y; q[8] = n.z;
  q[9] = at;
  q[10] = s.V00 * c0 * s.V00 + s.V01 * c1 * s.V01;
  q[11] = s.V00 * c0 * s.V10 + s.V01 * c1 * s.V11;
  q[12] = s.V10 * c0 * s.V10 + s.V11 * c1 * s.V11;
}

__device__ inline int warp_sum_i(int v) { for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o); return v; }
__device__ inline unsigned warp_and(unsigned v) { for (int o = 16; o; o >>= 1) v &= __shfl_xor_sync(0xffffffffu, v, o); return v; }
__device__ inline double warp_max_d(double v) { for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o)); return v; }

// StrainLimiting::rebuild_constraints + the Jacobian/derivatives used by
// accumulate_gradient and accumulate_hessian (strain_limiting.cpp:113-375),
// evaluated once per Newton iteration at the current positions. A face is
// active for singular value s when 1 + tau + eps - sigma_s <= eps.
__global__ void k_strain_face(MeshDev m, const double* x, StepParams p, unsigned char* flags, StrainSV* sv, Ctrl* ctrl) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  int nact = 0;
  if (f < m.T) {
    unsigned char fl = 0;
    if (m.rest_area[f] > 1e-12 && p.strain_eps > 0.0) {
      int i0 = m.tris[3 * f], i1 = m.tris[3 * f + 1], i2 = m.tris[3 * f + 2];
      d3 x0 = ld3(x, i0), x1 = ld3(x, i1), x2 = ld3(x, i2);
      d3 e1 = x1 - x0, e2 = x2 - x0;
      double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
      d3 F0 = e1 * da + e2 * dc, F1 = e1 * db + e2 * dd;
      Svd32 s = svd32(F0, F1);
      if (s.ok) {
        double sig[2] = {s.s0, s.s1};
        double top = 1.0 + p.strain_tau + p.strain_eps;
        bool act[2] = {in_domain(top - sig[0], p.strain_eps), in_domain(top - sig[1], p.strain_eps)};
        if (act[0] || act[1]) {
          d3 cen = (x0 + x1 + x2) / 3.0;
          d3 w[3] = {x0 - cen, x1 - cen, x2 - cen};
          double el = 0.0;  // w_r^T H_el(face 9x9) w_r; H_el blocks are diag(a, a, b)
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
              int sl = m.face_slot[9 * f + 3 * a + b];
              el += m.el_a[sl] * (w[a].x * w[b].x + w[a].y * w[b].y) + m.el_b[sl] * (w[a].z * w[b].z);
            }
          el = fmax(el, 0.0);
          double fmass = m.rest_area[f] * m.thickness * m.density;
          double min_gap = fmax(p.min_gap, 1e-8);
          bool avg = fabs(s.s0 - s.s1) < p.svd_eps;
          for (int q = 0; q < 2; ++q) {
            if (!act[q]) continue;
            double gap = top - sig[q];
            double gc = fmax(fabs(gap), min_gap);
            double k = fmass / (gc * gc) + el;
            d3 dS0, dS1;  // columns of dsigma/dF (3x2)
            if (avg) {
              dS0 = (s.U0 * s.V00 + s.U1 * s.V01) * 0.5;
              dS1 = (s.U0 * s.V10 + s.U1 * s.V11) * 0.5;
            } else if (q == 0) {
              dS0 = s.U0 * s.V00; dS1 = s.U0 * s.V10;
            } else {
              dS0 = s.U1 * s.V01; dS1 = s.U1 * s.V11;
            }
            d3 J1 = dS0 * da + dS1 * db, J2 = dS0 * dc + dS1 * dd, J0 = -(J1 + J2);
            StrainSV o;
            o.J[0] = J0.x; o.J[1] = J0.y; o.J[2] = J0.z; o.J[3] = J1.x; o.J[4] = J1.y; o.J[5] = J1.z;
            o.J[6] = J2.x; o.J[7] = J2.y; o.J[8] = J2.z;
            o.dV = bar_grad(gap, p.strain_eps, k);
            o.d2V = bar_hess(gap, p.strain_eps, k);
            sv[2 * f + q] = o;
            fl |= (unsigned char)(1u << q);
            ++nact;
          }
        }
      }
    }
    flags[f] = fl;
  }
  nact = warp_sum_i(nact);
  if ((threadIdx.x & 31) == 0 && nact) atomicAdd(&ctrl->strain_active, nact);
}

// Integrator::compute_gradient (integrator.cpp:246-396) for one vertex, in
// FP64: inertia, elastic + contact (per-step constants), strain limits, pins
// (Stiffness::compute_pin_stiffness + Barrier::compute_pin_gradient), walls
// (compute_wall_stiffness + compute_wall_gradient) and friction. It also
// writes the vertex's diagonal Hessian terms (mass, pin, wall, contact,
// friction blocks of assemble_system_matrix) for the assembly kernel, and
// folds |g|_inf into ctrl->gnorm_bits.
__global__ void __launch_bounds__(256, 3) k_gradient(MeshDev m, const double* x, const double* x_hat, const double* x_prev, const double* g_const,
                           const double* diag_const, const unsigned char* sflags, const StrainSV* sv,
                           const int* pin_vertex, const int* pin_head, const double* pin_target, int num_pins, const WallDev* walls,
                           const ContactDev* contacts, const ContactEntry* ents, const int* ebegin, const int* eend,
                           StepParams p, const unsigned char* fixed, double* g, float* b, double* diag_extra, Ctrl* ctrl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  double local = 0.0;
  if (i < m.V && fixed && fixed[i]) {
    // kinematic pin (CORRECTED): no degree of freedom, unit diagonal block
    st3(g, i, mk(0, 0, 0));
    b[3 * i] = 0.f; b[3 * i + 1] = 0.f; b[3 * i + 2] = 0.f;
    for (int k = 0; k < 9; ++k) diag_extra[9 * i + k] = (k % 4 == 0) ? 1.0 : 0.0;
  } else if (i < m.V) {
    double mi = m.mass[i];
    d3 xi = ld3(x, i), xh = ld3(x_hat, i);
    double mf = mi / (p.dt * p.dt);
    d3 gi = mk(mf * (xi.x - xh.x), mf * (xi.y - xh.y), mf * (xi.z - xh.z));
    gi = gi + ld3(g_const, i);
    if (p.enable_strain) {
      for (int k = m.vf_ptr[i]; k < m.vf_ptr[i + 1]; ++k) {
        int f = m.vf[k] / 3, a = m.vf[k] % 3;
        unsigned char fl = sflags[f];
        if (!fl) continue;
        for (int q = 0; q < 2; ++q) {
          if (!(fl & (1u << q))) continue;
          const StrainSV& S = sv[2 * f + q];
          if (fabs(S.dV) < 1e-12) continue;
          gi = gi + mk(S.J[3 * a], S.J[3 * a + 1], S.J[3 * a + 2]) * (-S.dV);
        }
      }
    }
    double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    double mdiag = mi * p.dt2inv;
    H[0] = H[4] = H[8] = mdiag;
    int ds = m.diag_slot[i];
    double A = mdiag + m.el_a[ds], B = mdiag + m.el_b[ds];
    double D0 = fmax(A, 1e-8), D2 = fmax(B, 1e-8);  // enforce_spd of the diagonal H_total block
    // CORRECTED pins attract: kappa / 2 |x - target|^2 per pin with
    // kappa = 100 (m / dt^2 + a), a the vertex's elastic diagonal coefficient
    if (num_pins > 0 && p.semantics == 1) {
      int lo = pin_head[i];
      double kp = PIN_SCALE * (mdiag + m.el_a[ds]);
      for (int k = lo; k >= 0 && k < num_pins && pin_vertex[k] == i; ++k) {
        gi = gi + (xi - mk(pin_target[3 * k], pin_target[3 * k + 1], pin_target[3 * k + 2])) * kp;
        H[0] += kp; H[4] += kp; H[8] += kp;
      }
    }
    // pins (sorted by vertex; pin_head[i] = first pin of vertex i or -1)
    if (num_pins > 0 && p.semantics == 0) {
      int lo = pin_head[i];
      for (int k = lo; k >= 0 && k < num_pins && pin_vertex[k] == i; ++k) {
        d3 off = xi - mk(pin_target[3 * k], pin_target[3 * k + 1], pin_target[3 * k + 2]);
        double len = nrm(off);
        d3 dir = len > 1e-9 ? off / len : mk(1, 0, 0);
        double kel = fmax(0.0, dir.x * (D0 * dir.x) + dir.y * (D0 * dir.y) + dir.z * (D2 * dir.z));
        double gh = fmax(fmax(len, p.min_gap), 1e-12);
        double kbar = mi / (gh * gh) + kel;
        double gap = len;
        if (!in_domain(gap, p.contact_gap_max) || gap <= p.normal_eps) continue;
        d3 n = off / gap;
        double dV = bar_grad(gap, p.contact_gap_max, kbar), d2V = bar_hess(gap, p.contact_gap_max, kbar);
        gi = gi + n * dV;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            double nn = comp(n, r) * comp(n, c);
            double val = d2V * nn + (dV / gap) * ((r == c ? 1.0 : 0.0) - nn);
            if (fabs(val) < p.barrier_tol) continue;
            H[3 * r + c] += val;
          }
      }
    }
    // walls
    for (int w = 0; w < p.num_walls; ++w) {
      const WallDev& W = walls[w];
      if (!W.active) continue;
      d3 wn = mk(W.n[0], W.n[1], W.n[2]);
      d3 n = normalize_or_default(wn, p.normal_eps);
      double gap = dot(n, xi) - W.offset;
      // REFERENCE: m / wall_gap^2; CORRECTED: m / g^2 at the current gap (as for contacts)
      double gh = fmax(fmax(p.semantics == 1 ? gap : p.wall_gap, p.min_gap), 1e-12);
      double wnn = nrm(wn);
      d3 ns = wnn > 1e-9 ? wn / wnn : mk(0, 1, 0);
      double kbar = mi / (gh * gh) + fmax(0.0, ns.x * (D0 * ns.x) + ns.y * (D0 * ns.y) + ns.z * (D2 * ns.z));
      if (!in_domain(gap, p.contact_gap_max)) continue;
      double dV = bar_grad(gap, p.contact_gap_max, kbar), d2V = bar_hess(gap, p.contact_gap_max, kbar);
      gi = gi + n * dV;
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
          double val = d2V * (comp(n, r) * comp(n, c));
          if (fabs(val) < p.barrier_tol) continue;
          H[3 * r + c] += val;
        }
    }
    // friction (integrator.cpp:374-395, 515-536; friction.cpp)
    if (p.enable_friction && p.friction_mu > 0.0) {
      d3 disp = xi - ld3(x_prev, i);
      for (int k = ebegin[i]; k < eend[i]; ++k) {
        ContactEntry E = ents[k];
        if (!(E.li & 8)) continue;
        const ContactDev& C = contacts[E.contact];
        d3 cn = mk(C.n[0], C.n[1], C.n[2]);
        d3 tg = disp - cn * dot(disp, cn);
        double tn = nrm(tg);
        if (!(tn > p.friction_thresh)) continue;
        double fn = C.kbar * fabs(C.gap);
        double den = fmax(p.friction_eps, fabs(tn));
        if (den <= 0.0) den = p.friction_eps;
        double kf = fmin(p.friction_mu * fabs(fn) / den, 1e8);
        gi = gi + tg * kf;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            double val = (r == c ? kf : 0.0) - kf * (comp(cn, r) * comp(cn, c)) + (r == c ? 1e-8 : 0.0);
            if (fabs(val) > 1e-12) H[3 * r + c] += val;
          }
      }
    }
    for (int k = 0; k < 9; ++k) H[k] += diag_const[9 * i + k];
    st3(g, i, gi);
    b[3 * i] = float(-gi.x); b[3 * i + 1] = float(-gi.y); b[3 * i + 2] = float(-gi.z);
    for (int k = 0; k < 9; ++k) diag_extra[9 * i + k] = H[k];
    auto mag = [](double v) { return v != v ? __longlong_as_double(0x7ff0000000000000ll) : fabs(v); };
    local = fmax(fmax(mag(gi.x), mag(gi.y)), mag(gi.z));
  }
  local = warp_max_d(local);
  if ((threadIdx.x & 31) == 0) atomicMax(&ctrl->gnorm_bits, (unsigned long long)__double_as_longlong(local));
}

__global__ void k_pin_heads(const int* pin_vertex, int num_pins, int* pin_head) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= num_pins) return;
  if (k == 0 || pin_vertex[k - 1] != pin_vertex[k]) pin_head[pin_vertex[k]] = k;
}

__global__ void k_check(Ctrl* c, double tol) {
  double gn = __longlong_as_double((long long)c->gnorm_bits);
  c->converged = gn < tol ? 1 : 0;
}

// assemble_system_matrix (integrator.cpp:398-544) as a per-slot gather: the
// constant elastic block, the strain-limit blocks of the faces sharing the
// slot (face order; StrainLimiting::accumulate_hessian drop rules), and for a
// diagonal slot the vertex's diagonal terms. Every contribution is symmetric
// by construction, so the reference's (H + H^T)/2 leaves it unchanged. The
// diagonal slot also yields the block-Jacobi inverse (pcg_solver.cpp:77-114).
// FP64 Hessian block of BSR slot s (row, col): the constant elastic block,
// the strain-limit blocks of the faces sharing the slot (face order;
// StrainLimiting::accumulate_hessian drop rules) and, for a diagonal slot, the
// vertex's diagonal terms.
// Projected exact membrane Hessian: the correction D_ab of face f's block
// (a, b) (k_membrane_face), D_ab = a_t / 2 g_a g_b^T + w_ab n n^T with
// g_a = G_a0 R1 - G_a1 R0 and w_ab = G_a W G_b^T, subtracted from H.
__device__ inline void membrane_correction(const MeshDev& m, int f, int a, int b, double H[9]) {
  const double* q = m.mface + (long long)MFACE * f;
  const double da = m.dm_inv[4 * f], db = m.dm_inv[4 * f + 1], dc = m.dm_inv[4 * f + 2], dd = m.dm_inv[4 * f + 3];
  const double Ga0 = a == 0 ? -(da + dc) : (a == 1 ? da : dc), Ga1 = a == 0 ? -(db + dd) : (a == 1 ? db : dd);
  const double Gb0 = b == 0 ? -(da + dc) : (b == 1 ? da : dc), Gb1 = b == 0 ? -(db + dd) : (b == 1 ? db : dd);
  const d3 R0 = mk(q[0], q[1], q[2]), R1 = mk(q[3], q[4], q[5]), n = mk(q[6], q[7], q[8]);
  const double at = q[9], W00 = q[10], W01 = q[11], W11 = q[12];
  const d3 ga = R1 * Ga0 - R0 * Ga1, gb = R1 * Gb0 - R0 * Gb1;
  const double w = Ga0 * (W00 * Gb0 + W01 * Gb1) + Ga1 * (W01 * Gb0 + W11 * Gb1);
  const double h = 0.5 * at;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) H[3 * r + c] -= h * comp(ga, r) * comp(gb, c) + w * comp(n, r) * comp(n, c);
}

__device__ inline void slot_block(const MeshDev& m, int s, int row, int col, const unsigned char* sflags, const StrainSV* sv,
                                  const double* diag_extra, int enable_strain, double H[9]) {
  for (int k = 0; k < 9; ++k) H[k] = 0.0;
  H[0] = H[4] = m.el_a[s]; H[8] = m.el_b[s];
  if (m.mface)
    for (int k = m.slot_cptr[s]; k < m.slot_cptr[s + 1]; ++k) {
      const int e = m.slot_contrib[k];
      membrane_correction(m, e / 9, (e % 9) / 3, e % 3, H);
    }
  if (enable_strain) {
    for (int k = m.slot_cptr[s]; k < m.slot_cptr[s + 1]; ++k) {
      int e = m.slot_contrib[k];
      int f = e / 9, a = (e % 9) / 3, bb = e % 3;
      unsigned char fl = sflags[f];
      if (!fl) continue;
      for (int q = 0; q < 2; ++q) {
        if (!(fl & (1u << q))) continue;
        const StrainSV& S = sv[2 * f + q];
        if (fabs(S.d2V) < 1e-12) continue;
        double blk[9], mx = 0.0;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) { blk[3 * r + c] = S.d2V * (S.J[3 * a + r] * S.J[3 * bb + c]); mx = fmax(mx, fabs(blk[3 * r + c])); }
        if (mx < 1e-12) continue;
        for (int k2 = 0; k2 < 9; ++k2) if (fabs(blk[k2]) >= 1e-12) H[k2] += blk[k2];
      }
    }
  }
  if (row == col) for (int k = 0; k < 9; ++k) H[k] += diag_extra[9 * row + k];
}

__global__ void k_assemble(MeshDev m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                           const unsigned char* fixed, float* val, float* precond, const Ctrl* ctrl) {
  if (ctrl->converged) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m.nnzb) return;
  int row = m.slot_row[s], col = m.cols[s];
  if (fixed && (fixed[row] || fixed[col])) {
    // kinematic pin: decoupled row and column, unit diagonal (diag_extra holds I)
    float one = row == col ? 1.f : 0.f;
    for (int k = 0; k < 9; ++k) val[9 * (long long)s + k] = (k % 4 == 0) ? one : 0.f;
    if (row == col) for (int k = 0; k < 9; ++k) precond[9 * (long long)row + k] = (k % 4 == 0) ? 1.f : 0.f;
    return;
  }
  double H[9];
  slot_block(m, s, row, col, sflags, sv, diag_extra, enable_strain, H);
  float hf[9];
  for (int k = 0; k < 9; ++k) { hf[k] = float(H[k]); val[9 * (long long)s + k] = hf[k]; }
  if (row == col) {
    double a0 = hf[0], a1 = hf[1], a2 = hf[2], a3 = hf[3], a4 = hf[4], a5 = hf[5], a6 = hf[6], a7 = hf[7], a8 = hf[8];
    double c00 = a4 * a8 - a5 * a7, c01 = a2 * a7 - a1 * a8, c02 = a1 * a5 - a2 * a4;
    double c10 = a5 * a6 - a3 * a8, c11 = a0 * a8 - a2 * a6, c12 = a2 * a3 - a0 * a5;
    double c20 = a3 * a7 - a4 * a6, c21 = a1 * a6 - a0 * a7, c22 = a0 * a4 - a1 * a3;
    double det = a0 * c00 + a1 * c10 + a2 * c20;
    float* P = precond + 9 * (long long)row;
    if (fabs(det) > 1e-16) {
      double inv = 1.0 / det;
      P[0] = float(c00 * inv); P[1] = float(c01 * inv); P[2] = float(c02 * inv);
      P[3] = float(c10 * inv); P[4] = float(c11 * inv); P[5] = float(c12 * inv);
      P[6] = float(c20 * inv); P[7] = float(c21 * inv); P[8] = float(c22 * inv);
    } else {
      P[0] = 1.f; P[1] = 0.f; P[2] = 0.f; P[3] = 0.f; P[4] = 1.f; P[5] = 0.f; P[6] = 0.f; P[7] = 0.f; P[8] = 1.f;
    }
  }
}

// ------------------------------------------------ scaled system (CORRECTED)
// Symmetric block scaling of the Newton system: with A_ii = L_i L_i^T (FP64
// Cholesky of the assembled diagonal block) the PCG runs on
// A^ = L^-1 A L^-T, whose diagonal blocks are I. Block-Jacobi PCG on A and CG
// on A^ are the same iteration in exact arithmetic. In FP32 they are not:
// contact and strain barriers make some diagonal blocks 1e10 times stiffer
// than the mass block next to them, FP32 sums over such a row cancel, and the
// unscaled iteration stalls; every stored entry of A^ is O(1). The scaling is
// applied in FP64, before the single rounding to FP32.
__device__ inline bool chol3(const double H[9], Tri3& L) {
  double a = H[0];
  if (!(a > 0.0)) return false;
  L.l00 = sqrt(a);
  L.l10 = H[3] / L.l00; L.l20 = H[6] / L.l00;
  double b = H[4] - L.l10 * L.l10;
  if (!(b > 0.0)) return false;
  L.l11 = sqrt(b);
  L.l21 = (H[7] - L.l20 * L.l10) / L.l11;
  double c = H[8] - L.l20 * L.l20 - L.l21 * L.l21;
  if (!(c > 0.0)) return false;
  L.l22 = sqrt(c);
  return true;
}
__device__ inline Tri3 tri_inv(const Tri3& L) {
  Tri3 M;
  M.l00 = 1.0 / L.l00; M.l11 = 1.0 / L.l11; M.l22 = 1.0 / L.l22;
  M.l10 = -L.l10 * M.l00 * M.l11;
  M.l21 = -L.l21 * M.l11 * M.l22;
  M.l20 = -(L.l20 * M.l00 + L.l21 * M.l10) * M.l22;
  return M;
}
// R = Mr H Mc^T with Mr, Mc lower triangular.
__device__ inline void scale_block(const Tri3& Mr, const double H[9], const Tri3& Mc, double R[9]) {
  double T[9];
  for (int c = 0; c < 3; ++c) {
    T[0 + c] = Mr.l00 * H[c];
    T[3 + c] = Mr.l10 * H[c] + Mr.l11 * H[3 + c];
    T[6 + c] = Mr.l20 * H[c] + Mr.l21 * H[3 + c] + Mr.l22 * H[6 + c];
  }
  for (int r = 0; r < 3; ++r) {
    const double* t = T + 3 * r;
    R[3 * r + 0] = t[0] * Mc.l00;
    R[3 * r + 1] = t[0] * Mc.l10 + t[1] * Mc.l11;
    R[3 * r + 2] = t[0] * Mc.l20 + t[1] * Mc.l21 + t[2] * Mc.l22;
  }
}
__device__ inline Tri3 ld_tri(const double* p, int i) {
  const double* q = p + 6 * (long long)i;
  Tri3 t; t.l00 = q[0]; t.l10 = q[1]; t.l11 = q[2]; t.l20 = q[3]; t.l21 = q[4]; t.l22 = q[5];
  return t;
}

// Per vertex: the FP64 diagonal block, its Cholesky factor L (a shifted
// factorisation when rounding made the block indefinite), L^-1 in FP64, L in
// FP32 (for the unscaled residual norm) and the scaled right-hand side
// b^ = -L^-1 g.
__global__ void k_diag_factor(MeshDev m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                              const unsigned char* fixed, const double* g, double* Linv, float* Lf, float* bhat,
                              unsigned char* chol_ok, const Ctrl* ctrl) {
  if (ctrl->converged) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.V) return;
  double H[9];
  if (fixed && fixed[i]) {
    for (int k = 0; k < 9; ++k) H[k] = (k % 4 == 0) ? 1.0 : 0.0;
  } else {
    slot_block(m, m.diag_slot[i], i, i, sflags, sv, diag_extra, enable_strain && ctrl->strain_active > 0, H);
  }
  Tri3 L;
  bool ok = chol3(H, L);
  if (!ok) {
    double tr = fabs(H[0]) + fabs(H[4]) + fabs(H[8]) + 1e-300;
    bool done = false;
    for (int t = 0; t < 3 && !done; ++t) {
      double Hs[9];
      for (int k = 0; k < 9; ++k) Hs[k] = H[k];
      double sh = tr * (t == 0 ? 1e-12 : (t == 1 ? 1e-8 : 1e-4));
      Hs[0] += sh; Hs[4] += sh; Hs[8] += sh;
      done = chol3(Hs, L);
    }
    if (!done) {
      L.l00 = sqrt(fmax(fabs(H[0]), 1e-300)); L.l11 = sqrt(fmax(fabs(H[4]), 1e-300)); L.l22 = sqrt(fmax(fabs(H[8]), 1e-300));
      L.l10 = L.l20 = L.l21 = 0.0;
    }
  }
  Tri3 M = tri_inv(L);
  double* q = Linv + 6 * (long long)i;
  q[0] = M.l00; q[1] = M.l10; q[2] = M.l11; q[3] = M.l20; q[4] = M.l21; q[5] = M.l22;
  float* lf = Lf + 6 * (long long)i;
  lf[0] = float(L.l00); lf[1] = float(L.l10); lf[2] = float(L.l11); lf[3] = float(L.l20); lf[4] = float(L.l21); lf[5] = float(L.l22);
  chol_ok[i] = ok ? 1 : 0;
  d3 gi = ld3(g, i);
  bhat[3 * i] = float(-(M.l00 * gi.x));
  bhat[3 * i + 1] = float(-(M.l10 * gi.x + M.l11 * gi.y));
  bhat[3 * i + 2] = float(-(M.l20 * gi.x + M.l21 * gi.y + M.l22 * gi.z));
}

// Per slot: the unscaled block (val, FP32; optional) and the scaled block
// valh = L_row^-1 H L_col^-T (FP32, computed in FP64). Diagonal slots of
// factored rows are exactly I.
// One scaled slot: R = the scaled block (FP32), H = the unscaled block. The
// scaled kernels pass enable_strain only when the strain pass of this Newton
// iteration counted an active face (ctrl->strain_active): with none, every
// face's flag is zero and the contribution walk adds nothing.
__device__ inline void scaled_slot(const MeshDev& m, int s, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra,
                                   int enable_strain, const unsigned char* fixed, const double* Linv, const unsigned char* chol_ok,
                                   float R[9], float Hf[9]) {
  int row = m.slot_row[s], col = m.cols[s];
  if (fixed && (fixed[row] || fixed[col])) {
    float one = row == col ? 1.f : 0.f;
    for (int k = 0; k < 9; ++k) { R[k] = (k % 4 == 0) ? one : 0.f; Hf[k] = R[k]; }
  } else {
    double H[9];
    slot_block(m, s, row, col, sflags, sv, diag_extra, enable_strain, H);
    for (int k = 0; k < 9; ++k) Hf[k] = float(H[k]);
    if (row == col && chol_ok[row]) {
      for (int k = 0; k < 9; ++k) R[k] = (k % 4 == 0) ? 1.f : 0.f;
    } else {
      double Rd[9];
      scale_block(ld_tri(Linv, row), H, ld_tri(Linv, col), Rd);
      for (int k = 0; k < 9; ++k) R[k] = float(Rd[k]);
    }
  }
}

__global__ void k_assemble_scaled(MeshDev m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                                  const unsigned char* fixed, const double* Linv, const unsigned char* chol_ok, float* val, float* valh,
                                  const int* sell_base, float* valh_sell, const Ctrl* ctrl) {
  if (ctrl->converged) return;
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= m.nnzb) return;
  float R[9], Hf[9];
  scaled_slot(m, s, sflags, sv, diag_extra, enable_strain && ctrl->strain_active > 0, fixed, Linv, chol_ok, R, Hf);
  if (val) for (int k = 0; k < 9; ++k) val[9 * (long long)s + k] = Hf[k];
  if (valh) for (int k = 0; k < 9; ++k) valh[9 * (long long)s + k] = R[k];
  float* vs = valh_sell + sell_base[s];
  for (int k = 0; k < 9; ++k) vs[32 * k] = R[k];
}

// The same values, one CTA per 32-row SELL slice: the slice's SELL region
// (contiguous, 9 x 32 floats per column slot) and, when asked for, its CSR
// slots' scaled and unscaled blocks (contiguous) are staged in shared memory
// and written with coalesced stores; the SELL padding gets zeros. wmax = the
// widest slice (column slots). The CSR-ordered copies are written only when
// a caller reads them (valh: the learned preconditioner's features; val:
// ando_last_system), and only their staging space is requested.
__global__ void __launch_bounds__(ASM_SLICE_TPB) k_assemble_scaled_slice(MeshDev m, const unsigned char* sflags, const StrainSV* sv,
                                                                         const double* diag_extra, int enable_strain,
                                                                         const unsigned char* fixed, const double* Linv,
                                                                         const unsigned char* chol_ok, float* val, float* valh,
                                                                         const int* sell_base, const int* chunk_off, int wmax,
                                                                         float* valh_sell, const Ctrl* ctrl) {
  if (ctrl->converged) return;
  extern __shared__ float asm_sm[];
  const int ch = blockIdx.x;
  const int r0 = 32 * ch, r1 = min(m.V, r0 + 32);
  const int k0 = m.rowptr[r0], nk = m.rowptr[r1] - k0;
  const int sell0 = 9 * chunk_off[ch], nsell = 9 * (chunk_off[ch + 1] - chunk_off[ch]);
  float* ss = asm_sm;                               // nsell: SELL order
  float* cs = valh ? ss + 9 * 32 * wmax : nullptr;  // 9 nk: scaled blocks, CSR order
  float* cv = val ? ss + 9 * 32 * wmax * (valh ? 2 : 1) : nullptr;  // 9 nk: unscaled blocks, CSR order
  for (int q = threadIdx.x; q < nsell; q += ASM_SLICE_TPB) ss[q] = 0.f;
  const int strain_on = enable_strain && ctrl->strain_active > 0;
  __syncthreads();
  for (int t = threadIdx.x; t < nk; t += ASM_SLICE_TPB) {
    const int s = k0 + t;
    float R[9], Hf[9];
    scaled_slot(m, s, sflags, sv, diag_extra, strain_on, fixed, Linv, chol_ok, R, Hf);
    const int sp = sell_base[s] - sell0;
    for (int k = 0; k < 9; ++k) ss[sp + 32 * k] = R[k];
    if (cs) for (int k = 0; k < 9; ++k) cs[9 * t + k] = R[k];
    if (cv) for (int k = 0; k < 9; ++k) cv[9 * t + k] = Hf[k];
  }
  __syncthreads();
  if (cs) {
    float* vh = valh + 9ll * k0;
    for (int q = threadIdx.x; q < 9 * nk; q += ASM_SLICE_TPB) vh[q] = cs[q];
  }
  if (cv) {
    float* vv = val + 9ll * k0;
    for (int q = threadIdx.x; q < 9 * nk; q += ASM_SLICE_TPB) vv[q] = cv[q];
  }
  float* vs = valh_sell + sell0;
  for (int q = threadIdx.x; q < nsell; q += ASM_SLICE_TPB) vs[q] = ss[q];
}

// Contact blocks outside the static pattern. Entries of the same (row, col)
// arrive adjacent (sorted by the 64-bit key row:col, stably, so in contact
// order) and merge into one block: the FP64 sum of k_extra_values' per-entry
// blocks, each with its |v| < barrier_tol drop rule. With Linv the merged
// block is scaled (L_row^-1 H L_col^-T) before the rounding to FP32.
__global__ void k_extra_key64(const ContactEntry* xent, const int* xkeys, int n, unsigned long long* key, int* idx) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  key[k] = ((unsigned long long)(unsigned)xkeys[k] << 32) | (unsigned long long)(unsigned)xent[k].col;
  idx[k] = k;
}
__global__ void k_run_heads(const unsigned long long* key, int n, int* flags) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  flags[k] = (k == 0 || key[k] != key[k - 1]) ? 1 : 0;
}
__global__ void k_extra_merge(const ContactDev* cs, const ContactEntry* xent, const unsigned long long* key, const int* idx, const int* heads,
                              int nu, int n, const unsigned char* fixed, StepParams p, const double* Linv, int* xrow, int* xcols,
                              float* xval, float* xvalh) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= nu) return;
  int k0 = heads[u], k1 = u + 1 < nu ? heads[u + 1] : n;
  int row = int(key[k0] >> 32), col = int(key[k0] & 0xffffffffull);
  if (xrow) { xrow[u] = row; xcols[u] = col; }
  double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  bool zero = fixed && (fixed[row] || fixed[col]);
  if (!zero) {
    for (int k = k0; k < k1; ++k) {
      ContactEntry E = xent[idx[k]];
      const ContactDev& C = cs[E.contact];
      int i = E.li & 3, j = E.lj;
      d3 nn = mk(C.nn[0], C.nn[1], C.nn[2]);
      d3 gi = nn * C.w[i], gj = nn * C.w[j];
      for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) {
          double v = C.d2V * (comp(gi, r) * comp(gj, q));
          if (!(fabs(v) < p.barrier_tol)) H[3 * r + q] += v;
        }
    }
  }
  if (xval) for (int q = 0; q < 9; ++q) xval[9 * (long long)u + q] = float(H[q]);
  if (xvalh) {
    double R[9];
    if (zero) for (int q = 0; q < 9; ++q) R[q] = 0.0;
    else scale_block(ld_tri(Linv, row), H, ld_tri(Linv, col), R);
    for (int q = 0; q < 9; ++q) xvalh[9 * (long long)u + q] = float(R[q]);
  }
}

// LineSearch::search / is_feasible (line_search.cpp:8-161) as a feasibility
// bitmask over the 20 halving levels: bit j <=> alpha = 2^-j is feasible.
// Wall part: every vertex against the first active wall.
__global__ void k_ls_wall(int V, const double* x, const float* d, WallDev w, Ctrl* ctrl) {
  if (ctrl->converged) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned mask = (1u << 20) - 1u;
  if (i < V) {
    d3 xi = ld3(x, i);
    d3 ext = mk(1.25 * double(d[3 * i]), 1.25 * double(d[3 * i + 1]), 1.25 * double(d[3 * i + 2]));
    d3 n = mk(w.n[0], w.n[1], w.n[2]);
    for (int j = 0; j < 20; ++j) {
      double a = ldexp(1.0, -j);
      d3 xn = xi + ext * a;
      if (dot(n, xn) - w.offset < 0.0) mask &= ~(1u << j);
    }
  }
  mask = warp_and(mask);
  if ((threadIdx.x & 31) == 0 && mask != ((1u << 20) - 1u)) atomicAnd(&ctrl->ls_mask, mask);
}

// LineSearch::ccd_point_triangle / ccd_edge_edge (line_search.cpp:163-247):
// 10 temporal samples t = i/10, a hit when the sampled distance is below 1e-6;
// the caller rejects the step when the returned time is < 1, so a hit at the
// last sample (t = 1) does not count and only samples 1..9 matter.
__device__ inline bool ccd_hit_pt(d3 p0, d3 p1, d3 a0, d3 a1, d3 b0, d3 b1, d3 c0, d3 c1) {
  if (sqn(p1 - p0) < 1e-12 && sqn(a1 - a0) < 1e-12 && sqn(b1 - b0) < 1e-12 && sqn(c1 - c0) < 1e-12) return false;
  for (int s = 1; s <= 9; ++s) {
    double t = double(s) / 10.0;
    double dist; d3 n, wq;
    narrow_pt(p0 + (p1 - p0) * t, a0 + (a1 - a0) * t, b0 + (b1 - b0) * t, c0 + (c1 - c0) * t, dist, n, wq);
    if (dist < 1e-6) return true;
  }
  return false;
}
__device__ inline bool ccd_hit_ee(d3 p00, d3 p01, d3 p10, d3 p11, d3 q00, d3 q01, d3 q10, d3 q11) {
  if (sqn(p01 - p00) < 1e-12 && sqn(p11 - p10) < 1e-12 && sqn(q01 - q00) < 1e-12 && sqn(q11 - q10) < 1e-12) return false;
  for (int s = 1; s <= 9; ++s) {
    double t = double(s) / 10.0;
    double dist;
    narrow_ee(p00 + (p01 - p00) * t, p10 + (p11 - p10) * t, q00 + (q01 - q00) * t, q10 + (q11 - q10) * t, dist);
    if (dist < 1e-6) return true;
  }
  return false;
}

__global__ void k_ls_contacts(const ContactDev* cs, int nc, const double* x, const float* d, Ctrl* ctrl) {
  if (ctrl->converged) return;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned mask = (1u << 20) - 1u;
  if (c < nc && (cs[c].type == 0 || cs[c].type == 1)) {
    const ContactDev& C = cs[c];
    d3 x0[4], e[4];
    for (int k = 0; k < 4; ++k) {
      x0[k] = ld3(x, C.idx[k]);
      e[k] = mk(1.25 * double(d[3 * C.idx[k]]), 1.25 * double(d[3 * C.idx[k] + 1]), 1.25 * double(d[3 * C.idx[k] + 2]));
    }
    for (int j = 0; j < 20; ++j) {
      double a = ldexp(1.0, -j);
      d3 x1[4];
      for (int k = 0; k < 4; ++k) x1[k] = x0[k] + e[k] * a;
      bool hit = C.type == 0 ? ccd_hit_pt(x0[0], x1[0], x0[1], x1[1], x0[2], x1[2], x0[3], x1[3])
                             : ccd_hit_ee(x0[0], x1[0], x0[1], x1[1], x0[2], x1[2], x0[3], x1[3]);
      // the end-state gap test (distance < 0) can never fail: a distance is >= 0
      if (hit) mask &= ~(1u << j);
    }
  }
  mask = warp_and(mask);
  if ((threadIdx.x & 31) == 0 && mask != ((1u << 20) - 1u)) atomicAnd(&ctrl->ls_mask, mask);
}

// First feasible level -> alpha; x += (alpha * 1.25) d when alpha >= 1e-8
// (integrator.cpp:216-228).
__global__ void k_update(int V, double* x, const float* d, Ctrl* ctrl) {
  if (ctrl->converged) return;
  unsigned mask = ctrl->ls_mask;
  double a = mask ? ldexp(1.0, -(__ffs(mask) - 1)) : 0.0;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ctrl->alpha = a;
  if (a < 1e-8 || i >= V) return;
  double s = a * 1.25;
  x[3 * i] += s * double(d[3 * i]);
  x[3 * i + 1] += s * double(d[3 * i + 1]);
  x[3 * i + 2] += s * double(d[3 * i + 2]);
}

// ------------------------------------------------------------- end of step
// v = (x - x_old) / (beta dt), then damping (integrator.cpp:123-140).
__global__ void k_velocity(int V, const double* x, const double* x_old, double beta_dt, double damp_scale, double* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * V) return;
  double vi = (x[i] - x_old[i]) / beta_dt;
  if (damp_scale != 1.0) vi *= damp_scale;
  v[i] = vi;
}

__device__ inline d3 mat3v(const double* M, d3 v) {
  return mk(M[0] * v.x + M[1] * v.y + M[2] * v.z, M[3] * v.x + M[4] * v.y + M[5] * v.z, M[6] * v.x + M[7] * v.y + M[8] * v.z);
}
// R * Ibody^-1 * R^T * v
__device__ inline d3 iworld_inv(const RigidDev& B, d3 v) {
  d3 t = mk(B.R[0] * v.x + B.R[3] * v.y + B.R[6] * v.z, B.R[1] * v.x + B.R[4] * v.y + B.R[7] * v.z, B.R[2] * v.x + B.R[5] * v.y + B.R[8] * v.z);
  return mat3v(B.R, mat3v(B.Iinv_body, t));
}

// Integrator::apply_contact_restitution, contact part (integrator.cpp:565-656).
// Impulses depend on earlier ones (shared vertices and bodies), so one thread
// walks the contact list in order.
__global__ void k_restitution_contacts(const ContactDev* cs, int nc, const double* mass, int V, double e, double gap_limit,
                                       RigidDev* bodies, int nb, double* v) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  auto impulse = [&](int idx, d3 nrm_) {
    if (idx < 0 || idx >= V) return;
    double nr = nrm(nrm_); if (nr < 1e-8) return;
    d3 n = nrm_ / nr;
    d3 vel = ld3(v, idx); double vn = dot(vel, n);
    if (vn < 0.0) st3(v, idx, vel - n * ((1.0 + e) * vn));
  };
  for (int c = 0; c < nc; ++c) {
    const ContactDev& C = cs[c];
    if (C.gap > gap_limit) continue;
    d3 n = mk(C.n[0], C.n[1], C.n[2]);
    if (C.type == 0) impulse(C.idx[0], n);
    else if (C.type == 1) { impulse(C.idx[0], n); impulse(C.idx[1], n); impulse(C.idx[2], -n); impulse(C.idx[3], -n); }
    else if (C.type == 2) impulse(C.idx[0], n);
    else if (C.type == 3 && C.rigid >= 0 && C.rigid < nb) {
      double nr = nrm(n); if (nr < 1e-8) continue;
      n = n / nr;
      int vi = C.idx[0]; if (vi < 0 || vi >= V) continue;
      RigidDev& B = bodies[C.rigid];
      d3 wq = mk(C.wq[0], C.wq[1], C.wq[2]);
      d3 pos = mk(B.pos[0], B.pos[1], B.pos[2]);
      d3 vv = ld3(v, vi);
      d3 bv = mk(B.lin[0], B.lin[1], B.lin[2]) + cross(mk(B.ang[0], B.ang[1], B.ang[2]), wq - pos);
      double vn = dot(vv - bv, n);
      if (vn >= 0.0) continue;
      double im = mass[vi] > 0.0 ? 1.0 / mass[vi] : 0.0;
      d3 cr = cross(wq - pos, n);
      double den = im + dot(cr, iworld_inv(B, cr));
      if (den <= 0.0) continue;
      double j = -(1.0 + e) * vn / den;
      d3 J = n * j;
      st3(v, vi, vv + J * im);
      if (B.mass > 0.0) {  // RigidBody::apply_impulse(witness_q, -J)
        d3 mJ = -J;
        B.lin[0] += mJ.x / B.mass; B.lin[1] += mJ.y / B.mass; B.lin[2] += mJ.z / B.mass;
        d3 dw = iworld_inv(B, cross(wq - pos, mJ));
        B.ang[0] += dw.x; B.ang[1] += dw.y; B.ang[2] += dw.z;
      }
    }
  }
}

// Wall part of apply_contact_restitution (integrator.cpp:657-673).
__global__ void k_restitution_walls(int V, const double* x, const WallDev* walls, int nw, double e, double gap_max, double* v) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  d3 xi = ld3(x, i);
  for (int w = 0; w < nw; ++w) {
    if (!walls[w].active) continue;
    d3 n = mk(walls[w].n[0], walls[w].n[1], walls[w].n[2]);
    double nr = nrm(n); if (nr < 1e-8) continue;
    n = n / nr;
    if (dot(n, xi) - walls[w].offset <= walls[w].gap + gap_max) {
      d3 vel = ld3(v, i); double vn = dot(vel, n);
      if (vn < 0.0) st3(v, i, vel - n * ((1.0 + e) * vn));
    }
  }
}

// Integrator::apply_rigid_coupling (integrator.cpp:676-754): one CTA per body
// sums barrier forces and torques over its contacts (fixed-order tree), then
// RigidBody::integrate (rigid_body.cpp:151-176).
__global__ void k_rigid_coupling(MeshDev m, const ContactDev* cs, StepParams p, RigidDev* bodies, int nb,
                                 const int* offsets, long long units, int ncontacts, double dt) {
  int bi = blockIdx.x;
  if (bi >= nb) return;
  RigidDev& B = bodies[bi];
  long long u0 = (long long)m.V + (long long)bi * m.V, u1 = u0 + m.V;
  int c0 = offsets[u0];
  int c1 = u1 < units ? offsets[u1] : ncontacts;
  d3 pos = mk(B.pos[0], B.pos[1], B.pos[2]);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) {
    const ContactDev& C = cs[c];
    if (C.type != 3) continue;
    double kbar = contact_kbar(m, C, p.dt);
    d3 n = mk(C.n[0], C.n[1], C.n[2]);
    double nr = nrm(n); if (nr < 1e-8) continue;
    n = n / nr;
    double dV = bar_grad(C.gap, p.contact_gap_max, kbar);
    if (fabs(dV) < 1e-12) continue;
    d3 F = -(n * dV);
    d3 tq = cross(mk(C.wq[0], C.wq[1], C.wq[2]) - pos, F);
    acc[0] += F.x; acc[1] += F.y; acc[2] += F.z; acc[3] += tq.x; acc[4] += tq.y; acc[5] += tq.z;
  }
  __shared__ double red[6][256];
  for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) for (int k = 0; k < 6; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x != 0 || B.mass <= 0.0) return;
  d3 F = mk(red[0][0], red[1][0], red[2][0]), T = mk(red[3][0], red[4][0], red[5][0]);
  d3 lin = mk(B.lin[0], B.lin[1], B.lin[2]) + (F / B.mass) * dt;
  d3 ang = mk(B.ang[0], B.ang[1], B.ang[2]) + iworld_inv(B, T) * dt;
  pos = pos + lin * dt;
  B.lin[0] = lin.x; B.lin[1] = lin.y; B.lin[2] = lin.z;
  B.ang[0] = ang.x; B.ang[1] = ang.y; B.ang[2] = ang.z;
  B.pos[0] = pos.x; B.pos[1] = pos.y; B.pos[2] = pos.z;
  double wn = nrm(ang);
  if (wn > 1e-8) {
    double th = wn * dt; d3 a = ang / wn;
    double c = cos(th), s = sin(th), t = 1.0 - c;
    double dR[9] = {t * a.x * a.x + c, t * a.x * a.y - s * a.z, t * a.x * a.z + s * a.y,
                    t * a.x * a.y + s * a.z, t * a.y * a.y + c, t * a.y * a.z - s * a.x,
                    t * a.x * a.z - s * a.y, t * a.y * a.z + s * a.x, t * a.z * a.z + c};
    double R2[9];
    for (int r = 0; r < 3; ++r)
      for (int q = 0; q < 3; ++q) R2[3 * r + q] = dR[3 * r] * B.R[q] + dR[3 * r + 1] * B.R[3 + q] + dR[3 * r + 2] * B.R[6 + q];
    for (int k = 0; k < 9; ++k) B.R[k] = R2[k];
  }
}

// ------------------------------------------------------- graph step control
__global__ void k_ctl_init(StepCtl* c, double beta_max, int max_it, cudaGraphConditionalHandle outer) {
  c->beta = 0.0; c->ret = 0.0; c->last_alpha = 0.0;
  c->bi = 0; c->newton_it = 0; c->max_it = max_it;
  c->newton_iters = c->pcg_iters = c->pcg_max = c->pcg_not_converged = c->line_search_fail = c->strain_active = c->error = 0;
  c->iterations_run = c->inner_steps = 0;
  c->phase = (0.0 < beta_max) ? 0 : 2;
  cudaGraphSetConditional(outer, c->phase != 2 ? 1u : 0u);
}

__global__ void k_inner_begin(StepCtl* c, cudaGraphConditionalHandle newton) {
  c->newton_it = 0;
  c->inner_steps++;
  cudaGraphSetConditional(newton, c->max_it > 0 ? 1u : 0u);
}

// After one Newton iteration: the decisions of inner_newton_step (integrator.cpp:169-235).
__global__ void k_newton_ctl(StepCtl* c, const Ctrl* ctrl, cudaGraphConditionalHandle newton) {
  bool stop = false;
  c->iterations_run++;
  c->strain_active = ctrl->strain_active;
  if (ctrl->converged) { c->ret = 1.0; stop = true; }
  else if (ctrl->pcg_status == PCG_TIMEOUT || ctrl->bar_err) { c->error = 1; c->ret = 0.0; stop = true; }
  else {
    c->newton_iters++;
    c->pcg_iters += ctrl->pcg_iters;
    c->pcg_max = max(c->pcg_max, ctrl->pcg_iters);
    if (!ctrl->pcg_converged) c->pcg_not_converged++;
    c->last_alpha = ctrl->alpha;
    if (ctrl->alpha < 1e-8) { c->ret = 0.0; stop = true; }
    else if (ctrl->alpha > 0.99) { c->ret = 1.0; stop = true; }
    else if (++c->newton_it >= c->max_it) { c->ret = 0.5; stop = true; }
  }
  cudaGraphSetConditional(newton, stop ? 0u : 1u);
}

// After one inner Newton step: beta accumulation and the error-reduction pass
// (integrator.cpp:98-121).
__global__ void k_outer_ctl(StepCtl* c, double beta_max, cudaGraphConditionalHandle outer) {
  if (c->error) { c->phase = 2; cudaGraphSetConditional(outer, 0u); return; }
  if (c->phase == 0) {
    double a = c->ret;
    c->beta = c->beta + (1.0 - c->beta) * a;
    c->bi++;
    bool more = true;
    if (a < 1e-6) { c->line_search_fail++; more = false; }
    if (more && !(c->beta < beta_max && c->bi < 20)) more = false;
    if (!more) c->phase = c->beta > 1e-6 ? 1 : 2;
  } else {
    c->phase = 2;
  }
  cudaGraphSetConditional(outer, c->phase != 2 ? 1u : 0u);
}

__global__ void k_velocity_ctl(int V, const double* x, const double* x_old, double dt, double damp_scale, double* v, const StepCtl* c) {
  double beta = c->beta;
  if (!(beta > 1e-6)) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * V) return;
  double vi = (x[i] - x_old[i]) / (beta * dt);
  if (damp_scale != 1.0) vi *= damp_scale;
  v[i] = vi;
}

}  // namespace

void launch_ctl_init(StepCtl* c, double beta_max, int max_it, cudaGraphConditionalHandle outer, cudaStream_t s) {
  k_ctl_init<<<1, 1, 0, s>>>(c, beta_max, max_it, outer);
}
void launch_inner_begin(StepCtl* c, cudaGraphConditionalHandle newton, cudaStream_t s) { k_inner_begin<<<1, 1, 0, s>>>(c, newton); }
void launch_newton_ctl(StepCtl* c, const Ctrl* ctrl, cudaGraphConditionalHandle newton, cudaStream_t s) {
  k_newton_ctl<<<1, 1, 0, s>>>(c, ctrl, newton);
}
void launch_outer_ctl(StepCtl* c, double beta_max, cudaGraphConditionalHandle outer, cudaStream_t s) {
  k_outer_ctl<<<1, 1, 0, s>>>(c, beta_max, outer);
}
void launch_velocity_ctl(int V, const double* x, const double* x_old, double dt, double damp_scale, double* v, const StepCtl* c, cudaStream_t s) {
  if (V) k_velocity_ctl<<<nblk(3ll * V), TPB, 0, s>>>(V, x, x_old, dt, damp_scale, v, c);
}

// ------------------------------------------------------------------ launchers
void launch_elastic_slots(const MeshDev& m, double mu, double thickness, int semantics, double* el_a, double* el_b, cudaStream_t s) {
  if (m.nnzb) k_elastic_slots<<<nblk(m.nnzb), TPB, 0, s>>>(m, mu, thickness, semantics, el_a, el_b);
}
void launch_elastic_gradient(const MeshDev& m, const double* X, double mu, double thickness, double* g, cudaStream_t s) {
  if (m.V) k_elastic_gradient<<<nblk(m.V), TPB, 0, s>>>(m, X, mu, thickness, g);
}
void launch_membrane_face(const MeshDev& m, const double* X, double mu, double thickness, double* out, cudaStream_t s) {
  if (m.T) k_membrane_face<<<nblk(m.T), TPB, 0, s>>>(m, X, mu, thickness, out);
}
void launch_arap_gradient(const MeshDev& m, const double* X, double mu, double thickness, double* g, cudaStream_t s) {
  if (m.V) k_arap_gradient<<<nblk(m.V), TPB, 0, s>>>(m, X, mu, thickness, g);
}
void launch_predict(int V, const double* x, const double* v, double dt, double* x_old, double* x_hat, cudaStream_t s) {
  if (V) k_predict<<<nblk(3ll * V), TPB, 0, s>>>(V, x, v, dt, x_old, x_hat);
}
void launch_gravity(int V, double* x, double* v, double gx, double gy, double gz, double dt, cudaStream_t s) {
  if (V) k_gravity<<<nblk(V), TPB, 0, s>>>(V, x, v, gx, gy, gz, dt);
}
void launch_rigid_world(RigidDev* bodies_dev, const RigidDev* bodies_host, int nb, cudaStream_t s) {
  int maxv = 0;
  for (int b = 0; b < nb; ++b) maxv = bodies_host[b].nv > maxv ? bodies_host[b].nv : maxv;
  if (nb && maxv) k_rigid_world<<<dim3(nblk(maxv), nb), TPB, 0, s>>>(bodies_dev, nb);
}
void launch_detect_count(const MeshDev& m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, int* counts, cudaStream_t s) {
  long long units = (long long)m.V * (1 + nb);
  if (units) k_detect_count<<<nblk(units), TPB, 0, s>>>(m, x, bodies, nb, literal_pt, thresh, counts);
}
void launch_detect_write(const MeshDev& m, const double* x, const RigidDev* bodies, int nb, int literal_pt, double thresh, const int* offsets, ContactDev* out, cudaStream_t s) {
  long long units = (long long)m.V * (1 + nb);
  if (units) k_detect_write<<<nblk(units), TPB, 0, s>>>(m, x, bodies, nb, literal_pt, thresh, offsets, out);
}
void launch_contact_prep(const MeshDev& m, ContactDev* c, int nc, const StepParams& p, cudaStream_t s) {
  if (nc) k_contact_prep<<<nblk(nc), TPB, 0, s>>>(m, c, nc, p);
}
void launch_contact_entries(const ContactDev* c, int nc, int V, int friction, int* keys, ContactEntry* ents, cudaStream_t s) {
  if (nc) k_contact_entries<<<nblk(16ll * nc), TPB, 0, s>>>(c, nc, V, friction, keys, ents);
}
void launch_vertex_ranges(const int* keys, int n, int V, int* begin, int* end, cudaStream_t s) {
  if (V) k_vertex_ranges<<<nblk(V), TPB, 0, s>>>(keys, n, V, begin, end);
}
void launch_contact_vertex(const MeshDev& m, const ContactDev* c, const ContactEntry* ents, const int* begin, const int* end,
                           const StepParams& p, const double* g_base, double* g_const, double* diag_const, cudaStream_t s) {
  if (m.V) k_contact_vertex<<<nblk(m.V), TPB, 0, s>>>(m, c, ents, begin, end, p, g_base, g_const, diag_const);
}
void launch_extra_flags(const ContactEntry* ents, const int* keys, int n, int* flags, cudaStream_t s) {
  if (n) k_extra_flags<<<nblk(n), TPB, 0, s>>>(ents, keys, n, flags);
}
void launch_ctrl_reset(Ctrl* ctrl, cudaStream_t s) { k_ctrl_reset<<<1, 1, 0, s>>>(ctrl); }
void launch_strain_face(const MeshDev& m, const double* x, const StepParams& p, unsigned char* flags, StrainSV* sv, Ctrl* ctrl, cudaStream_t s) {
  if (m.T) k_strain_face<<<nblk(m.T), TPB, 0, s>>>(m, x, p, flags, sv, ctrl);
}
void launch_pin_heads(const int* pin_vertex, int num_pins, int* pin_head, cudaStream_t s) {
  if (num_pins) k_pin_heads<<<nblk(num_pins), TPB, 0, s>>>(pin_vertex, num_pins, pin_head);
}
void launch_gradient(const MeshDev& m, const double* x, const double* x_hat, const double* x_prev, const double* g_const,
                     const double* diag_const, const unsigned char* sflags, const StrainSV* sv,
                     const int* pin_vertex, const int* pin_head, const double* pin_target, int num_pins, const WallDev* walls,
                     const ContactDev* contacts, const ContactEntry* ents, const int* ebegin, const int* eend,
                     const StepParams& p, const unsigned char* fixed, double* g, float* b, double* diag_extra, Ctrl* ctrl, cudaStream_t s) {
  if (m.V) k_gradient<<<nblk(m.V), TPB, 0, s>>>(m, x, x_hat, x_prev, g_const, diag_const, sflags, sv, pin_vertex, pin_head, pin_target, num_pins, walls,
                                                contacts, ents, ebegin, eend, p, fixed, g, b, diag_extra, ctrl);
}
void launch_check(Ctrl* ctrl, double tol, cudaStream_t s) { k_check<<<1, 1, 0, s>>>(ctrl, tol); }
void launch_assemble(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                     const unsigned char* fixed, float* val, float* precond, const Ctrl* ctrl, cudaStream_t s) {
  if (m.nnzb) k_assemble<<<nblk(m.nnzb), TPB, 0, s>>>(m, sflags, sv, diag_extra, enable_strain, fixed, val, precond, ctrl);
}
void launch_diag_factor(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                        const unsigned char* fixed, const double* g, double* Linv, float* Lf, float* bhat, unsigned char* chol_ok,
                        const Ctrl* ctrl, cudaStream_t s, int tpb) {
  if (m.V) k_diag_factor<<<nblk(m.V, tpb), tpb, 0, s>>>(m, sflags, sv, diag_extra, enable_strain, fixed, g, Linv, Lf, bhat, chol_ok, ctrl);
}
void launch_assemble_scaled(const MeshDev& m, const unsigned char* sflags, const StrainSV* sv, const double* diag_extra, int enable_strain,
                            const unsigned char* fixed, const double* Linv, const unsigned char* chol_ok, float* val, float* valh,
                            const int* sell_base, float* valh_sell, const Ctrl* ctrl, cudaStream_t s, int tpb, const int* chunk_off,
                            int wmax) {
  if (!m.nnzb) return;
  if (chunk_off && wmax > 0 && wmax <= ASM_SLICE_WMAX) {
    static std::atomic<unsigned> attr{0};  // one bit per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 32 && !(attr.load() & (1u << dev))) {
      if (cudaFuncSetAttribute(k_assemble_scaled_slice, cudaFuncAttributeMaxDynamicSharedMemorySize, int(asm_slice_smem(ASM_SLICE_WMAX, 3))) ==
          cudaSuccess)
        attr.fetch_or(1u << dev);
    }
    if (dev < 32 && (attr.load() & (1u << dev))) {
      const int copies = 1 + (valh ? 1 : 0) + (val ? 1 : 0);
      k_assemble_scaled_slice<<<(m.V + 31) / 32, ASM_SLICE_TPB, asm_slice_smem(wmax, copies), s>>>(
          m, sflags, sv, diag_extra, enable_strain, fixed, Linv, chol_ok, val, valh, sell_base, chunk_off, wmax, valh_sell, ctrl);
      return;
    }
  }
  k_assemble_scaled<<<nblk(m.nnzb, tpb), tpb, 0, s>>>(m, sflags, sv, diag_extra, enable_strain, fixed, Linv, chol_ok, val, valh, sell_base,
                                                      valh_sell, ctrl);
}
void launch_extra_key64(const ContactEntry* xent, const int* xkeys, int n, unsigned long long* key, int* idx, cudaStream_t s) {
  if (n) k_extra_key64<<<nblk(n), TPB, 0, s>>>(xent, xkeys, n, key, idx);
}
void launch_run_heads(const unsigned long long* key, int n, int* flags, cudaStream_t s) {
  if (n) k_run_heads<<<nblk(n), TPB, 0, s>>>(key, n, flags);
}
void launch_extra_merge(const ContactDev* c, const ContactEntry* xent, const unsigned long long* key, const int* idx, const int* heads, int nu,
                        int n, const unsigned char* fixed, const StepParams& p, const double* Linv, int* xrow, int* xcols, float* xval,
                        float* xvalh, cudaStream_t s) {
  if (nu) k_extra_merge<<<nblk(nu), TPB, 0, s>>>(c, xent, key, idx, heads, nu, n, fixed, p, Linv, xrow, xcols, xval, xvalh);
}
void launch_ls_wall(int V, const double* x, const float* d, WallDev w, Ctrl* ctrl, cudaStream_t s) {
  if (V) k_ls_wall<<<nblk(V), TPB, 0, s>>>(V, x, d, w, ctrl);
}
void launch_ls_contacts(const ContactDev* c, int nc, const double* x, const float* d, Ctrl* ctrl, cudaStream_t s) {
  if (nc) k_ls_contacts<<<nblk(nc), TPB, 0, s>>>(c, nc, x, d, ctrl);
}
void launch_update(int V, double* x, const float* d, Ctrl* ctrl, cudaStream_t s) {
  k_update<<<nblk(V > 0 ? V : 1), TPB, 0, s>>>(V, x, d, ctrl);
}
void launch_velocity(int V, const double* x, const double* x_old, double beta_dt, double damp_scale, double* v, cudaStream_t s) {
  if (V) k_velocity<<<nblk(3ll * V), TPB, 0, s>>>(V, x, x_old, beta_dt, damp_scale, v);
}
void launch_restitution_contacts(const ContactDev* c, int nc, const double* mass, int V, double e, double gap_limit,
                                 RigidDev* bodies, int nb, double* v, cudaStream_t s) {
  if (nc) k_restitution_contacts<<<1, 1, 0, s>>>(c, nc, mass, V, e, gap_limit, bodies, nb, v);
}
void launch_restitution_walls(int V, const double* x, const WallDev* walls, int nw, double e, double gap_max, double* v, cudaStream_t s) {
  if (V && nw) k_restitution_walls<<<nblk(V), TPB, 0, s>>>(V, x, walls, nw, e, gap_max, v);
}
void launch_rigid_coupling(const MeshDev& m, const ContactDev* c, int nc, const StepParams& p, RigidDev* bodies, int nb,
                           const int* offsets, long long units, double dt, cudaStream_t s) {
  if (nb) k_rigid_coupling<<<nb, 256, 0, s>>>(m, c, p, bodies, nb, offsets, units, nc, dt);
}

}  // namespace ando
