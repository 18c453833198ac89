// ando_oracle.hpp -- CPU oracle for the AndoSim implicit cloth/shell step.
//
// TEST INFRASTRUCTURE ONLY. This header restates, in plain C++17 with no
// third-party dependency, the algorithm of the reference implementation
// (Slaymish/AndoSim, src/core/*.cpp). It is the checker the CUDA path is
// compared against and the CPU baseline timed beside it; the product
// (andosim_b200/) never includes, links or calls it.
//
// Everything is templated on the scalar type R: R=double is the FP64 run the
// position-error gate is judged against, R=float mirrors the reference's
// default build (types.h:12-16, Real=float).
//
// Two switches:
//   Lookup::LITERAL  -- the reference's full-matrix scans per vertex / contact
//                       (stiffness.cpp:13-49,213-234, strain_limiting.cpp:52-104);
//                       O(V*nnz) per Newton iteration, kept for faithful timing.
//   Lookup::INDEXED  -- the same arithmetic with O(1) block access.
//   Both give identical numbers (the scans only *find* entries).
//
// Broad phase:
//   BroadPhase::LITERAL  -- the reference's median-split BVH, including the
//                           leaf defect (collision.cpp:81-86): leaves of 2..4
//                           primitives carry no primitive, so a mesh with >= 2
//                           triangles yields no self-contact candidates.
//   BroadPhase::INTENDED -- brute force over the reference's own overlap
//                           predicate (collision.h:37-41, point box +-1e-4,
//                           incident-face and shared-vertex exclusions).
//
// Third-party arithmetic the reference delegates to Eigen 3.4 (not present
// here) is restated from its mathematical definition:
//   * SelfAdjointEigenSolver<Mat3> in Stiffness::enforce_spd -> cyclic Jacobi
//     eigen-decomposition of the symmetric 3x3 (exact for the diagonal blocks
//     the reference actually feeds it);
//   * JacobiSVD<Mat32> in StrainLimiting::compute_svd -> eigen-decomposition of
//     F^T F (2x2, closed form), sigma sorted descending, u_s = F v_s / sigma_s;
//   * SparseMatrix::setFromTriplets -> CSR with duplicates summed in insertion
//     order, columns sorted;
//   * Matrix3::determinant/inverse -> cofactor expansion / adjugate.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>
#include <cstdlib>
#include <thread>

namespace ando_oracle {

// Loop over [0, n) on the host's cores (ANDO_ORACLE_THREADS, default all),
// in static chunks: used only where every index computes and writes its own
// results, so the outcome is the same bits as one thread's.
inline int oracle_threads() {
  static const int t = [] {
    const char* e = std::getenv("ANDO_ORACLE_THREADS");
    int v = e ? std::atoi(e) : int(std::thread::hardware_concurrency());
    return v > 0 ? v : 1;
  }();
  return t;
}
template <class F> void parallel_for(long long n, F&& f) {
  const int T = oracle_threads();
  if (T <= 1 || n < 4096) { for (long long i = 0; i < n; ++i) f(i); return; }
  const long long chunk = (n + T - 1) / T;
  std::vector<std::thread> th;
  for (int k = 0; k < T; ++k) {
    const long long lo = k * chunk, hi = std::min(n, lo + chunk);
    if (lo >= hi) break;
    th.emplace_back([lo, hi, &f] { for (long long i = lo; i < hi; ++i) f(i); });
  }
  for (auto& t : th) t.join();
}


enum class Lookup { LITERAL, INDEXED };
enum class BroadPhase { LITERAL, INTENDED };

// ---------------------------------------------------------------- small math
template <class R> struct V3 {
  R x = 0, y = 0, z = 0;
  V3() = default;
  V3(R a, R b, R c) : x(a), y(b), z(c) {}
  R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3& o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(const V3& o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator-() const { return {-x, -y, -z}; }
  V3 operator*(R s) const { return {x * s, y * s, z * s}; }
  V3 operator/(R s) const { return {x / s, y / s, z / s}; }
  V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  R dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
  R sq() const { return x * x + y * y + z * z; }
  R norm() const { return std::sqrt(sq()); }
  V3 cross(const V3& o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
  // Eigen-style normalized(): zero vector stays zero.
  V3 normalized() const { R n2 = sq(); return n2 > R(0) ? (*this) / std::sqrt(n2) : *this; }
};
template <class R> V3<R> operator*(R s, const V3<R>& v) { return v * s; }

template <class R> struct M3 {
  R m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  static M3 identity() { M3 a; a.m[0][0] = a.m[1][1] = a.m[2][2] = R(1); return a; }
  R& operator()(int i, int j) { return m[i][j]; }
  R operator()(int i, int j) const { return m[i][j]; }
  V3<R> operator*(const V3<R>& v) const {
    return {m[0][0] * v.x + m[0][1] * v.y + m[0][2] * v.z,
            m[1][0] * v.x + m[1][1] * v.y + m[1][2] * v.z,
            m[2][0] * v.x + m[2][1] * v.y + m[2][2] * v.z};
  }
  M3 operator*(const M3& o) const {
    M3 r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][0] * o.m[0][j] + m[i][1] * o.m[1][j] + m[i][2] * o.m[2][j];
    return r;
  }
  M3 operator+(const M3& o) const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] + o.m[i][j]; return r; }
  M3 operator-(const M3& o) const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] - o.m[i][j]; return r; }
  M3 operator*(R s) const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[i][j] * s; return r; }
  M3 transpose() const { M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = m[j][i]; return r; }
  static M3 outer(const V3<R>& a, const V3<R>& b) {
    M3 r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.m[i][j] = a[i] * b[j]; return r;
  }
  R determinant() const {
    return m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) -
           m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2]) +
           m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
  }
  // Adjugate / determinant (pcg_solver.cpp:106-108 delegates to Matrix3::inverse).
  M3 inverse() const {
    M3 c;
    c.m[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
    c.m[0][1] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
    c.m[0][2] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
    c.m[1][0] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
    c.m[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
    c.m[1][2] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
    c.m[2][0] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
    c.m[2][1] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
    c.m[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
    R det = m[0][0] * c.m[0][0] + m[0][1] * c.m[1][0] + m[0][2] * c.m[2][0];
    R inv = R(1) / det;
    return c * inv;
  }
};

template <class R> struct M2 {
  R a = 0, b = 0, c = 0, d = 0;  // [[a b][c d]]
  M2 inverse() const { R det = a * d - b * c; R inv = R(1) / det; return {d * inv, -b * inv, -c * inv, a * inv}; }
  M2 transpose() const { return {a, c, b, d}; }
  M2 operator*(const M2& o) const { return {a * o.a + b * o.c, a * o.b + b * o.d, c * o.a + d * o.c, c * o.b + d * o.d}; }
  M2 operator*(R s) const { return {a * s, b * s, c * s, d * s}; }
};

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations; eigenvalues
// ascending, eigenvectors in columns. Restates the role of Eigen's
// SelfAdjointEigenSolver<Mat3> (stiffness.cpp:241). A diagonal input needs no
// rotation and is reproduced exactly.
template <class R> void sym_eigen3(const M3<R>& A, V3<R>& evals, M3<R>& evecs) {
  double a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) a[i][j] = double(A(i, j));
  for (int sweep = 0; sweep < 64; ++sweep) {
    double off = std::fabs(a[0][1]) + std::fabs(a[0][2]) + std::fabs(a[1][2]);
    if (off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- A J
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq; a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {  // A <- J^T A
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk; a[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          double vkp = v[k][p], vkq = v[k][q];
          v[k][p] = c * vkp - s * vkq; v[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int idx[3] = {0, 1, 2};
  std::sort(idx, idx + 3, [&](int i, int j) { return a[i][i] < a[j][j]; });
  for (int k = 0; k < 3; ++k) {
    evals[k] = R(a[idx[k]][idx[k]]);
    for (int r = 0; r < 3; ++r) evecs(r, k) = R(v[r][idx[k]]);
  }
}

// ---------------------------------------------------------------- data model
using Index = int32_t;
struct Triangle { Index v[3] = {-1, -1, -1}; Triangle() = default; Triangle(Index a, Index b, Index c) { v[0] = a; v[1] = b; v[2] = c; } };
struct Edge { Index v[2] = {-1, -1}; };
// One interior edge of the quadratic bending energy (CORRECTED semantics):
// v = the edge's ends, then the vertex opposite it in each of its two faces;
// w = the cotangent stencil over v at rest; c = 6 / (rest area of the two faces).
struct Hinge { Index v[4] = {-1, -1, -1, -1}; double w[4] = {0, 0, 0, 0}; double c = 0; };

// types.h:51-57
template <class R> struct Material {
  R youngs_modulus = R(1e6), poisson_ratio = R(0.3), density = R(1000.0), thickness = R(0.001), bending_stiffness = R(0);
};

// types.h:60-100 (all defaults as in the reference)
template <class R> struct SimParams {
  R dt = R(0.002); R beta_max = R(0.25); int min_newton_steps = 2; int max_newton_steps = 8;
  int friction_min_newton_steps = 32;
  R pcg_tol = R(1e-3); int pcg_max_iters = 1000;
  R contact_gap_max = R(0.001); R wall_gap = R(0.001); bool enable_ccd = true;
  R contact_normal_epsilon = R(1e-8); R barrier_tolerance = R(1e-12);
  bool enable_friction = false; R friction_mu = R(0.1); R friction_epsilon = R(1e-5); R friction_tangent_threshold = R(1e-6);
  R velocity_damping = R(0); R contact_restitution = R(0);
  bool enable_strain_limiting = false; R strain_limit = R(0.05); R strain_tau = R(0.05); R strain_epsilon = R(0); R strain_svd_epsilon = R(1e-6);
  R hessian_epsilon = R(1e-8); R min_gap = R(1e-8);
  // CORRECTED only: 0 = the constant fixed-rotation membrane Hessian, 1 = the
  // exact membrane Hessian projected to positive semidefinite per face
  int membrane_hessian = 0;
};

// mesh.cpp:8-151
template <class R> struct Mesh {
  std::vector<V3<R>> vertices;
  std::vector<Triangle> triangles;
  std::vector<Edge> edges;
  std::vector<M2<R>> Dm_inv;
  std::vector<R> rest_areas;
  std::vector<std::vector<Index>> vertex_to_faces, vertex_to_edges;
  std::vector<Hinge> hinges;
  Material<R> material;

  void initialize(const std::vector<V3<R>>& verts, const std::vector<Triangle>& tris, const Material<R>& mat) {
    vertices = verts; triangles = tris; material = mat; compute_rest_state();
  }
  void compute_rest_state() {
    compute_edges();
    vertex_to_faces.assign(vertices.size(), {});
    vertex_to_edges.assign(vertices.size(), {});
    for (size_t i = 0; i < triangles.size(); ++i)
      for (int j = 0; j < 3; ++j) vertex_to_faces[triangles[i].v[j]].push_back(Index(i));
    for (size_t i = 0; i < edges.size(); ++i) { vertex_to_edges[edges[i].v[0]].push_back(Index(i)); vertex_to_edges[edges[i].v[1]].push_back(Index(i)); }
    Dm_inv.assign(triangles.size(), M2<R>{});
    rest_areas.assign(triangles.size(), R(0));
    const R eps = R(1e-12);
    for (size_t i = 0; i < triangles.size(); ++i) {
      const auto& t = triangles[i];
      V3<R> e1 = vertices[t.v[1]] - vertices[t.v[0]], e2 = vertices[t.v[2]] - vertices[t.v[0]];
      R l1 = e1.sq(), l2 = e2.sq();
      if (l1 < eps || l2 < eps) continue;  // degenerate: zero area and Dm_inv (mesh.cpp:31-35)
      V3<R> n = e1.cross(e2);
      R nl = n.norm();
      if (nl < eps) continue;
      rest_areas[i] = nl * R(0.5);
      V3<R> nu = n / nl, t1 = e1 / std::sqrt(l1), t2 = nu.cross(t1);
      M2<R> Dm{e1.dot(t1), e2.dot(t1), e1.dot(t2), e2.dot(t2)};
      Dm_inv[i] = Dm.inverse();
    }
    compute_hinges();
  }
  // Quadratic bending (no reference counterpart: the reference declares
  // Material::bending_stiffness, types.h:56, and never reads it). For every
  // edge shared by exactly two faces (ends i, j; opposite vertices k in one
  // face, l in the other) the stencil K over (i, j, k, l) at rest is
  //   K = [cot a_j + cot b_j, cot a_i + cot b_i, -(cot a_i + cot a_j), -(cot b_i + cot b_j)]
  // with a_i, a_j the rest angles of the first face at i and j and b_i, b_j
  // those of the second. K annihilates every affine map of a flat rest sheet,
  // and for an isometric fold by a dihedral angle t, |K x|^2 = |e|^2 (2 sin t/2)^2:
  // E = k_b sum_e 3 / A_e |K_e x|^2 is the discrete-shell hinge energy
  // k_b sum_e 3 |e|^2 / A_e t_e^2 to second order in t (A_e = rest area of the
  // two faces), quadratic in x (Bergou, Wardetzky, Harmon, Zorin, Grinspun,
  // "A Quadratic Bending Model for Inextensible Surfaces", SGP 2006). The rest
  // shape is taken as flat. Edges with a degenerate face are skipped.
  void compute_hinges() {
    hinges.clear();
    std::unordered_map<uint64_t, std::vector<std::pair<Index, Index>>> faces_of;  // edge key -> (face, opposite vertex)
    for (size_t f = 0; f < triangles.size(); ++f)
      for (int i = 0; i < 3; ++i) {
        Index a = triangles[f].v[i], b = triangles[f].v[(i + 1) % 3], o = triangles[f].v[(i + 2) % 3];
        Index lo = std::min(a, b), hi = std::max(a, b);
        faces_of[(uint64_t(uint32_t(lo)) << 32) | uint64_t(uint32_t(hi))].push_back({Index(f), o});
      }
    auto cot = [&](Index at, Index p, Index q, bool& ok) {
      double u[3], w[3];
      for (int k = 0; k < 3; ++k) { u[k] = double(vertices[p][k]) - double(vertices[at][k]); w[k] = double(vertices[q][k]) - double(vertices[at][k]); }
      double cr[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
      double s = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
      if (!(s > 0.0)) { ok = false; return 0.0; }
      return (u[0] * w[0] + u[1] * w[1] + u[2] * w[2]) / s;
    };
    for (const auto& e : edges) {
      uint64_t key = (uint64_t(uint32_t(e.v[0])) << 32) | uint64_t(uint32_t(e.v[1]));
      auto it = faces_of.find(key);
      if (it == faces_of.end() || it->second.size() != 2) continue;
      Index i = e.v[0], j = e.v[1], k = it->second[0].second, l = it->second[1].second;
      bool ok = true;
      double ai = cot(i, j, k, ok), aj = cot(j, i, k, ok), bi = cot(i, j, l, ok), bj = cot(j, i, l, ok);
      double area = double(rest_areas[size_t(it->second[0].first)]) + double(rest_areas[size_t(it->second[1].first)]);
      if (!ok || !(area > 0.0)) continue;
      Hinge h;
      h.v[0] = i; h.v[1] = j; h.v[2] = k; h.v[3] = l;
      h.w[0] = aj + bj; h.w[1] = ai + bi; h.w[2] = -(ai + aj); h.w[3] = -(bi + bj);
      h.c = 6.0 / area;
      hinges.push_back(h);
    }
  }
  // mesh.cpp:77-98: unique edges in first-seen order over faces.
  void compute_edges() {
    std::unordered_set<uint64_t> seen;
    edges.clear();
    for (const auto& t : triangles)
      for (int i = 0; i < 3; ++i) {
        Index a = t.v[i], b = t.v[(i + 1) % 3];
        Index lo = std::min(a, b), hi = std::max(a, b);
        uint64_t key = (uint64_t(uint32_t(lo)) << 32) | uint64_t(uint32_t(hi));
        if (seen.insert(key).second) { Edge e; e.v[0] = lo; e.v[1] = hi; edges.push_back(e); }
      }
  }
  // mesh.cpp:126-151: F in the deformed local frame of mesh.vertices.
  M2<R> compute_F(size_t f) const {
    const auto& t = triangles[f];
    V3<R> e1 = vertices[t.v[1]] - vertices[t.v[0]], e2 = vertices[t.v[2]] - vertices[t.v[0]];
    V3<R> n = e1.cross(e2).normalized(), t1 = e1.normalized(), t2 = n.cross(t1);
    M2<R> Ds{e1.dot(t1), e2.dot(t1), e1.dot(t2), e2.dot(t2)};
    return Ds * Dm_inv[f];
  }
};

// state.cpp:6-32
template <class R> struct State {
  std::vector<V3<R>> positions, velocities, positions_prev;
  // CORRECTED semantics only: where the last step ended (or what the caller
  // set), the start of the intersection-free move of the next step.
  std::vector<V3<R>> positions_safe;
  std::vector<R> masses;
  void initialize(const Mesh<R>& mesh) {
    if (mesh.vertices.empty()) throw std::invalid_argument("Mesh must be initialised before creating a state");
    positions = mesh.vertices; positions_prev = mesh.vertices; positions_safe = mesh.vertices;
    velocities.assign(mesh.vertices.size(), V3<R>());
    masses.assign(mesh.vertices.size(), R(0));
    for (size_t i = 0; i < mesh.triangles.size(); ++i) {
      R face_mass = mesh.rest_areas[i] * mesh.material.thickness * mesh.material.density;
      R vm = R(double(face_mass) / 3.0);
      for (int j = 0; j < 3; ++j) masses[mesh.triangles[i].v[j]] += vm;
    }
  }
  // bindings.cpp:284-300
  void apply_gravity(const V3<R>& g, R dt) {
    if (positions.empty()) throw std::runtime_error("State has not been initialised");
    for (size_t i = 0; i < positions.size(); ++i) { velocities[i] += g * dt; positions[i] += velocities[i] * dt; }
  }
};

// constraints.h:26-70, constraints.cpp:5-20
template <class R> struct Pin { Index vertex_idx = 0; V3<R> target_position; bool active = true; };
template <class R> struct Wall { V3<R> normal; R offset = 0; R gap = 0; bool active = true; };
template <class R> struct StrainConstraint { Index face_idx = 0; R sigma = 0; int singular_index = 0; R stiffness = 0; bool active = true; };
template <class R> struct Constraints {
  std::vector<Pin<R>> pins;
  std::vector<Wall<R>> walls;
  std::vector<StrainConstraint<R>> strain_limits;
  void add_pin(Index i, const V3<R>& t) { Pin<R> p; p.vertex_idx = i; p.target_position = t; pins.push_back(p); }
  void add_wall(const V3<R>& n, R off, R gap) { Wall<R> w; w.normal = n.normalized(); w.offset = off; w.gap = gap; walls.push_back(w); }
  size_t num_active_pins() const { size_t c = 0; for (auto& p : pins) c += p.active; return c; }
  size_t num_active_walls() const { size_t c = 0; for (auto& w : walls) c += w.active; return c; }
};

enum class ContactType { POINT_TRIANGLE = 0, EDGE_EDGE = 1, WALL = 2, RIGID_POINT_TRIANGLE = 3 };

// collision.h:78-103
template <class R> struct ContactPair {
  ContactType type = ContactType::POINT_TRIANGLE;
  Index idx0 = -1, idx1 = -1, idx2 = -1, idx3 = -1;
  R gap = 0; V3<R> normal, witness_p, witness_q, barycentric;
  std::array<R, 4> weights{{0, 0, 0, 0}};
  int vertex_count = 0; int rigid_body_index = -1;
};

// rigid_body.cpp
template <class R> struct RigidBody {
  std::vector<V3<R>> local; std::vector<Triangle> tris;
  R mass = R(1); M3<R> I_body = M3<R>::identity(), I_body_inv = M3<R>::identity();
  V3<R> position; M3<R> rotation = M3<R>::identity(); V3<R> lin_vel, ang_vel, acc_force, acc_torque;

  void initialize(const std::vector<V3<R>>& verts, const std::vector<Triangle>& t, R density) {
    tris = t;
    if (verts.empty()) { local.clear(); mass = 0; I_body = M3<R>(); I_body_inv = M3<R>(); return; }
    V3<R> c; for (auto& v : verts) c += v; c = c / R(verts.size());
    local.resize(verts.size()); for (size_t i = 0; i < verts.size(); ++i) local[i] = verts[i] - c;
    position = c; rotation = M3<R>::identity(); lin_vel = V3<R>(); ang_vel = V3<R>();
    V3<R> lo(std::numeric_limits<R>::max(), std::numeric_limits<R>::max(), std::numeric_limits<R>::max()), hi = -lo;
    for (auto& v : local) { V3<R> w = v + position; for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], w[k]); hi[k] = std::max(hi[k], w[k]); } }
    V3<R> ext = hi - lo;
    R vol = std::max(ext.x, R(1e-6)) * std::max(ext.y, R(1e-6)) * std::max(ext.z, R(1e-6));
    mass = std::max(density * vol, R(1e-3));
    R x2 = ext.x * ext.x, y2 = ext.y * ext.y, z2 = ext.z * ext.z;
    I_body = M3<R>();
    I_body(0, 0) = (mass / R(12)) * (y2 + z2); I_body(1, 1) = (mass / R(12)) * (x2 + z2); I_body(2, 2) = (mass / R(12)) * (x2 + y2);
    for (int i = 0; i < 3; ++i) if (I_body(i, i) < R(1e-6)) I_body(i, i) = R(1e-6);
    I_body_inv = I_body.inverse();
    acc_force = V3<R>(); acc_torque = V3<R>();
  }
  std::vector<V3<R>> world_vertices() const { std::vector<V3<R>> o; o.reserve(local.size()); for (auto& v : local) o.push_back(position + rotation * v); return o; }
  M3<R> inertia_world_inv() const { return rotation * I_body_inv * rotation.transpose(); }
  V3<R> velocity_at_point(const V3<R>& p) const { return lin_vel + ang_vel.cross(p - position); }
  void apply_impulse(const V3<R>& p, const V3<R>& J) {
    if (mass <= R(0)) return;
    lin_vel += J / mass; ang_vel += inertia_world_inv() * ((p - position).cross(J));
  }
  void apply_force(const V3<R>& p, const V3<R>& F, R dt) {
    if (mass <= R(0)) return;
    acc_force += F; acc_torque += (p - position).cross(F);
    if (dt > R(0)) {
      lin_vel += (F * dt) / mass; ang_vel += inertia_world_inv() * (acc_torque * dt);
      acc_force = V3<R>(); acc_torque = V3<R>();
    }
  }
  // rigid_body.cpp:151-176: semi-implicit Euler, rotation by the axis-angle (Rodrigues) matrix.
  void integrate(R dt) {
    if (mass <= R(0)) return;
    lin_vel += (acc_force / mass) * dt;
    ang_vel += (inertia_world_inv() * acc_torque) * dt;
    position += lin_vel * dt;
    R wn = ang_vel.norm();
    if (wn > R(1e-8)) {
      R th = wn * dt; V3<R> a = ang_vel / wn;
      R c = std::cos(th), s = std::sin(th), t = R(1) - c;
      M3<R> dR;
      dR(0, 0) = t * a.x * a.x + c;       dR(0, 1) = t * a.x * a.y - s * a.z; dR(0, 2) = t * a.x * a.z + s * a.y;
      dR(1, 0) = t * a.x * a.y + s * a.z; dR(1, 1) = t * a.y * a.y + c;       dR(1, 2) = t * a.y * a.z - s * a.x;
      dR(2, 0) = t * a.x * a.z - s * a.y; dR(2, 1) = t * a.y * a.z + s * a.x; dR(2, 2) = t * a.z * a.z + c;
      rotation = dR * rotation;
    }
    acc_force = V3<R>(); acc_torque = V3<R>();
  }
};

// ------------------------------------------------------------ sparse matrix
template <class R> struct Triplet { Index row, col; R value; };

// Row-major CSR with sorted columns. from_triplets sums duplicates in
// insertion order (Eigen::SparseMatrix::setFromTriplets semantics).
template <class R> struct Csr {
  Index n = 0;
  std::vector<Index> rowptr, cols;
  std::vector<R> vals;
  static Csr from_triplets(Index n, const std::vector<Triplet<R>>& t) {
    Csr A; A.n = n; A.rowptr.assign(n + 1, 0);
    std::vector<Index> cnt(n + 1, 0);
    for (auto& e : t) cnt[e.row + 1]++;
    for (Index i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    std::vector<Index> order(t.size()); std::vector<Index> pos(cnt.begin(), cnt.end() - 1);
    for (size_t k = 0; k < t.size(); ++k) order[pos[t[k].row]++] = Index(k);
    for (Index r = 0; r < n; ++r) {
      auto b = order.begin() + cnt[r], e = order.begin() + cnt[r + 1];
      std::stable_sort(b, e, [&](Index a, Index c) { return t[a].col < t[c].col; });
      for (auto it = b; it != e;) {
        Index c = t[*it].col; R v = t[*it].value; ++it;
        while (it != e && t[*it].col == c) { v = v + t[*it].value; ++it; }
        A.cols.push_back(c); A.vals.push_back(v);
      }
      A.rowptr[r + 1] = Index(A.cols.size());
    }
    return A;
  }
  R at(Index r, Index c) const {
    auto b = cols.begin() + rowptr[r], e = cols.begin() + rowptr[r + 1];
    auto it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? vals[it - cols.begin()] : R(0);
  }
  bool has(Index r, Index c) const {
    auto b = cols.begin() + rowptr[r], e = cols.begin() + rowptr[r + 1];
    auto it = std::lower_bound(b, e, c); return it != e && *it == c;
  }
  // (H + H^T) * 0.5 over the union pattern (integrator.cpp:541-543).
  Csr symmetrized() const {
    std::vector<Triplet<R>> t;
    for (Index r = 0; r < n; ++r) for (Index k = rowptr[r]; k < rowptr[r + 1]; ++k) t.push_back({r, cols[k], vals[k]});
    std::vector<Triplet<R>> tt; tt.reserve(t.size());
    for (auto& e : t) tt.push_back({e.col, e.row, e.value});
    Csr T = from_triplets(n, tt);
    Csr S; S.n = n; S.rowptr.assign(n + 1, 0);
    for (Index r = 0; r < n; ++r) {
      Index a = rowptr[r], ae = rowptr[r + 1], b = T.rowptr[r], be = T.rowptr[r + 1];
      while (a < ae || b < be) {
        Index ca = a < ae ? cols[a] : std::numeric_limits<Index>::max();
        Index cb = b < be ? T.cols[b] : std::numeric_limits<Index>::max();
        R v; Index c;
        if (ca == cb) { v = vals[a] + T.vals[b]; c = ca; ++a; ++b; }
        else if (ca < cb) { v = vals[a]; c = ca; ++a; }
        else { v = T.vals[b]; c = cb; ++b; }
        S.cols.push_back(c); S.vals.push_back(R(v * R(0.5)));
      }
      S.rowptr[r + 1] = Index(S.cols.size());
    }
    return S;
  }
  void multiply(const std::vector<R>& x, std::vector<R>& y) const {
    y.assign(n, R(0));
    // rows on the host's cores; each row sums in the same order
    parallel_for(n, [&](long long r) { R s = 0; for (Index k = rowptr[r]; k < rowptr[r + 1]; ++k) s += vals[k] * x[cols[k]]; y[size_t(r)] = s; });
  }
  size_t nnz() const { return vals.size(); }
};

// Stiffness::extract_hessian_block (stiffness.cpp:213-234). LITERAL scans every
// stored entry of the matrix; INDEXED reads the three rows directly.
template <class R> M3<R> extract_hessian_block(const Csr<R>& H, Index v, Lookup lk) {
  M3<R> b; Index base = v * 3;
  if (lk == Lookup::LITERAL) {
    for (Index r = 0; r < H.n; ++r)
      for (Index k = H.rowptr[r]; k < H.rowptr[r + 1]; ++k) {
        Index c = H.cols[k];
        if (r >= base && r < base + 3 && c >= base && c < base + 3) b(r - base, c - base) = H.vals[k];
      }
  } else {
    for (int i = 0; i < 3; ++i)
      for (Index k = H.rowptr[base + i]; k < H.rowptr[base + i + 1]; ++k) {
        Index c = H.cols[k]; if (c >= base && c < base + 3) b(i, c - base) = H.vals[k];
      }
  }
  return b;
}

// extract_submatrix (stiffness.cpp:13-49): sums entries whose row and column
// vertex are both in `verts`, mapped to the LAST list position of the vertex.
template <class R> std::vector<R> extract_submatrix(const Csr<R>& H, const std::vector<Index>& verts, Lookup lk) {
  int nb = int(verts.size());
  std::vector<R> sub(size_t(9 * nb * nb), R(0));
  std::unordered_map<Index, int> map;
  for (int i = 0; i < nb; ++i) map[verts[i]] = i;
  auto add = [&](Index r, Index c, R val) {
    auto ri = map.find(r / 3); if (ri == map.end()) return;
    auto ci = map.find(c / 3); if (ci == map.end()) return;
    sub[size_t((ri->second * 3 + r % 3) * 3 * nb + ci->second * 3 + c % 3)] += val;
  };
  if (lk == Lookup::LITERAL) {
    for (Index r = 0; r < H.n; ++r) for (Index k = H.rowptr[r]; k < H.rowptr[r + 1]; ++k) add(r, H.cols[k], H.vals[k]);
  } else {
    std::vector<Index> uniq;
    for (auto& kv : map) uniq.push_back(kv.first);
    std::sort(uniq.begin(), uniq.end());
    for (Index vr : uniq) for (int i = 0; i < 3; ++i) { Index r = vr * 3 + i; if (r >= H.n) continue;
      for (Index k = H.rowptr[r]; k < H.rowptr[r + 1]; ++k) add(r, H.cols[k], H.vals[k]); }
  }
  return sub;
}

// --------------------------------------------------------------- stiffness
// Stiffness::enforce_spd (stiffness.cpp:236-254)
template <class R> M3<R> enforce_spd(const M3<R>& H, R eps = R(1e-8)) {
  M3<R> S = (H + H.transpose()) * R(0.5);
  V3<R> ev; M3<R> Q; sym_eigen3(S, ev, Q);
  for (int i = 0; i < 3; ++i) if (ev[i] < eps) ev[i] = eps;
  M3<R> L; L(0, 0) = ev[0]; L(1, 1) = ev[1]; L(2, 2) = ev[2];
  return Q * L * Q.transpose();
}

// Stiffness::compute_contact_stiffness (stiffness.cpp:53-116)
template <class R> R contact_stiffness(const ContactPair<R>& c, const std::vector<R>& masses, R dt, const Csr<R>& H_el, Lookup lk) {
  if (dt <= R(0)) return R(0);
  V3<R> n = c.normal; R nn = n.norm();
  if (nn < R(1e-12)) return R(0);
  n = n / nn;
  Index ids[4] = {c.idx0, c.idx1, c.idx2, c.idx3};
  int cnt = std::max(c.vertex_count, 1);
  std::vector<Index> vv; std::vector<R> ww;
  for (int i = 0; i < cnt; ++i) {
    if (ids[i] < 0 || size_t(ids[i]) >= masses.size()) continue;
    if (c.weights[i] == R(0)) continue;
    vv.push_back(ids[i]); ww.push_back(c.weights[i]);
  }
  if (vv.empty()) return R(0);
  R inertial = 0;
  for (size_t i = 0; i < vv.size(); ++i) inertial += masses[vv[i]] * ww[i] * ww[i];
  inertial /= (dt * dt);
  int nb = int(vv.size());
  std::vector<R> Wn(size_t(3 * nb));
  for (int i = 0; i < nb; ++i) for (int k = 0; k < 3; ++k) Wn[size_t(3 * i + k)] = ww[i] * n[k];
  auto sub = extract_submatrix(H_el, vv, lk);
  R el = 0;
  for (int r = 0; r < 3 * nb; ++r) { R hr = 0; for (int q = 0; q < 3 * nb; ++q) hr += sub[size_t(r * 3 * nb + q)] * Wn[size_t(q)]; el += Wn[size_t(r)] * hr; }
  if (el < R(0)) el = R(0);
  return inertial + el;
}

// Stiffness::compute_pin_stiffness (stiffness.cpp:118-144)
template <class R> R pin_stiffness(R mass, R dt, const V3<R>& offset, const M3<R>& Hb, R min_gap) {
  (void)dt;
  M3<R> H = enforce_spd(Hb);
  V3<R> d = offset; R len = d.norm();
  if (len > R(1e-9)) d = d / len; else d = V3<R>(1, 0, 0);
  R ke = std::max(R(0), d.dot(H * d));
  R gh = std::max(std::max(len, min_gap), R(1e-12));
  return mass / (gh * gh) + ke;
}

// Stiffness::compute_wall_stiffness (stiffness.cpp:146-172)
template <class R> R wall_stiffness(R mass, R wall_gap, const V3<R>& normal, const M3<R>& Hb, R min_gap) {
  R gh = std::max(std::max(wall_gap, min_gap), R(1e-12));
  R ki = mass / (gh * gh);
  M3<R> H = enforce_spd(Hb);
  V3<R> n = normal; R nn = n.norm();
  if (nn > R(1e-9)) n = n / nn; else n = V3<R>(0, 1, 0);
  return ki + std::max(R(0), n.dot(H * n));
}

// CORRECTED dynamic stiffness. The cubic barrier (k / 2 g_max)(g_max - g)^3
// (barrier.cpp:29-65) is finite at g = 0, so its force saturates at
// 1.5 k g_max: with the reference's contact stiffness sum(m w^2) / dt^2 +
// elastic (stiffness.cpp:53-116) a pair pressed harder than that closes to
// zero distance, where no time-of-impact line search can move it again. The
// reference's own pin (stiffness.cpp:118-144) and strain-limit
// (strain_limiting.cpp:113-193) stiffnesses take the inertial part as
// mass / g^2 at the current gap, which makes the force grow without bound as
// the gap closes; CORRECTED uses that form for contacts and walls as well.
// The elastic part is the reference's.
template <class R> R corrected_gap_scale(R gap, R min_gap) { return std::max(std::max(gap, min_gap), R(1e-12)); }
template <class R> R corrected_contact_stiffness(const ContactPair<R>& c, const std::vector<R>& masses, const Csr<R>& H_el, R min_gap) {
  // contact_stiffness divides sum(m w^2) by its `dt` argument squared
  return contact_stiffness(c, masses, corrected_gap_scale(c.gap, min_gap), H_el, Lookup::INDEXED);
}
template <class R> R corrected_wall_stiffness(R mass, R gap, const V3<R>& normal, const M3<R>& Hb, R min_gap) {
  return wall_stiffness(mass, corrected_gap_scale(gap, min_gap), normal, Hb, min_gap);
}
// CORRECTED pins attract: E = kappa / 2 |x - target|^2 inside the implicit
// solve, with kappa = 100 (m / dt^2 + a) where a is the vertex's elastic
// diagonal coefficient, so a pinned vertex follows its target within about
// 1 % of the elastic load on it while contacts can still push it aside
// (the reference's pins repel: barrier.cpp:161-215).
constexpr double kPinScale = 100.0;
template <class R> R corrected_pin_stiffness(R mass, R dt, R el_diag) { return R(kPinScale * (double(mass) / (double(dt) * double(dt)) + double(el_diag))); }

// ------------------------------------------------------------------ barrier
// barrier.cpp:29-65
template <class R> R barrier_energy(R g, R gm, R k) {
  if (gm <= R(0) || g >= gm) return R(0);
  R d = gm - g; if (d <= R(0)) return R(0);
  R inv = R(1) / gm; return R(0.5) * k * inv * d * d * d;
}
template <class R> R barrier_gradient(R g, R gm, R k) {
  if (gm <= R(0) || g >= gm) return R(0);
  R d = gm - g; R inv = R(1) / gm; return -R(1.5) * k * inv * d * d;
}
template <class R> R barrier_hessian(R g, R gm, R k) {
  if (gm <= R(0) || g >= gm) return R(0);
  R d = gm - g; R inv = R(1) / gm; return R(3) * k * inv * d;
}
template <class R> bool in_domain(R g, R gm) { return gm > R(0) && g <= gm; }
template <class R> V3<R> normalize_or_default(const V3<R>& n, R eps) { return n.sq() > eps * eps ? n.normalized() : V3<R>(0, 1, 0); }

// ------------------------------------------------------------------ elasticity
// elasticity.cpp:18-61 -- on mesh.vertices, not on the state.
template <class R> void elastic_gradient(const Mesh<R>& mesh, std::vector<R>& g) {
  g.assign(mesh.vertices.size() * 3, R(0));
  for (size_t i = 0; i < mesh.triangles.size(); ++i) {
    const auto& t = mesh.triangles[i];
    M2<R> F = mesh.compute_F(i);
    R mu = R(double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio))));
    R k = mesh.rest_areas[i] * mesh.material.thickness * mu;
    M2<R> FmI{F.a - R(1), F.b, F.c, F.d - R(1)};
    M2<R> P = FmI * R(2.0 * double(k));
    M2<R> H = P * mesh.Dm_inv[i].transpose();
    V3<R> e1 = mesh.vertices[t.v[1]] - mesh.vertices[t.v[0]], e2 = mesh.vertices[t.v[2]] - mesh.vertices[t.v[0]];
    V3<R> n = e1.cross(e2).normalized(), t1 = e1.normalized(), t2 = n.cross(t1);
    V3<R> f1 = t1 * H.a + t2 * H.c, f2 = t1 * H.b + t2 * H.d, f0 = -(f1 + f2);
    for (int k2 = 0; k2 < 3; ++k2) {
      g[size_t(t.v[0]) * 3 + k2] += f0[k2]; g[size_t(t.v[1]) * 3 + k2] += f1[k2]; g[size_t(t.v[2]) * 3 + k2] += f2[k2];
    }
  }
}

// elasticity.cpp:93-103
template <class R> R elastic_energy(const Mesh<R>& mesh) {
  R e = 0;
  for (size_t i = 0; i < mesh.triangles.size(); ++i) {
    M2<R> F = mesh.compute_F(i);
    R mu = R(double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio))));
    R k = mesh.rest_areas[i] * mesh.material.thickness * mu;
    R a = F.a - 1, b = F.b, c = F.c, d = F.d - 1;
    e += k * (a * a + b * b + c * c + d * d);
  }
  return e;
}

// Constant face Hessian blocks (elasticity.cpp:135-181), each SPD-clamped.
template <class R> void face_hessian_blocks(const Mesh<R>& mesh, size_t f, M3<R> H[3][3]) {
  R mu = R(double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio))));
  R k = mesh.rest_areas[f] * mesh.material.thickness * mu;
  M2<R> Di = mesh.Dm_inv[f];
  M2<R> K = (Di.transpose() * Di) * k;
  auto diag2 = [](R v) { M3<R> m; m(0, 0) = v; m(1, 1) = v; return m; };
  H[0][0] = diag2(R(K.a + K.d + R(2.0) * K.b));
  H[1][1] = diag2(K.a);
  H[2][2] = diag2(K.d);
  H[0][1] = diag2(-K.a); H[1][0] = H[0][1].transpose();
  H[0][2] = diag2(-K.d); H[2][0] = H[0][2].transpose();
  H[1][2] = diag2(-K.b); H[2][1] = H[1][2].transpose();
}

// Elasticity::compute_hessian (elasticity.cpp:63-91): 81 triplets per face.
template <class R> void elastic_hessian_triplets(const Mesh<R>& mesh, std::vector<Triplet<R>>& out) {
  for (size_t f = 0; f < mesh.triangles.size(); ++f) {
    const auto& t = mesh.triangles[f];
    M3<R> H[3][3]; face_hessian_blocks(mesh, f, H);
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
      M3<R> S = enforce_spd(H[a][b]);
      for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) out.push_back({t.v[a] * 3 + r, t.v[b] * 3 + c, S(r, c)});
    }
  }
}

// ------------------------------------------------------------ strain limiting
template <class R> struct Svd32 { V3<R> U[2]; R sigma[2]; R V[2][2]; };  // V[row][col]

// Thin SVD of a 3x2 matrix through the eigen-decomposition of F^T F.
template <class R> bool svd32(const V3<R> F[2], Svd32<R>& s) {
  double c0[3] = {double(F[0].x), double(F[0].y), double(F[0].z)}, c1[3] = {double(F[1].x), double(F[1].y), double(F[1].z)};
  double a = c0[0] * c0[0] + c0[1] * c0[1] + c0[2] * c0[2];
  double b = c0[0] * c1[0] + c0[1] * c1[1] + c0[2] * c1[2];
  double d = c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2];
  double tr = a + d, diff = a - d, disc = std::sqrt(diff * diff + 4.0 * b * b);
  double l0 = 0.5 * (tr + disc), l1 = 0.5 * (tr - disc);
  if (l1 < 0) l1 = 0;
  double v0x, v0y;
  if (b == 0.0) { if (a >= d) { v0x = 1; v0y = 0; } else { v0x = 0; v0y = 1; } }
  else { v0x = l0 - d; v0y = b; double nr = std::sqrt(v0x * v0x + v0y * v0y); v0x /= nr; v0y /= nr; }
  double v1x = -v0y, v1y = v0x;
  double s0 = std::sqrt(l0), s1 = std::sqrt(l1);
  s.V[0][0] = R(v0x); s.V[1][0] = R(v0y); s.V[0][1] = R(v1x); s.V[1][1] = R(v1y);
  s.sigma[0] = R(s0); s.sigma[1] = R(s1);
  double u0[3], u1[3];
  for (int k = 0; k < 3; ++k) { u0[k] = c0[k] * v0x + c1[k] * v0y; u1[k] = c0[k] * v1x + c1[k] * v1y; }
  if (s0 > 0) for (int k = 0; k < 3; ++k) u0[k] /= s0;
  if (s1 > 1e-300) for (int k = 0; k < 3; ++k) u1[k] /= s1;
  else {  // complete an orthonormal pair
    double t[3] = {0, 0, 0}; int ax = std::fabs(u0[0]) < 0.57 ? 0 : (std::fabs(u0[1]) < 0.57 ? 1 : 2); t[ax] = 1;
    double cx = u0[1] * t[2] - u0[2] * t[1], cy = u0[2] * t[0] - u0[0] * t[2], cz = u0[0] * t[1] - u0[1] * t[0];
    double nr = std::sqrt(cx * cx + cy * cy + cz * cz); u1[0] = cx / nr; u1[1] = cy / nr; u1[2] = cz / nr;
  }
  s.U[0] = V3<R>(R(u0[0]), R(u0[1]), R(u0[2])); s.U[1] = V3<R>(R(u1[0]), R(u1[1]), R(u1[2]));
  const R thr = R(1e-6);  // strain_limiting.h:57 kDegenerateThreshold
  if (s.sigma[0] < thr || s.sigma[1] < thr) { s.sigma[0] = std::max(s.sigma[0], thr); s.sigma[1] = std::max(s.sigma[1], thr); }
  return std::isfinite(double(s.sigma[0])) && std::isfinite(double(s.sigma[1]));
}

template <class R> R to_fraction(R v) { return v > R(1) ? v * R(0.01) : v; }

template <class R> void strain_F(const State<R>& st, const Mesh<R>& mesh, size_t f, V3<R> F[2]) {
  const auto& t = mesh.triangles[f];
  V3<R> e1 = st.positions[t.v[1]] - st.positions[t.v[0]], e2 = st.positions[t.v[2]] - st.positions[t.v[0]];
  const M2<R>& D = mesh.Dm_inv[f];
  F[0] = e1 * D.a + e2 * D.c; F[1] = e1 * D.b + e2 * D.d;
}

// StrainLimiting::rebuild_constraints (strain_limiting.cpp:113-193)
template <class R> void strain_rebuild(const Mesh<R>& mesh, const State<R>& st, const SimParams<R>& p, const Csr<R>& H_el, Constraints<R>& C, Lookup lk) {
  C.strain_limits.clear();
  if (!p.enable_strain_limiting) return;
  R tau = to_fraction(p.strain_tau);
  R eps = p.strain_epsilon > R(0) ? to_fraction(p.strain_epsilon) : tau;
  if (eps <= R(0)) return;
  R min_gap = std::max(p.min_gap, R(1e-8));
  for (size_t f = 0; f < mesh.triangles.size(); ++f) {
    if (mesh.rest_areas[f] <= R(1e-12)) continue;
    V3<R> F[2]; strain_F(st, mesh, f, F);
    Svd32<R> s; if (!svd32(F, s)) continue;
    const auto& t = mesh.triangles[f];
    R fm = mesh.rest_areas[f] * mesh.material.thickness * mesh.material.density;
    V3<R> x0 = st.positions[t.v[0]], x1 = st.positions[t.v[1]], x2 = st.positions[t.v[2]];
    V3<R> cen = (x0 + x1 + x2) / R(3);
    V3<R> w[3] = {x0 - cen, x1 - cen, x2 - cen};
    // 9x9 face block of H_el (last-match local index, strain_limiting.cpp:61-93)
    R Hf[9][9] = {};
    auto lidx = [&](Index gv) { int l = -1; for (int i = 0; i < 3; ++i) if (t.v[i] == gv) l = i; return l; };
    auto visit = [&](Index r, Index k) {
      int lr = lidx(r / 3), lc = lidx(H_el.cols[k] / 3);
      if (lr < 0 || lc < 0) return;
      Hf[lr * 3 + r % 3][lc * 3 + H_el.cols[k] % 3] += H_el.vals[k];
    };
    if (lk == Lookup::LITERAL) { for (Index r = 0; r < H_el.n; ++r) for (Index k = H_el.rowptr[r]; k < H_el.rowptr[r + 1]; ++k) visit(r, k); }
    else {
      std::vector<Index> uv = {t.v[0], t.v[1], t.v[2]}; std::sort(uv.begin(), uv.end()); uv.erase(std::unique(uv.begin(), uv.end()), uv.end());
      for (Index gv : uv) for (int i = 0; i < 3; ++i) { Index r = gv * 3 + i; for (Index k = H_el.rowptr[r]; k < H_el.rowptr[r + 1]; ++k) visit(r, k); }
    }
    R el = 0;
    for (int r = 0; r < 9; ++r) { R hr = 0; for (int c = 0; c < 9; ++c) hr += (Hf[r][c] + Hf[c][r]) * R(0.5) * w[c / 3][c % 3]; el += w[r / 3][r % 3] * hr; }
    el = std::max(el, R(0));
    for (int si = 0; si < 2; ++si) {
      R gap = (R(1) + tau + eps) - s.sigma[si];
      if (!in_domain(gap, eps)) continue;
      R gc = std::max(std::fabs(gap), min_gap);
      StrainConstraint<R> sc; sc.face_idx = Index(f); sc.sigma = s.sigma[si]; sc.singular_index = si;
      sc.stiffness = fm / (gc * gc) + el;
      C.strain_limits.push_back(sc);
    }
  }
}

// dsigma/dx for a constraint (strain_limiting.cpp:224-245, 300-317). Returns
// false when the SVD fails. J = [dsig/dx0, dsig/dx1, dsig/dx2].
template <class R> bool strain_jacobian(const Mesh<R>& mesh, const State<R>& st, const SimParams<R>& p, size_t f, int idx, R& sigma_idx, V3<R> J[3]) {
  V3<R> F[2]; strain_F(st, mesh, f, F);
  Svd32<R> s; if (!svd32(F, s)) return false;
  R svd_eps = std::max(p.strain_svd_epsilon, R(1e-8));
  V3<R> dS[2];  // columns of the 3x2 dsigma/dF
  if (std::fabs(s.sigma[0] - s.sigma[1]) < svd_eps) {
    for (int c = 0; c < 2; ++c) dS[c] = (s.U[0] * s.V[c][0] + s.U[1] * s.V[c][1]) * R(0.5);
  } else {
    for (int c = 0; c < 2; ++c) dS[c] = s.U[idx] * s.V[c][idx];
  }
  const M2<R>& D = mesh.Dm_inv[f];
  // (3x2) * Dm_inv^T
  J[1] = dS[0] * D.a + dS[1] * D.b;
  J[2] = dS[0] * D.c + dS[1] * D.d;
  J[0] = -(J[1] + J[2]);
  sigma_idx = s.sigma[idx];
  return true;
}

template <class R> void strain_gradient(const Mesh<R>& mesh, const State<R>& st, const Constraints<R>& C, const SimParams<R>& p, std::vector<R>& g) {
  if (!p.enable_strain_limiting || C.strain_limits.empty()) return;
  R tau = to_fraction(p.strain_tau);
  R eps = p.strain_epsilon > R(0) ? to_fraction(p.strain_epsilon) : tau;
  for (const auto& sc : C.strain_limits) {
    if (!sc.active || sc.face_idx < 0 || size_t(sc.face_idx) >= mesh.triangles.size()) continue;
    int idx = std::clamp(sc.singular_index, 0, 1);
    R sig; V3<R> J[3];
    if (!strain_jacobian(mesh, st, p, size_t(sc.face_idx), idx, sig, J)) continue;
    R gap = (R(1) + tau + eps) - sig;
    if (!in_domain(gap, eps)) continue;
    R dV = barrier_gradient(gap, eps, sc.stiffness);
    if (std::fabs(dV) < R(1e-12)) continue;
    // dPsi/dF = -dV * dsig/dF  ->  mapped = dPsi/dF * Dm_inv^T = -dV * J
    const auto& t = mesh.triangles[size_t(sc.face_idx)];
    V3<R> g1 = J[1] * (-dV), g2 = J[2] * (-dV), g0 = -(g1 + g2);
    for (int k = 0; k < 3; ++k) { g[size_t(t.v[0]) * 3 + k] += g0[k]; g[size_t(t.v[1]) * 3 + k] += g1[k]; g[size_t(t.v[2]) * 3 + k] += g2[k]; }
  }
}

template <class R> void strain_hessian(const Mesh<R>& mesh, const State<R>& st, const Constraints<R>& C, const SimParams<R>& p, std::vector<Triplet<R>>& out) {
  if (!p.enable_strain_limiting || C.strain_limits.empty()) return;
  R tau = to_fraction(p.strain_tau);
  R eps = p.strain_epsilon > R(0) ? to_fraction(p.strain_epsilon) : tau;
  for (const auto& sc : C.strain_limits) {
    if (!sc.active || sc.face_idx < 0 || size_t(sc.face_idx) >= mesh.triangles.size()) continue;
    int idx = std::clamp(sc.singular_index, 0, 1);
    R sig; V3<R> J[3];
    if (!strain_jacobian(mesh, st, p, size_t(sc.face_idx), idx, sig, J)) continue;
    R gap = (R(1) + tau + eps) - sig;
    if (!in_domain(gap, eps)) continue;
    R d2V = barrier_hessian(gap, eps, sc.stiffness);
    if (std::fabs(d2V) < R(1e-12)) continue;
    const auto& t = mesh.triangles[size_t(sc.face_idx)];
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) {
      R blk[3][3]; R mx = 0;
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) { blk[i][j] = d2V * (J[a][i] * J[b][j]); mx = std::max(mx, std::fabs(blk[i][j])); }
      if (mx < R(1e-12)) continue;
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) {
        if (std::fabs(blk[i][j]) < R(1e-12)) continue;
        out.push_back({t.v[a] * 3 + i, t.v[b] * 3 + j, blk[i][j]});
      }
    }
  }
}

// ---------------------------------------------------------------- collision
template <class R> struct AABB {
  V3<R> lo{std::numeric_limits<R>::max(), std::numeric_limits<R>::max(), std::numeric_limits<R>::max()};
  V3<R> hi{-std::numeric_limits<R>::max(), -std::numeric_limits<R>::max(), -std::numeric_limits<R>::max()};
  void expand(const V3<R>& p) { for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); } }
  void expand(const AABB& o) { for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], o.lo[k]); hi[k] = std::max(hi[k], o.hi[k]); } }
  // collision.h:37-41 (inclusive on every axis)
  bool overlaps(const AABB& o) const {
    return lo[0] <= o.hi[0] && hi[0] >= o.lo[0] && lo[1] <= o.hi[1] && hi[1] >= o.lo[1] && lo[2] <= o.hi[2] && hi[2] >= o.lo[2];
  }
  V3<R> center() const { return (lo + hi) * R(0.5); }
  int longest_axis() const { V3<R> e = hi - lo; if (e[0] > e[1] && e[0] > e[2]) return 0; if (e[1] > e[2]) return 1; return 2; }
};

struct BVHNode { int left = -1, right = -1, prim = -1; bool is_leaf() const { return prim >= 0; } };
template <class R> struct BVH { std::vector<BVHNode> nodes; std::vector<AABB<R>> boxes; };

// collision.cpp:65-105, leaf defect included.
template <class R> int bvh_build_rec(BVH<R>& b, const std::vector<AABB<R>>& pb, std::vector<int>& idx, int s, int e) {
  int ni = int(b.nodes.size());
  b.nodes.emplace_back(); b.boxes.emplace_back();
  AABB<R> box; for (int i = s; i < e; ++i) box.expand(pb[size_t(idx[size_t(i)])]);
  b.boxes[size_t(ni)] = box;
  int np = e - s;
  if (np <= 4) { if (np == 1) b.nodes[size_t(ni)].prim = idx[size_t(s)]; return ni; }
  int ax = box.longest_axis();
  std::sort(idx.begin() + s, idx.begin() + e, [&](int a, int c) { return pb[size_t(a)].center()[ax] < pb[size_t(c)].center()[ax]; });
  int mid = s + np / 2;
  int l = bvh_build_rec(b, pb, idx, s, mid);
  int r = bvh_build_rec(b, pb, idx, mid, e);
  b.nodes[size_t(ni)].left = l; b.nodes[size_t(ni)].right = r;
  return ni;
}
template <class R> BVH<R> bvh_build(const std::vector<AABB<R>>& pb) {
  BVH<R> b; if (pb.empty()) return b;
  std::vector<int> idx(pb.size()); for (size_t i = 0; i < idx.size(); ++i) idx[i] = int(i);
  bvh_build_rec(b, pb, idx, 0, int(idx.size()));
  return b;
}

template <class R> std::vector<AABB<R>> triangle_boxes(const Mesh<R>& m, const std::vector<V3<R>>& x) {
  std::vector<AABB<R>> b(m.triangles.size());
  for (size_t i = 0; i < m.triangles.size(); ++i) for (int k = 0; k < 3; ++k) b[i].expand(x[size_t(m.triangles[i].v[k])]);
  return b;
}
template <class R> std::vector<AABB<R>> edge_boxes(const Mesh<R>& m, const std::vector<V3<R>>& x) {
  std::vector<AABB<R>> b(m.edges.size());
  for (size_t i = 0; i < m.edges.size(); ++i) { b[i].expand(x[size_t(m.edges[i].v[0])]); b[i].expand(x[size_t(m.edges[i].v[1])]); }
  return b;
}
template <class R> AABB<R> point_box(const V3<R>& p) {
  const R e = R(1e-4); AABB<R> b; b.lo = p - V3<R>(e, e, e); b.hi = p + V3<R>(e, e, e); return b;
}

// Candidate vertex-triangle pairs (v, t) and edge-edge pairs (e1 < e2).
// `pad` inflates every box (triangle, edge and point) in the INTENDED mode;
// the LITERAL mode is the reference's query and ignores it.
template <class R> void inflate(AABB<R>& b, R pad) { for (int k = 0; k < 3; ++k) { b.lo[k] = b.lo[k] - pad; b.hi[k] = b.hi[k] + pad; } }

template <class R> void broad_phase(const Mesh<R>& m, const std::vector<V3<R>>& x, BroadPhase mode,
                                    std::vector<std::pair<int, int>>& vt, std::vector<std::pair<int, int>>& ee, R pad = R(0)) {
  vt.clear(); ee.clear();
  auto tb = triangle_boxes(m, x);
  auto eb = edge_boxes(m, x);
  if (mode == BroadPhase::INTENDED && pad > R(0)) { for (auto& b : tb) inflate(b, pad); for (auto& b : eb) inflate(b, pad); }
  if (mode == BroadPhase::LITERAL) {
    BVH<R> tbvh = bvh_build(tb), ebvh = bvh_build(eb);
    if (!tbvh.nodes.empty()) {
      for (size_t v = 0; v < x.size(); ++v) {  // collision.cpp:198-244
        AABB<R> pbx = point_box(x[v]);
        std::function<void(int)> trav = [&](int ni) {
          if (ni < 0 || ni >= int(tbvh.nodes.size())) return;
          if (!pbx.overlaps(tbvh.boxes[size_t(ni)])) return;
          const BVHNode& nd = tbvh.nodes[size_t(ni)];
          if (nd.is_leaf()) {
            const auto& t = m.triangles[size_t(nd.prim)];
            if (t.v[0] == int(v) || t.v[1] == int(v) || t.v[2] == int(v)) return;
            vt.push_back({int(v), nd.prim});
          } else { trav(nd.left); trav(nd.right); }
        };
        trav(0);
      }
    }
    if (!ebvh.nodes.empty()) {  // collision.cpp:162-195, 247-276
      std::vector<std::pair<int, int>> ov;
      std::function<void(int, int)> pair = [&](int a, int b) {
        if (a < 0 || b < 0) return;
        if (!ebvh.boxes[size_t(a)].overlaps(ebvh.boxes[size_t(b)])) return;
        const BVHNode &na = ebvh.nodes[size_t(a)], &nb = ebvh.nodes[size_t(b)];
        if (na.is_leaf() && nb.is_leaf()) { ov.push_back({na.prim, nb.prim}); return; }
        if (na.is_leaf()) { pair(a, nb.left); pair(a, nb.right); }
        else if (nb.is_leaf()) { pair(na.left, b); pair(na.right, b); }
        else { pair(na.left, nb.left); pair(na.left, nb.right); pair(na.right, nb.left); pair(na.right, nb.right); }
      };
      pair(0, 0);
      for (auto& pr : ov) {
        if (pr.first >= pr.second) continue;
        const Edge &e1 = m.edges[size_t(pr.first)], &e2 = m.edges[size_t(pr.second)];
        if (e1.v[0] == e2.v[0] || e1.v[0] == e2.v[1] || e1.v[1] == e2.v[0] || e1.v[1] == e2.v[1]) continue;
        ee.push_back(pr);
      }
    }
  } else {
    for (size_t v = 0; v < x.size(); ++v) {
      AABB<R> pbx = point_box(x[v]);
      if (pad > R(0)) inflate(pbx, pad);
      for (size_t t = 0; t < tb.size(); ++t) {
        if (!pbx.overlaps(tb[t])) continue;
        const auto& tri = m.triangles[t];
        if (tri.v[0] == int(v) || tri.v[1] == int(v) || tri.v[2] == int(v)) continue;
        vt.push_back({int(v), int(t)});
      }
    }
    for (size_t a = 0; a < eb.size(); ++a)
      for (size_t b = a + 1; b < eb.size(); ++b) {
        if (!eb[a].overlaps(eb[b])) continue;
        const Edge &e1 = m.edges[a], &e2 = m.edges[b];
        if (e1.v[0] == e2.v[0] || e1.v[0] == e2.v[1] || e1.v[1] == e2.v[0] || e1.v[1] == e2.v[1]) continue;
        ee.push_back({int(a), int(b)});
      }
  }
}

// collision.cpp:279-386 (closest point by Voronoi region)
template <class R> void narrow_pt(const V3<R>& p, const V3<R>& a, const V3<R>& b, const V3<R>& c, R& dist, V3<R>& normal, V3<R>& wp, V3<R>& wq) {
  V3<R> ab = b - a, ac = c - a, ap = p - a;
  R d1 = ab.dot(ap), d2 = ac.dot(ap);
  auto finish_vertex = [&](const V3<R>& q) { wq = q; wp = p; V3<R> df = p - q; dist = df.norm(); normal = dist > R(1e-10) ? df / dist : V3<R>(0, 0, 1); };
  if (d1 <= R(0) && d2 <= R(0)) { finish_vertex(a); return; }
  V3<R> bp = p - b; R d3 = ab.dot(bp), d4 = ac.dot(bp);
  if (d3 >= R(0) && d4 <= d3) { finish_vertex(b); return; }
  V3<R> cp = p - c; R d5 = ab.dot(cp), d6 = ac.dot(cp);
  if (d6 >= R(0) && d5 <= d6) { finish_vertex(c); return; }
  R vc = d1 * d4 - d3 * d2;
  if (vc <= R(0) && d1 >= R(0) && d3 <= R(0)) { R v = d1 / (d1 - d3); finish_vertex(a + ab * v); return; }
  R vb = d5 * d2 - d1 * d6;
  if (vb <= R(0) && d2 >= R(0) && d6 <= R(0)) { R w = d2 / (d2 - d6); finish_vertex(a + ac * w); return; }
  R va = d3 * d6 - d5 * d4;
  if (va <= R(0) && (d4 - d3) >= R(0) && (d5 - d6) >= R(0)) { R w = (d4 - d3) / ((d4 - d3) + (d5 - d6)); finish_vertex(b + (c - b) * w); return; }
  R den = R(1.0) / (va + vb + vc);
  R v = vb * den, w = vc * den;
  wq = a + ab * v + ac * w; wp = p;
  V3<R> df = p - wq; dist = df.norm();
  V3<R> tn = ab.cross(ac); R ta = tn.norm();
  if (ta > R(1e-10)) { tn = tn / ta; if (tn.dot(df) < R(0)) tn = -tn; normal = tn; }
  else normal = dist > R(1e-10) ? df / dist : V3<R>(0, 0, 1);
}

// collision.cpp:389-452 (clamped segment-segment closest points)
template <class R> void narrow_ee(const V3<R>& p0, const V3<R>& p1, const V3<R>& q0, const V3<R>& q1, R& dist, V3<R>& normal, V3<R>& wp, V3<R>& wq,
                                  R* s_out = nullptr, R* t_out = nullptr) {
  V3<R> d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  R a = d1.dot(d1), e = d2.dot(d2), f = d2.dot(r);
  R s, t; const R eps = R(1e-10);
  auto cl = [](R v) { return std::clamp(v, R(0), R(1)); };
  if (a <= eps && e <= eps) { s = t = 0; wp = p0; wq = q0; }
  else {
    if (a <= eps) { s = 0; t = cl(f / e); }
    else {
      R c = d1.dot(r);
      if (e <= eps) { t = 0; s = cl(-c / a); }
      else {
        R b = d1.dot(d2); R den = a * e - b * b;
        s = den != R(0) ? cl((b * f - c * e) / den) : R(0);
        t = (b * s + f) / e;
        if (t < R(0)) { t = 0; s = cl(-c / a); }
        else if (t > R(1)) { t = 1; s = cl((b - c) / a); }
      }
    }
    wp = p0 + d1 * s; wq = q0 + d2 * t;
  }
  V3<R> df = wp - wq; dist = df.norm(); normal = dist > R(1e-10) ? df / dist : V3<R>(0, 0, 1);
  if (s_out) *s_out = s;
  if (t_out) *t_out = t;
}

// collision.cpp:11-43
template <class R> V3<R> triangle_barycentric(const V3<R>& p, const V3<R>& a, const V3<R>& b, const V3<R>& c) {
  V3<R> v0 = b - a, v1 = c - a, v2 = p - a;
  R d00 = v0.dot(v0), d01 = v0.dot(v1), d11 = v1.dot(v1), d20 = v2.dot(v0), d21 = v2.dot(v1);
  R den = d00 * d11 - d01 * d01; R v = 0, w = 0;
  if (std::fabs(den) > std::numeric_limits<R>::epsilon()) { v = (d11 * d20 - d01 * d21) / den; w = (d00 * d21 - d01 * d20) / den; }
  v = std::clamp(v, R(0), R(1)); w = std::clamp(w, R(0), R(1));
  if (v + w > R(1)) { R sm = v + w; if (sm > std::numeric_limits<R>::epsilon()) { v /= sm; w /= sm; } }
  return V3<R>(R(1) - v - w, v, w);
}

// Collision::detect_all_collisions (collision.cpp:478-580)
template <class R> std::vector<ContactPair<R>> detect_all(const Mesh<R>& m, const State<R>& st, const std::vector<RigidBody<R>>* rigids, BroadPhase mode) {
  std::vector<ContactPair<R>> out;
  std::vector<std::pair<int, int>> vt, ee;
  broad_phase(m, st.positions, mode, vt, ee);
  for (auto& pr : vt) {
    ContactPair<R> c; c.type = ContactType::POINT_TRIANGLE; c.idx0 = pr.first;
    const auto& t = m.triangles[size_t(pr.second)]; c.idx1 = t.v[0]; c.idx2 = t.v[1]; c.idx3 = t.v[2];
    const auto &p = st.positions[size_t(c.idx0)], &a = st.positions[size_t(c.idx1)], &b = st.positions[size_t(c.idx2)], &cc = st.positions[size_t(c.idx3)];
    narrow_pt(p, a, b, cc, c.gap, c.normal, c.witness_p, c.witness_q);
    if (c.gap < R(0.01)) {
      V3<R> bc = triangle_barycentric(c.witness_q, a, b, cc); c.barycentric = bc;
      c.weights = {R(1), -bc[0], -bc[1], -bc[2]}; c.vertex_count = 4; out.push_back(c);
    }
  }
  for (auto& pr : ee) {
    ContactPair<R> c; c.type = ContactType::EDGE_EDGE;
    const Edge &e1 = m.edges[size_t(pr.first)], &e2 = m.edges[size_t(pr.second)];
    c.idx0 = e1.v[0]; c.idx1 = e1.v[1]; c.idx2 = e2.v[0]; c.idx3 = e2.v[1];
    narrow_ee(st.positions[size_t(c.idx0)], st.positions[size_t(c.idx1)], st.positions[size_t(c.idx2)], st.positions[size_t(c.idx3)], c.gap, c.normal, c.witness_p, c.witness_q);
    if (c.gap < R(0.01)) { c.vertex_count = 4; c.weights = {R(0.5), R(0.5), R(-0.5), R(-0.5)}; out.push_back(c); }
  }
  if (rigids) {
    for (size_t rb = 0; rb < rigids->size(); ++rb) {
      const auto& body = (*rigids)[rb];
      auto wv = body.world_vertices();
      for (size_t v = 0; v < st.positions.size(); ++v)
        for (const auto& t : body.tris) {
          ContactPair<R> c; c.type = ContactType::RIGID_POINT_TRIANGLE; c.idx0 = Index(v);
          c.idx1 = t.v[0]; c.idx2 = t.v[1]; c.idx3 = t.v[2]; c.rigid_body_index = int(rb);
          narrow_pt(st.positions[v], wv[size_t(t.v[0])], wv[size_t(t.v[1])], wv[size_t(t.v[2])], c.gap, c.normal, c.witness_p, c.witness_q);
          if (c.gap < R(0.01)) { c.vertex_count = 1; c.weights[0] = R(1); out.push_back(c); }
        }
    }
  }
  return out;
}

// -------------------------------------------------------------- line search
// line_search.cpp:163-247: 10 temporal samples, hit when distance < 1e-6.
template <class R> R ccd_pt(const V3<R>& p0, const V3<R>& p1, const V3<R>& a0, const V3<R>& a1, const V3<R>& b0, const V3<R>& b1, const V3<R>& c0, const V3<R>& c1) {
  if ((p1 - p0).sq() < R(1e-12) && (a1 - a0).sq() < R(1e-12) && (b1 - b0).sq() < R(1e-12) && (c1 - c0).sq() < R(1e-12)) return R(1);
  for (int i = 1; i <= 10; ++i) {
    R t = R(i) / R(10);
    R d; V3<R> n, wp, wq;
    narrow_pt(p0 + (p1 - p0) * t, a0 + (a1 - a0) * t, b0 + (b1 - b0) * t, c0 + (c1 - c0) * t, d, n, wp, wq);
    if (d < R(1e-6)) return t;
  }
  return R(1);
}
template <class R> R ccd_ee(const V3<R>& p00, const V3<R>& p01, const V3<R>& p10, const V3<R>& p11, const V3<R>& q00, const V3<R>& q01, const V3<R>& q10, const V3<R>& q11) {
  if ((p01 - p00).sq() < R(1e-12) && (p11 - p10).sq() < R(1e-12) && (q01 - q00).sq() < R(1e-12) && (q11 - q10).sq() < R(1e-12)) return R(1);
  for (int i = 1; i <= 10; ++i) {
    R t = R(i) / R(10);
    R d; V3<R> n, wp, wq;
    narrow_ee(p00 + (p01 - p00) * t, p10 + (p11 - p10) * t, q00 + (q01 - q00) * t, q10 + (q11 - q10) * t, d, n, wp, wq);
    if (d < R(1e-6)) return t;
  }
  return R(1);
}

// LineSearch::is_feasible (line_search.cpp:52-161), gap_min = 0.
template <class R> bool is_feasible(const std::vector<V3<R>>& xo, const std::vector<V3<R>>& xn, const std::vector<ContactPair<R>>& contacts,
                                    const std::vector<Pin<R>>& pins, const V3<R>& wn, R woff) {
  const R gap_min = R(0);
  for (const auto& c : contacts) {
    if (c.type == ContactType::POINT_TRIANGLE) {
      size_t i0 = size_t(c.idx0), i1 = size_t(c.idx1), i2 = size_t(c.idx2), i3 = size_t(c.idx3);
      if (ccd_pt(xo[i0], xn[i0], xo[i1], xn[i1], xo[i2], xn[i2], xo[i3], xn[i3]) < R(1)) return false;
      R d; V3<R> n, wp, wq; narrow_pt(xn[i0], xn[i1], xn[i2], xn[i3], d, n, wp, wq);
      if (d < gap_min) return false;
    } else if (c.type == ContactType::EDGE_EDGE) {
      size_t i0 = size_t(c.idx0), i1 = size_t(c.idx1), i2 = size_t(c.idx2), i3 = size_t(c.idx3);
      if (ccd_ee(xo[i0], xn[i0], xo[i1], xn[i1], xo[i2], xn[i2], xo[i3], xn[i3]) < R(1)) return false;
      R d; V3<R> n, wp, wq; narrow_ee(xn[i0], xn[i1], xn[i2], xn[i3], d, n, wp, wq);
      if (d < gap_min) return false;
    }
  }
  for (const auto& p : pins) if ((xn[size_t(p.vertex_idx)] - p.target_position).norm() < gap_min) return false;
  if (wn.sq() > R(0.5)) for (size_t i = 0; i < xn.size(); ++i) if (wn.dot(xn[i]) - woff < gap_min) return false;
  return true;
}

// LineSearch::search (line_search.cpp:8-50)
template <class R> R line_search(const std::vector<V3<R>>& x, const std::vector<R>& dir, const std::vector<ContactPair<R>>& contacts,
                                 const std::vector<Pin<R>>& pins, const V3<R>& wn, R woff, R extension = R(1.25), R min_alpha = R(1e-6)) {
  R alpha = 1;
  std::vector<V3<R>> ext(x.size()), xn(x.size());
  for (size_t i = 0; i < x.size(); ++i) ext[i] = V3<R>(extension * dir[3 * i], extension * dir[3 * i + 1], extension * dir[3 * i + 2]);
  for (int it = 0; it < 20; ++it) {
    for (size_t i = 0; i < x.size(); ++i) xn[i] = x[i] + ext[i] * alpha;
    if (is_feasible(x, xn, contacts, pins, wn, woff)) return alpha;
    alpha *= R(0.5);
    if (alpha < min_alpha) return R(0);
  }
  return alpha;
}

// --------------------------------------------------------------------- PCG
template <class R> struct PcgResult { bool converged = false; int iters = 0; R rel_res = 0; };

// PCGSolver::solve (pcg_solver.cpp:8-146): block-Jacobi, x0 as given, relative L-inf stop.
// Inverse of the lower Cholesky factor of a symmetric 3x3 block, in FP64, with
// the shifted retries of the GPU's diagonal factorisation (tr * 1e-12, 1e-8,
// 1e-4 added to the diagonal; last resort: sqrt|diagonal|). Row-major 3x3.
inline void chol_inverse3(const double H[9], double Linv[9]) {
  auto chol = [](const double A[9], double L[9]) {
    for (int k = 0; k < 9; ++k) L[k] = 0.0;
    double d0 = A[0]; if (!(d0 > 0.0)) return false;
    L[0] = std::sqrt(d0); L[3] = A[3] / L[0]; L[6] = A[6] / L[0];
    double d1 = A[4] - L[3] * L[3]; if (!(d1 > 0.0)) return false;
    L[4] = std::sqrt(d1); L[7] = (A[7] - L[6] * L[3]) / L[4];
    double d2 = A[8] - L[6] * L[6] - L[7] * L[7]; if (!(d2 > 0.0)) return false;
    L[8] = std::sqrt(d2); return true;
  };
  double L[9];
  bool ok = chol(H, L);
  if (!ok) {
    double tr = std::fabs(H[0]) + std::fabs(H[4]) + std::fabs(H[8]) + 1e-300;
    const double shift[3] = {1e-12, 1e-8, 1e-4};
    for (int t = 0; t < 3 && !ok; ++t) {
      double Hs[9]; for (int k = 0; k < 9; ++k) Hs[k] = H[k];
      Hs[0] += tr * shift[t]; Hs[4] += tr * shift[t]; Hs[8] += tr * shift[t];
      ok = chol(Hs, L);
    }
    if (!ok) {
      for (int k = 0; k < 9; ++k) L[k] = 0.0;
      L[0] = std::sqrt(std::max(std::fabs(H[0]), 1e-300)); L[4] = std::sqrt(std::max(std::fabs(H[4]), 1e-300)); L[8] = std::sqrt(std::max(std::fabs(H[8]), 1e-300));
    }
  }
  for (int k = 0; k < 9; ++k) Linv[k] = 0.0;
  Linv[0] = 1.0 / L[0]; Linv[4] = 1.0 / L[4]; Linv[8] = 1.0 / L[8];
  Linv[3] = -L[3] * Linv[0] / L[4];
  Linv[7] = -L[7] * Linv[4] / L[8];
  Linv[6] = -(L[6] * Linv[0] + L[7] * Linv[3]) / L[8];
}

// PCGSolver::solve (pcg_solver.cpp:8-146): block-Jacobi PCG from x0, stop on
// the relative L-inf residual. With scaled_stop (the CORRECTED step) the test
// is taken on the block-scaled residual max_i |L_i^-1 r_i| < tol *
// max_i |L_i^-1 b_i| (A_ii = L_i L_i^T), which a few rows with forces orders of
// magnitude above the rest cannot dominate; the iteration is unchanged.
template <class R> PcgResult<R> pcg_solve(const Csr<R>& A, const std::vector<R>& b, std::vector<R>& x, R tol, int max_iters,
                                          bool scaled_stop = false) {
  PcgResult<R> res;
  const int n = int(b.size()), nv = n / 3;
  std::vector<M3<R>> P(static_cast<size_t>(nv));
  std::vector<double> Li(scaled_stop ? size_t(9) * size_t(nv) : 0);
  for (int i = 0; i < nv; ++i) {
    M3<R> blk;
    for (int lr = 0; lr < 3; ++lr) { Index r = 3 * i + lr;
      for (Index k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) { Index c = A.cols[k]; if (c >= 3 * i && c < 3 * i + 3) blk(lr, c - 3 * i) = A.vals[k]; } }
    R det = blk.determinant();
    P[size_t(i)] = std::fabs(det) > R(1e-16) ? blk.inverse() : M3<R>::identity();
    if (scaled_stop) {
      double H[9]; for (int q = 0; q < 9; ++q) H[q] = double(blk(q / 3, q % 3));
      chol_inverse3(H, &Li[size_t(9) * size_t(i)]);
    }
  }
  auto linf = [&](const std::vector<R>& v) {
    double m = 0;
    if (!scaled_stop) { for (R e : v) m = std::max(m, double(std::fabs(e))); return R(m); }
    for (int i = 0; i < nv; ++i) {
      const double* q = &Li[size_t(9) * size_t(i)];
      for (int r = 0; r < 3; ++r) {
        double u = q[3 * r] * double(v[size_t(3 * i)]) + q[3 * r + 1] * double(v[size_t(3 * i + 1)]) + q[3 * r + 2] * double(v[size_t(3 * i + 2)]);
        m = std::max(m, std::fabs(u));
      }
    }
    return R(m);
  };
  const R binf = linf(b);
  auto rel = [&](const std::vector<R>& r) { R ri = linf(r); return binf < R(1e-16) ? ri : ri / binf; };
  auto dot = [](const std::vector<R>& a, const std::vector<R>& c) { R s = 0; for (size_t k = 0; k < a.size(); ++k) s += a[k] * c[k]; return s; };
  auto apply = [&](const std::vector<R>& r, std::vector<R>& z) {
    parallel_for(nv, [&](long long i) { V3<R> rb(r[size_t(3 * i)], r[size_t(3 * i + 1)], r[size_t(3 * i + 2)]); V3<R> zb = P[size_t(i)] * rb;
      z[size_t(3 * i)] = zb.x; z[size_t(3 * i + 1)] = zb.y; z[size_t(3 * i + 2)] = zb.z; });
  };
  std::vector<R> Ax; A.multiply(x, Ax);
  std::vector<R> r(static_cast<size_t>(n)); for (int i = 0; i < n; ++i) r[size_t(i)] = b[size_t(i)] - Ax[size_t(i)];
  res.rel_res = rel(r);
  if (res.rel_res < tol) { res.converged = true; return res; }
  std::vector<R> z(static_cast<size_t>(n), R(0)); apply(r, z);
  std::vector<R> p = z, Ap;
  R rz = dot(r, z);
  for (int it = 0; it < max_iters; ++it) {
    A.multiply(p, Ap);
    R pAp = dot(p, Ap);
    res.iters = it + 1;
    if (std::fabs(pAp) < R(1e-16)) { res.converged = false; return res; }
    R al = rz / pAp;
    parallel_for(n, [&](long long i) { x[size_t(i)] += al * p[size_t(i)]; r[size_t(i)] -= al * Ap[size_t(i)]; });
    res.rel_res = rel(r);
    if (res.rel_res < tol) { res.converged = true; return res; }
    apply(r, z);
    R rzn = dot(r, z); R be = rzn / rz; rz = rzn;
    parallel_for(n, [&](long long i) { p[size_t(i)] = z[size_t(i)] + be * p[size_t(i)]; });
  }
  return res;
}

// -------------------------------------------------------------- integrator
template <class R> struct StepStats {
  int newton_iters = 0, pcg_iters = 0, line_search_fail = 0, contacts = 0, pcg_not_converged = 0, strain_active = 0, substeps = 1;
  R beta = 0; std::vector<R> alphas; std::vector<int> pcg_per_newton;
};

template <class R> struct Options { Lookup lookup = Lookup::INDEXED; BroadPhase broad = BroadPhase::LITERAL; };

template <class R> class Integrator {
 public:
  // Integrator::step (integrator.cpp:70-150)
  static void step(Mesh<R>& mesh, State<R>& st, Constraints<R>& C, const SimParams<R>& p, std::vector<RigidBody<R>>* rigids,
                   const Options<R>& opt, StepStats<R>* stats = nullptr) {
    StepStats<R> local; StepStats<R>& S = stats ? *stats : local;
    S = StepStats<R>();
    const size_t n = st.positions.size(); const R dt = p.dt;
    std::vector<V3<R>> x_old = st.positions, x_target(n);
    for (size_t i = 0; i < n; ++i) x_target[i] = st.positions[i] + st.velocities[i] * dt;
    auto contacts = detect_all(mesh, st, rigids, opt.broad);
    S.contacts = int(contacts.size());
    R beta = 0; int bi = 0;
    while (beta < p.beta_max && bi < 20) {
      R alpha = inner_newton(mesh, st, x_target, contacts, C, p, opt, S);
      beta = R(double(beta) + (1.0 - double(beta)) * double(alpha));
      ++bi;
      if (alpha < R(1e-6)) { S.line_search_fail++; break; }
    }
    if (beta > R(1e-6)) inner_newton(mesh, st, x_target, contacts, C, p, opt, S);
    S.beta = beta;
    if (beta > R(1e-6)) {
      R bdt = beta * dt;
      for (size_t i = 0; i < n; ++i) st.velocities[i] = V3<R>((st.positions[i].x - x_old[i].x) / bdt, (st.positions[i].y - x_old[i].y) / bdt, (st.positions[i].z - x_old[i].z) / bdt);
      if (p.velocity_damping > R(0)) { R sc = R(1) - std::clamp(p.velocity_damping, R(0), R(1)); for (auto& v : st.velocities) v = v * sc; }
      if (p.contact_restitution > R(0)) restitution(mesh, C, st, p, rigids, opt);
    }
    if (rigids && !rigids->empty()) rigid_coupling(mesh, st, *rigids, p, opt);
  }

  // Integrator::inner_newton_step (integrator.cpp:152-236)
  static R inner_newton(const Mesh<R>& mesh, State<R>& st, const std::vector<V3<R>>& x_target, const std::vector<ContactPair<R>>& contacts,
                        Constraints<R>& C, const SimParams<R>& p, const Options<R>& opt, StepStats<R>& S) {
    const size_t n = st.positions.size();
    int max_it = p.max_newton_steps;
    if (p.enable_friction) max_it = std::max(max_it, p.friction_min_newton_steps);
    for (int it = 0; it < max_it; ++it) {
      std::vector<R> g(3 * n, R(0));
      gradient(mesh, st, x_target, contacts, C, p, opt, g);
      R gn = 0; for (R e : g) gn = std::max(gn, std::fabs(e));
      if (gn < p.pcg_tol) return R(1);
      S.newton_iters++;
      Csr<R> H = assemble(mesh, st, contacts, C, p, opt);
      std::vector<R> d(3 * n, R(0)), ng(3 * n);
      for (size_t i = 0; i < 3 * n; ++i) ng[i] = -g[i];
      auto pr = pcg_solve(H, ng, d, p.pcg_tol, p.pcg_max_iters);
      S.pcg_iters += pr.iters; S.pcg_per_newton.push_back(pr.iters);
      if (!pr.converged) S.pcg_not_converged++;
      std::vector<Pin<R>> pins; for (auto& pn : C.pins) if (pn.active) pins.push_back(pn);
      V3<R> wn(0, 0, 0); R woff = 0;
      for (auto& w : C.walls) if (w.active) { wn = w.normal; woff = w.offset; break; }
      R alpha = line_search(st.positions, d, contacts, pins, wn, woff, R(1.25));
      S.alphas.push_back(alpha);
      if (alpha < R(1e-8)) return R(0);
      R s = R(double(alpha) * 1.25);
      for (size_t i = 0; i < n; ++i) st.positions[i] = st.positions[i] + V3<R>(d[3 * i], d[3 * i + 1], d[3 * i + 2]) * s;
      if (alpha > R(0.99)) return R(1);
    }
    return R(0.5);
  }

  static void base_matrices(const Mesh<R>& mesh, const State<R>& st, const SimParams<R>& p, bool skip_zero_mass, Csr<R>& H_total, Csr<R>& H_el) {
    const Index n = Index(st.positions.size());
    std::vector<Triplet<R>> base, el;
    R dt2 = p.dt * p.dt;
    for (Index i = 0; i < n; ++i) {
      R v = skip_zero_mass ? st.masses[size_t(i)] * (R(1) / dt2) : st.masses[size_t(i)] * R(1.0 / double(dt2));
      if (skip_zero_mass && v == R(0)) continue;
      for (int j = 0; j < 3; ++j) base.push_back({3 * i + j, 3 * i + j, v});
    }
    elastic_hessian_triplets(mesh, el);
    base.insert(base.end(), el.begin(), el.end());
    H_total = Csr<R>::from_triplets(3 * n, base);
    H_el = Csr<R>::from_triplets(3 * n, el);
  }

  // Integrator::compute_gradient (integrator.cpp:246-396)
  static void gradient(const Mesh<R>& mesh, const State<R>& st, const std::vector<V3<R>>& x_target, const std::vector<ContactPair<R>>& contacts,
                       Constraints<R>& C, const SimParams<R>& p, const Options<R>& opt, std::vector<R>& g) {
    const size_t n = st.positions.size(); const R dt = p.dt;
    for (size_t i = 0; i < n; ++i) { R mf = st.masses[i] / (dt * dt); for (int j = 0; j < 3; ++j) g[3 * i + size_t(j)] += mf * (st.positions[i][j] - x_target[i][j]); }
    std::vector<R> ge; elastic_gradient(mesh, ge);
    for (size_t i = 0; i < g.size() && i < ge.size(); ++i) g[i] += ge[i];
    Csr<R> H_total, H_el; base_matrices(mesh, st, p, false, H_total, H_el);
    if (p.enable_strain_limiting) { strain_rebuild(mesh, st, p, H_el, C, opt.lookup); strain_gradient(mesh, st, C, p, g); }
    else C.strain_limits.clear();
    for (const auto& c : contacts) {
      if (c.type != ContactType::POINT_TRIANGLE && c.type != ContactType::RIGID_POINT_TRIANGLE) continue;
      if (opt.lookup == Lookup::LITERAL) (void)extract_hessian_block(H_total, c.idx0, opt.lookup);  // unused by the reference too
      R kb = contact_stiffness(c, st.masses, dt, H_el, opt.lookup);
      if (!in_domain(c.gap, p.contact_gap_max)) continue;
      V3<R> nrm = normalize_or_default(c.normal, p.contact_normal_epsilon);
      R dV = barrier_gradient(c.gap, p.contact_gap_max, kb);
      if (dV == R(0)) continue;
      Index ids[4] = {c.idx0, c.idx1, c.idx2, c.idx3};
      int cnt = std::max(c.vertex_count, 1);
      for (int i = 0; i < cnt; ++i) {
        if (ids[i] < 0 || c.weights[size_t(i)] == R(0)) continue;
        V3<R> add = nrm * (dV * c.weights[size_t(i)]);
        for (int k = 0; k < 3; ++k) g[size_t(ids[i]) * 3 + size_t(k)] += add[k];
      }
    }
    for (const auto& pin : C.pins) {
      if (!pin.active) continue;
      V3<R> off = st.positions[size_t(pin.vertex_idx)] - pin.target_position;
      M3<R> Hb = extract_hessian_block(H_total, pin.vertex_idx, opt.lookup);
      R kb = pin_stiffness(st.masses[size_t(pin.vertex_idx)], dt, off, Hb, p.min_gap);
      R gap = off.norm();
      if (!in_domain(gap, p.contact_gap_max) || gap <= p.contact_normal_epsilon) continue;
      V3<R> nn = off / gap; R dV = barrier_gradient(gap, p.contact_gap_max, kb);
      for (int k = 0; k < 3; ++k) g[size_t(pin.vertex_idx) * 3 + size_t(k)] += dV * nn[k];
    }
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nrm = normalize_or_default(w.normal, p.contact_normal_epsilon);
      for (size_t vi = 0; vi < n; ++vi) {
        M3<R> Hb = extract_hessian_block(H_total, Index(vi), opt.lookup);
        R kb = wall_stiffness(st.masses[vi], p.wall_gap, w.normal, Hb, p.min_gap);
        R gap = nrm.dot(st.positions[vi]) - w.offset;
        if (!in_domain(gap, p.contact_gap_max)) continue;
        R dV = barrier_gradient(gap, p.contact_gap_max, kb);
        for (int k = 0; k < 3; ++k) g[vi * 3 + size_t(k)] += dV * nrm[k];
      }
    }
    if (p.enable_friction && p.friction_mu > R(0)) {
      for (const auto& c : contacts) {
        R kf; V3<R> tang;
        if (!friction_data(c, st, dt, H_el, p, opt, kf, tang)) continue;
        V3<R> fg = tang * kf;  // friction.cpp:49-58
        for (int k = 0; k < 3; ++k) g[size_t(c.idx0) * 3 + size_t(k)] += fg[k];
      }
    }
  }

  // compute_friction_data (integrator.cpp:28-66)
  static bool friction_data(const ContactPair<R>& c, const State<R>& st, R dt, const Csr<R>& H_el, const SimParams<R>& p, const Options<R>& opt, R& kf, V3<R>& tang) {
    V3<R> disp = st.positions[size_t(c.idx0)] - st.positions_prev[size_t(c.idx0)];
    tang = disp - c.normal * disp.dot(c.normal);
    R tn = tang.norm();
    if (!(tn > p.friction_tangent_threshold)) return false;
    R kc = contact_stiffness(c, st.masses, dt, H_el, opt.lookup);
    R fn = kc * std::fabs(c.gap);
    R den = std::max(p.friction_epsilon, std::fabs(tn));
    if (den <= R(0)) den = p.friction_epsilon;
    kf = std::min(p.friction_mu * std::fabs(fn) / den, R(1e8));
    return true;
  }

  // Integrator::assemble_system_matrix (integrator.cpp:398-544)
  static Csr<R> assemble(const Mesh<R>& mesh, const State<R>& st, const std::vector<ContactPair<R>>& contacts, Constraints<R>& C,
                         const SimParams<R>& p, const Options<R>& opt) {
    const Index n = Index(st.positions.size()); const R dt = p.dt;
    std::vector<Triplet<R>> tr, el;
    R dinv = R(1) / (dt * dt);
    if (dt > R(0))
      for (Index row = 0; row < 3 * n; ++row) { R v = st.masses[size_t(row / 3)] * dinv; if (v == R(0)) continue; tr.push_back({row, row, v}); }
    elastic_hessian_triplets(mesh, el);
    tr.insert(tr.end(), el.begin(), el.end());
    Csr<R> H_base = Csr<R>::from_triplets(3 * n, tr), H_el = Csr<R>::from_triplets(3 * n, el);
    if (p.enable_strain_limiting) {
      if (C.strain_limits.empty()) strain_rebuild(mesh, st, p, H_el, C, opt.lookup);
      strain_hessian(mesh, st, C, p, tr);
    } else C.strain_limits.clear();
    for (const auto& c : contacts) {
      if (c.type != ContactType::POINT_TRIANGLE && c.type != ContactType::RIGID_POINT_TRIANGLE) continue;
      if (opt.lookup == Lookup::LITERAL) (void)extract_hessian_block(H_base, c.idx0, opt.lookup);
      R kb = contact_stiffness(c, st.masses, dt, H_el, opt.lookup);
      if (!in_domain(c.gap, p.contact_gap_max)) continue;
      V3<R> nrm = normalize_or_default(c.normal, p.contact_normal_epsilon);
      R d2V = barrier_hessian(c.gap, p.contact_gap_max, kb);
      if (d2V == R(0)) continue;
      Index ids[4] = {c.idx0, c.idx1, c.idx2, c.idx3};
      int cnt = std::max(c.vertex_count, 1);
      for (int i = 0; i < cnt; ++i) {
        if (c.weights[size_t(i)] == R(0)) continue;
        V3<R> gi = nrm * c.weights[size_t(i)];
        for (int j = 0; j < cnt; ++j) {
          if (c.weights[size_t(j)] == R(0)) continue;
          V3<R> gj = nrm * c.weights[size_t(j)];
          for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) {
            if (ids[i] < 0 || ids[j] < 0) continue;
            R v = d2V * (gi[r] * gj[q]);
            if (std::fabs(v) < p.barrier_tolerance) continue;
            tr.push_back({ids[i] * 3 + r, ids[j] * 3 + q, v});
          }
        }
      }
    }
    for (const auto& pin : C.pins) {
      if (!pin.active) continue;
      M3<R> Hb = extract_hessian_block(H_base, pin.vertex_idx, opt.lookup);
      V3<R> off = st.positions[size_t(pin.vertex_idx)] - pin.target_position;
      R kb = pin_stiffness(st.masses[size_t(pin.vertex_idx)], dt, off, Hb, p.min_gap);
      R gap = off.norm();
      if (!in_domain(gap, p.contact_gap_max) || gap <= p.contact_normal_epsilon) continue;
      V3<R> nn = off / gap;
      R dV = barrier_gradient(gap, p.contact_gap_max, kb), d2V = barrier_hessian(gap, p.contact_gap_max, kb);
      M3<R> nnT = M3<R>::outer(nn, nn);
      M3<R> Hm = nnT * d2V + (M3<R>::identity() - nnT) * (dV / gap);
      for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) { if (std::fabs(Hm(r, q)) < p.barrier_tolerance) continue; tr.push_back({pin.vertex_idx * 3 + r, pin.vertex_idx * 3 + q, Hm(r, q)}); }
    }
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nrm = normalize_or_default(w.normal, p.contact_normal_epsilon);
      for (Index vi = 0; vi < n; ++vi) {
        M3<R> Hb = extract_hessian_block(H_base, vi, opt.lookup);
        R kb = wall_stiffness(st.masses[size_t(vi)], p.wall_gap, w.normal, Hb, p.min_gap);
        R gap = nrm.dot(st.positions[size_t(vi)]) - w.offset;
        if (!in_domain(gap, p.contact_gap_max)) continue;
        R d2V = barrier_hessian(gap, p.contact_gap_max, kb);
        M3<R> Hm = M3<R>::outer(nrm, nrm) * d2V;
        for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) { if (std::fabs(Hm(r, q)) < p.barrier_tolerance) continue; tr.push_back({vi * 3 + r, vi * 3 + q, Hm(r, q)}); }
      }
    }
    if (p.enable_friction && p.friction_mu > R(0)) {
      for (const auto& c : contacts) {
        R kf; V3<R> tang;
        if (!friction_data(c, st, dt, H_el, p, opt, kf, tang)) continue;
        M3<R> Hf = (M3<R>::identity() * kf - M3<R>::outer(c.normal, c.normal) * kf) + M3<R>::identity() * R(1e-8);
        for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) { if (std::fabs(Hf(r, q)) > R(1e-12)) tr.push_back({c.idx0 * 3 + r, c.idx0 * 3 + q, Hf(r, q)}); }
      }
    }
    return Csr<R>::from_triplets(3 * n, tr).symmetrized();
  }

  // Integrator::apply_contact_restitution (integrator.cpp:565-674)
  static void restitution(const Mesh<R>& mesh, const Constraints<R>& C, State<R>& st, const SimParams<R>& p, std::vector<RigidBody<R>>* rigids, const Options<R>& opt) {
    R e = std::clamp(p.contact_restitution, R(0), R(1));
    if (e <= R(0)) return;
    auto impulse = [&](Index idx, const V3<R>& normal) {
      if (idx < 0 || size_t(idx) >= st.velocities.size()) return;
      V3<R> nn = normal; R nr = nn.norm(); if (nr < R(1e-8)) return; nn = nn / nr;
      V3<R>& v = st.velocities[size_t(idx)]; R vn = v.dot(nn);
      if (vn < R(0)) v -= nn * ((R(1) + e) * vn);
    };
    auto cs = detect_all(mesh, st, rigids, opt.broad);
    R gl = std::max(p.contact_gap_max, R(1e-5));
    for (const auto& c : cs) {
      if (c.gap > gl) continue;
      if (c.type == ContactType::POINT_TRIANGLE) impulse(c.idx0, c.normal);
      else if (c.type == ContactType::EDGE_EDGE) { impulse(c.idx0, c.normal); impulse(c.idx1, c.normal); impulse(c.idx2, -c.normal); impulse(c.idx3, -c.normal); }
      else if (c.type == ContactType::WALL) impulse(c.idx0, c.normal);
      else if (c.type == ContactType::RIGID_POINT_TRIANGLE && rigids && c.rigid_body_index >= 0 && c.rigid_body_index < int(rigids->size())) {
        V3<R> nn = c.normal; R nr = nn.norm(); if (nr < R(1e-8)) continue; nn = nn / nr;
        Index vi = c.idx0; if (vi < 0 || size_t(vi) >= st.velocities.size()) continue;
        auto& body = (*rigids)[size_t(c.rigid_body_index)];
        V3<R> vv = st.velocities[size_t(vi)], rel = vv - body.velocity_at_point(c.witness_q);
        R vn = rel.dot(nn); if (vn >= R(0)) continue;
        R im = st.masses[size_t(vi)] > R(0) ? R(1) / st.masses[size_t(vi)] : R(0);
        V3<R> rr = c.witness_q - body.position, cr = rr.cross(nn);
        R den = im + cr.dot(body.inertia_world_inv() * cr);
        if (den <= R(0)) continue;
        R j = -(R(1) + e) * vn / den; V3<R> J = nn * j;
        vv += J * im; st.velocities[size_t(vi)] = vv; body.apply_impulse(c.witness_q, -J);
      }
    }
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nn = w.normal; R nr = nn.norm(); if (nr < R(1e-8)) continue; nn = nn / nr;
      for (size_t i = 0; i < st.positions.size(); ++i) if (nn.dot(st.positions[i]) - w.offset <= w.gap + p.contact_gap_max) impulse(Index(i), nn);
    }
  }

  // Integrator::apply_rigid_coupling (integrator.cpp:676-754)
  static void rigid_coupling(const Mesh<R>& mesh, const State<R>& st, std::vector<RigidBody<R>>& rigids, const SimParams<R>& p, const Options<R>& opt) {
    if (rigids.empty()) return;
    auto cs = detect_all(mesh, st, &rigids, opt.broad);
    Csr<R> H_total, H_el; base_matrices(mesh, st, p, false, H_total, H_el);
    for (auto& b : rigids) { b.acc_force = V3<R>(); b.acc_torque = V3<R>(); }
    for (const auto& c : cs) {
      if (c.type != ContactType::RIGID_POINT_TRIANGLE) continue;
      if (c.rigid_body_index < 0 || c.rigid_body_index >= int(rigids.size())) continue;
      if (opt.lookup == Lookup::LITERAL) (void)extract_hessian_block(H_total, c.idx0, opt.lookup);
      R kb = contact_stiffness(c, st.masses, p.dt, H_el, opt.lookup);
      V3<R> nn = c.normal; R nr = nn.norm(); if (nr < R(1e-8)) continue; nn = nn / nr;
      R dV = barrier_gradient(c.gap, p.contact_gap_max, kb);
      if (std::fabs(dV) < R(1e-12)) continue;
      rigids[size_t(c.rigid_body_index)].apply_force(c.witness_q, -(nn * dV), R(0));
    }
    for (auto& b : rigids) b.integrate(p.dt);
  }
};


// ======================================================================
// CORRECTED semantics: the step the reference intends (its docs/dev/
// PROJECT_SPEC.md), with the defects listed in the REFERENCE path fixed:
//   * elasticity on the current positions; the constant Hessian is the exact
//     Hessian of k |F - R|^2 for a fixed frame R: 2k (G G^T) (x) I3 with
//     G = [[-1,-1],[1,0],[0,1]] Dm_inv (no SPD clamp needed, it is PSD);
//   * kinematic pins: a pinned vertex is placed on its target at the start of
//     the step and its degrees of freedom are removed from the solve;
//   * self contact from the intended broad phase (boxes inflated by the
//     barrier activation distance), vertex-triangle AND edge-edge barriers,
//     gaps, normals and weights refreshed at every Newton iteration (edge-edge
//     weights are the closest-point parameters [1-s, s, -(1-t), -t]);
//   * line search: a conservative time of impact along the extended direction
//     (conservative advancement with exact distances, FP64) over every pair
//     whose swept boxes overlap, plus the exact linear time of impact of every
//     active wall; the step taken is x += toi * d. The extended direction is
//     first capped so that no vertex moves more than 4 mean rest edge lengths
//     in one Newton iteration (bounds the swept boxes).
// ======================================================================

// Correct BVH query (leaves keep up to 4 primitives): the same candidate set
// as the brute-force INTENDED broad phase in O(n log n).
template <class R> struct QBVH {
  struct Node { AABB<R> box; int left = -1, right = -1, start = 0, end = 0; };
  std::vector<Node> nodes; std::vector<int> idx;
  int build(const std::vector<AABB<R>>& pb, int s, int e) {
    int ni = int(nodes.size()); nodes.emplace_back();
    AABB<R> box; for (int i = s; i < e; ++i) box.expand(pb[size_t(idx[size_t(i)])]);
    nodes[size_t(ni)].box = box; nodes[size_t(ni)].start = s; nodes[size_t(ni)].end = e;
    if (e - s <= 4) return ni;
    int ax = box.longest_axis();
    std::sort(idx.begin() + s, idx.begin() + e, [&](int a, int c) { return pb[size_t(a)].center()[ax] < pb[size_t(c)].center()[ax]; });
    int mid = s + (e - s) / 2;
    int l = build(pb, s, mid), r = build(pb, mid, e);
    nodes[size_t(ni)].left = l; nodes[size_t(ni)].right = r;
    return ni;
  }
  void init(const std::vector<AABB<R>>& pb) {
    nodes.clear(); idx.resize(pb.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = int(i);
    if (!pb.empty()) build(pb, 0, int(pb.size()));
  }
  template <class F> void query(const AABB<R>& q, const std::vector<AABB<R>>& pb, F&& visit) const {
    if (nodes.empty()) return;
    std::vector<int> st = {0};
    while (!st.empty()) {
      int ni = st.back(); st.pop_back();
      const Node& nd = nodes[size_t(ni)];
      if (!q.overlaps(nd.box)) continue;
      if (nd.left < 0) { for (int i = nd.start; i < nd.end; ++i) if (q.overlaps(pb[size_t(idx[size_t(i)])])) visit(idx[size_t(i)]); }
      else { st.push_back(nd.right); st.push_back(nd.left); }
    }
  }
};

// Candidate pairs with the reference predicate over boxes spanning positions
// x0 and x1 (x1 == nullptr: boxes at x0), inflated by pad; sorted.
template <class R> void candidates(const Mesh<R>& m, const std::vector<V3<R>>& x0, const std::vector<V3<R>>* x1, R pad,
                                   std::vector<std::pair<int, int>>& vt, std::vector<std::pair<int, int>>& ee) {
  vt.clear(); ee.clear();
  auto tb = triangle_boxes(m, x0);
  auto eb = edge_boxes(m, x0);
  if (x1) {
    auto tb1 = triangle_boxes(m, *x1); auto eb1 = edge_boxes(m, *x1);
    for (size_t i = 0; i < tb.size(); ++i) tb[i].expand(tb1[i]);
    for (size_t i = 0; i < eb.size(); ++i) eb[i].expand(eb1[i]);
  }
  for (auto& b : tb) inflate(b, pad);
  for (auto& b : eb) inflate(b, pad);
  QBVH<R> tq, eq; tq.init(tb); eq.init(eb);
  // queries on the host's cores into per-query lists, concatenated in query
  // order: the same pairs in the same order as one thread finds them
  const long long nv = (long long)x0.size(), ne = (long long)eb.size();
  std::vector<std::vector<int>> vt_of(static_cast<size_t>(nv)), ee_of(static_cast<size_t>(ne));
  parallel_for(nv, [&](long long v) {
    AABB<R> pbx = point_box(x0[size_t(v)]);
    if (x1) pbx.expand(point_box((*x1)[size_t(v)]));
    inflate(pbx, pad);
    tq.query(pbx, tb, [&](int t) {
      const auto& tri = m.triangles[size_t(t)];
      if (tri.v[0] == int(v) || tri.v[1] == int(v) || tri.v[2] == int(v)) return;
      vt_of[size_t(v)].push_back(t);
    });
  });
  parallel_for(ne, [&](long long a) {
    eq.query(eb[size_t(a)], eb, [&](int b) {
      if (int(a) >= b) return;
      const Edge &e1 = m.edges[size_t(a)], &e2 = m.edges[size_t(b)];
      if (e1.v[0] == e2.v[0] || e1.v[0] == e2.v[1] || e1.v[1] == e2.v[0] || e1.v[1] == e2.v[1]) return;
      ee_of[size_t(a)].push_back(b);
    });
  });
  for (long long v = 0; v < nv; ++v) for (int t : vt_of[size_t(v)]) vt.push_back({int(v), t});
  for (long long a = 0; a < ne; ++a) for (int b : ee_of[size_t(a)]) ee.push_back({int(a), b});
  std::sort(vt.begin(), vt.end()); std::sort(ee.begin(), ee.end());
}

// Contacts inside the activation distance at positions x (refreshed every Newton iteration).
template <class R> std::vector<ContactPair<R>> detect_corrected(const Mesh<R>& m, const std::vector<V3<R>>& x, const std::vector<RigidBody<R>>* rigids, R gap_max) {
  std::vector<ContactPair<R>> out;
  std::vector<std::pair<int, int>> vt, ee;
  candidates(m, x, (const std::vector<V3<R>>*)nullptr, gap_max, vt, ee);
  for (auto& pr : vt) {
    ContactPair<R> c; c.type = ContactType::POINT_TRIANGLE; c.idx0 = pr.first;
    const auto& t = m.triangles[size_t(pr.second)]; c.idx1 = t.v[0]; c.idx2 = t.v[1]; c.idx3 = t.v[2];
    const auto &p = x[size_t(c.idx0)], &a = x[size_t(c.idx1)], &b = x[size_t(c.idx2)], &cc = x[size_t(c.idx3)];
    narrow_pt(p, a, b, cc, c.gap, c.normal, c.witness_p, c.witness_q);
    if (!(c.gap < gap_max)) continue;
    V3<R> bc = triangle_barycentric(c.witness_q, a, b, cc); c.barycentric = bc;
    c.weights = {R(1), -bc[0], -bc[1], -bc[2]}; c.vertex_count = 4; out.push_back(c);
  }
  for (auto& pr : ee) {
    ContactPair<R> c; c.type = ContactType::EDGE_EDGE;
    const Edge &e1 = m.edges[size_t(pr.first)], &e2 = m.edges[size_t(pr.second)];
    c.idx0 = e1.v[0]; c.idx1 = e1.v[1]; c.idx2 = e2.v[0]; c.idx3 = e2.v[1];
    R sp, tp;
    narrow_ee(x[size_t(c.idx0)], x[size_t(c.idx1)], x[size_t(c.idx2)], x[size_t(c.idx3)], c.gap, c.normal, c.witness_p, c.witness_q, &sp, &tp);
    if (!(c.gap < gap_max)) continue;
    c.vertex_count = 4; c.weights = {R(1) - sp, sp, -(R(1) - tp), -tp}; out.push_back(c);
  }
  if (rigids) {
    for (size_t rb = 0; rb < rigids->size(); ++rb) {
      const auto& body = (*rigids)[rb];
      auto wv = body.world_vertices();
      for (size_t v = 0; v < x.size(); ++v)
        for (const auto& t : body.tris) {
          ContactPair<R> c; c.type = ContactType::RIGID_POINT_TRIANGLE; c.idx0 = Index(v);
          c.idx1 = t.v[0]; c.idx2 = t.v[1]; c.idx3 = t.v[2]; c.rigid_body_index = int(rb);
          narrow_pt(x[v], wv[size_t(t.v[0])], wv[size_t(t.v[1])], wv[size_t(t.v[2])], c.gap, c.normal, c.witness_p, c.witness_q);
          if (c.gap < gap_max) { c.vertex_count = 1; c.weights[0] = R(1); out.push_back(c); }
        }
    }
  }
  return out;
}

// Constant elastic Hessian of the CORRECTED energy: per face the 3x3 vertex
// blocks c_ab I3 with c_ab = 2k (G G^T)_ab.
template <class R> void corrected_face_coeffs(const Mesh<R>& mesh, size_t f, R c[3][3]) {
  R mu = R(double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio))));
  R k = mesh.rest_areas[f] * mesh.material.thickness * mu;
  const M2<R>& D = mesh.Dm_inv[f];
  R G[3][2] = {{-(D.a + D.c), -(D.b + D.d)}, {D.a, D.b}, {D.c, D.d}};
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) c[a][b] = R(2) * k * (G[a][0] * G[b][0] + G[a][1] * G[b][1]);
}
template <class R> void corrected_elastic_triplets(const Mesh<R>& mesh, std::vector<Triplet<R>>& out) {
  for (size_t f = 0; f < mesh.triangles.size(); ++f) {
    const auto& t = mesh.triangles[f];
    R c[3][3]; corrected_face_coeffs(mesh, f, c);
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) for (int k = 0; k < 3; ++k) out.push_back({t.v[a] * 3 + k, t.v[b] * 3 + k, c[a][b]});
  }
  // quadratic bending: its (constant) Hessian 2 k_b (3 / A_e) K K^T (x) I3 per hinge
  const double kb = double(mesh.material.bending_stiffness);
  if (kb > 0.0)
    for (const auto& h : mesh.hinges)
      for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) for (int k = 0; k < 3; ++k)
        out.push_back({h.v[a] * 3 + k, h.v[b] * 3 + k, R(kb * h.c * h.w[a] * h.w[b])});
}
// Quadratic bending energy k_b sum_e (3 / A_e) |K_e x|^2 (Mesh::compute_hinges)
// at X; adds its gradient 2 k_b (3 / A_e) K_e (K_e . x) to grad (3 per vertex).
template <class R> double bending_at(const Mesh<R>& mesh, const std::vector<V3<R>>& X, std::vector<double>& grad) {
  const double kb = double(mesh.material.bending_stiffness);
  if (!(kb > 0.0)) return 0.0;
  double E = 0.0;
  for (const auto& h : mesh.hinges) {
    double s[3] = {0, 0, 0};
    for (int a = 0; a < 4; ++a) for (int q = 0; q < 3; ++q) s[q] += h.w[a] * double(X[size_t(h.v[a])][q]);
    E += 0.5 * kb * h.c * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int a = 0; a < 4; ++a) for (int q = 0; q < 3; ++q) grad[3 * size_t(h.v[a]) + size_t(q)] += kb * h.c * h.w[a] * s[q];
  }
  return E;
}
// CORRECTED elasticity. The reference's membrane energy k |F - I|^2 is taken
// in a frame aligned with edge e1, and its force formula (elasticity.cpp:18-61)
// drops the rotation of that frame, so away from the rest shape it is not the
// gradient of that energy (central differences differ by tens of percent on a
// sheared face). CORRECTED uses the as-rigid-as-possible membrane energy
// E = k |F - R|^2 = k ((s0 - 1)^2 + (s1 - 1)^2), F = [x1 - x0, x2 - x0] Dm^-1
// (3 x 2), R = U V^T from its thin SVD, k = area * thickness * mu. Its
// gradient 2k (F - R) G^T (G = [[-1,-1],[1,0],[0,1]] Dm^-1) is exact, and
// 2k (G G^T) (x) I3 (corrected_elastic_triplets) is its Hessian at fixed R.
// Returns the face energy; adds the face's gradient to grad[0..2].
template <class R> double arap_face(const Mesh<R>& mesh, const std::vector<V3<R>>& X, size_t f, double grad[3][3]) {
  const auto& t = mesh.triangles[f];
  const double mu = double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio)));
  const double k = double(mesh.rest_areas[f]) * double(mesh.material.thickness) * mu;
  const M2<R>& D = mesh.Dm_inv[f];
  const double da = D.a, db = D.b, dc = D.c, dd = D.d;
  double e1[3], e2[3], F0[3], F1[3];
  for (int q = 0; q < 3; ++q) {
    e1[q] = double(X[size_t(t.v[1])][q]) - double(X[size_t(t.v[0])][q]);
    e2[q] = double(X[size_t(t.v[2])][q]) - double(X[size_t(t.v[0])][q]);
    F0[q] = e1[q] * da + e2[q] * dc; F1[q] = e1[q] * db + e2[q] * dd;
  }
  V3<double> Fc[2] = {V3<double>(F0[0], F0[1], F0[2]), V3<double>(F1[0], F1[1], F1[2])};
  Svd32<double> sv; svd32(Fc, sv);
  // R = U V^T: column c is U0 V[c][0] + U1 V[c][1]
  V3<double> Rc[2] = {sv.U[0] * sv.V[0][0] + sv.U[1] * sv.V[0][1], sv.U[0] * sv.V[1][0] + sv.U[1] * sv.V[1][1]};
  double P0[3], P1[3], E = 0.0;
  for (int q = 0; q < 3; ++q) {
    double a = F0[q] - Rc[0][q], b = F1[q] - Rc[1][q];
    E += a * a + b * b;
    P0[q] = 2.0 * k * a; P1[q] = 2.0 * k * b;
  }
  const double G[3][2] = {{-(da + dc), -(db + dd)}, {da, db}, {dc, dd}};
  for (int a = 0; a < 3; ++a) for (int q = 0; q < 3; ++q) grad[a][q] += P0[q] * G[a][0] + P1[q] * G[a][1];
  return k * E;
}
// Exact membrane Hessian, projected to positive semidefinite per face
// (CORRECTED, membrane_hessian = 1). For E = k |F - R|^2 with F = U S V^T
// (3 x 2, thin SVD), R = U V^T, n = U0 x U1, the Hessian in F is
// 2k (I - dR/dF); its eigenpairs are 2k on the three symmetric in-plane modes,
// 2k (1 - 2 / (s0 + s1)) on the twist R J / sqrt 2 (J the 2 x 2 rotation by
// 90 degrees) and 2k (1 - 1 / s_i) on the flips n v_i^T. Clamping each at zero
// gives H = 2k I - a_t t t^T - sum_i c_i f_i f_i^T with a_t = 2k min(1, 2 / (s0 + s1))
// and c_i = 2k min(1, 1 / s_i): the fixed-rotation Hessian 2k I (the constant
// elastic blocks) minus, per vertex pair (a, b) of the face,
//   D_ab = a_t / 2 g_a g_b^T + w_ab n n^T,  g_a = G_a0 R1 - G_a1 R0,  w_ab = G_a W G_b^T,
// W = V diag(c0, c1) V^T. Near rest (s = 1) the twist and flips, which are
// the face's rotations, cost nothing, as the energy says. Writes D (FP64).
template <class R> void membrane_correction_face(const Mesh<R>& mesh, const std::vector<V3<R>>& X, size_t f, double D[3][3][9]) {
  const auto& t = mesh.triangles[f];
  const double mu = double(mesh.material.youngs_modulus) / (2.0 * (1.0 + double(mesh.material.poisson_ratio)));
  const double k = double(mesh.rest_areas[f]) * double(mesh.material.thickness) * mu;
  const M2<R>& Dm = mesh.Dm_inv[f];
  const double da = Dm.a, db = Dm.b, dc = Dm.c, dd = Dm.d;
  double e1[3], e2[3], F0[3], F1[3];
  for (int q = 0; q < 3; ++q) {
    e1[q] = double(X[size_t(t.v[1])][q]) - double(X[size_t(t.v[0])][q]);
    e2[q] = double(X[size_t(t.v[2])][q]) - double(X[size_t(t.v[0])][q]);
    F0[q] = e1[q] * da + e2[q] * dc; F1[q] = e1[q] * db + e2[q] * dd;
  }
  V3<double> Fc[2] = {V3<double>(F0[0], F0[1], F0[2]), V3<double>(F1[0], F1[1], F1[2])};
  Svd32<double> sv; svd32(Fc, sv);
  const V3<double> R0 = sv.U[0] * sv.V[0][0] + sv.U[1] * sv.V[0][1], R1 = sv.U[0] * sv.V[1][0] + sv.U[1] * sv.V[1][1];
  V3<double> n = sv.U[0].cross(sv.U[1]);
  const double nl = n.norm();
  if (nl > 0.0) n = n / nl;
  const double s0 = double(sv.sigma[0]), s1 = double(sv.sigma[1]);
  const double at = 2.0 * k * std::min(1.0, 2.0 / (s0 + s1));
  const double c0 = 2.0 * k * std::min(1.0, 1.0 / s0), c1 = 2.0 * k * std::min(1.0, 1.0 / s1);
  double W[2][2];
  for (int p2 = 0; p2 < 2; ++p2)
    for (int q2 = 0; q2 < 2; ++q2) W[p2][q2] = sv.V[p2][0] * c0 * sv.V[q2][0] + sv.V[p2][1] * c1 * sv.V[q2][1];
  const double G[3][2] = {{-(da + dc), -(db + dd)}, {da, db}, {dc, dd}};
  V3<double> g[3];
  for (int a = 0; a < 3; ++a) g[a] = R1 * G[a][0] - R0 * G[a][1];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double w = 0.0;
      for (int p2 = 0; p2 < 2; ++p2) for (int q2 = 0; q2 < 2; ++q2) w += G[a][p2] * W[p2][q2] * G[b][q2];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) D[a][b][3 * r + c] = 0.5 * at * g[a][r] * g[b][c] + w * n[r] * n[c];
    }
}
// The projection's correction of every face at X as triplets (subtracted).
template <class R> void membrane_correction_triplets(const Mesh<R>& mesh, const std::vector<V3<R>>& X, std::vector<Triplet<R>>& out) {
  for (size_t f = 0; f < mesh.triangles.size(); ++f) {
    double D[3][3][9];
    membrane_correction_face(mesh, X, f, D);
    const auto& t = mesh.triangles[f];
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c)
      out.push_back({t.v[a] * 3 + r, t.v[b] * 3 + c, R(-D[a][b][3 * r + c])});
  }
}
template <class R> void elastic_gradient_at(const Mesh<R>& mesh, const std::vector<V3<R>>& X, std::vector<R>& g) {
  std::vector<double> acc(3 * X.size(), 0.0);
  for (size_t f = 0; f < mesh.triangles.size(); ++f) {
    double gr[3][3] = {};
    arap_face(mesh, X, f, gr);
    const auto& t = mesh.triangles[f];
    for (int a = 0; a < 3; ++a) for (int q = 0; q < 3; ++q) acc[3 * size_t(t.v[a]) + size_t(q)] += gr[a][q];
  }
  bending_at(mesh, X, acc);
  g.assign(acc.size(), R(0));
  for (size_t i = 0; i < acc.size(); ++i) g[i] = R(acc[i]);
}
template <class R> double elastic_energy_at(const Mesh<R>& mesh, const std::vector<V3<R>>& X) {
  double e = 0.0;
  for (size_t f = 0; f < mesh.triangles.size(); ++f) { double gr[3][3] = {}; e += arap_face(mesh, X, f, gr); }
  std::vector<double> unused(3 * X.size(), 0.0);
  return e + bending_at(mesh, X, unused);
}

// Conservative time of impact of one pair along the motion x -> x + e: advance
// by (d - eta) / l until the distance falls to eta = 0.1 d0 (l bounds how fast
// the distance can shrink per unit time). Returns t in [0, 1].
// A pair that already touches (d0 = 0; only a kinematic pin snap makes one)
// cannot be advanced conservatively and does not bound the step.
// With eta_min > 0 (the kinematic pin pass) the move may not bring a pair
// closer than eta_min at all.
// A pair closer than `near` at the start is sampled instead of advanced
// (geometric times 2^-40..2^-1, then 0.5..1 in steps of 1/32): the step is
// allowed up to the last sample before the distance first falls below half
// its starting value (conservative advancement cannot tell such a pair moving
// apart from one closing in).
template <class R> R advance_toi(const std::function<R(R)>& dist, R l, R eta_min = R(0), R near = R(0)) {
  if (!(l > R(0))) return R(1);
  R d0 = dist(R(0));
  if (!(d0 > R(0))) return R(1);
  if (d0 <= eta_min) return R(0);
  if (d0 < near) {
    R prev = 0;
    for (int k = 40; k >= 1; --k) {
      R ts = R(std::ldexp(1.0, -k));
      if (!(dist(ts) >= R(0.5) * d0)) return prev;
      prev = ts;
    }
    for (int k = 17; k <= 32; ++k) {
      R ts = R(double(k) / 32.0);
      if (!(dist(ts) >= R(0.5) * d0)) return prev;
      prev = ts;
    }
    return R(1);
  }
  R eta = std::max(R(0.1) * d0, eta_min), t = 0;
  for (int it = 0; it < 200; ++it) {
    R d = it == 0 ? d0 : dist(t);
    if (d <= eta) return t;
    t += (d - eta) / l;
    if (t >= R(1)) return R(1);
  }
  return t;
}

// Discrete intersection check of one configuration (test infrastructure; the
// reference's CollisionValidator only reads a contact list,
// collision_validator.cpp:133-180, and cannot see a crossing that no contact
// reports). Counts (mesh edge, triangle) pairs that share no vertex and where
// the edge's segment passes through the triangle, over a uniform grid of cell
// `cell`. Segment-triangle test in FP64: the segment's end points lie strictly
// on opposite sides of the triangle's plane and the crossing point lies inside
// the triangle (barycentric coordinates in [0, 1]).
template <class R> long long count_edge_triangle_crossings(const Mesh<R>& m, const std::vector<V3<R>>& x, double cell) {
  if (m.triangles.empty() || m.edges.empty() || !(cell > 0.0)) return 0;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (const auto& p : x) for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], double(p[k])); hi[k] = std::max(hi[k], double(p[k])); }
  long long dims[3];
  for (int k = 0; k < 3; ++k) dims[k] = std::max<long long>(1, std::min<long long>(1 << 10, (long long)((hi[k] - lo[k]) / cell) + 1));
  auto key = [&](long long i, long long j, long long k) { return (i * dims[1] + j) * dims[2] + k; };
  auto cidx = [&](double v, int k) { return std::min<long long>(dims[k] - 1, std::max<long long>(0, (long long)((v - lo[k]) / cell))); };
  std::unordered_map<long long, std::vector<int>> grid;
  for (size_t t = 0; t < m.triangles.size(); ++t) {
    long long a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      double mn = 1e300, mx = -1e300;
      for (int q = 0; q < 3; ++q) { double v = double(x[size_t(m.triangles[t].v[q])][k]); mn = std::min(mn, v); mx = std::max(mx, v); }
      a[k] = cidx(mn, k); b[k] = cidx(mx, k);
    }
    for (long long i = a[0]; i <= b[0]; ++i) for (long long j = a[1]; j <= b[1]; ++j) for (long long k = a[2]; k <= b[2]; ++k) grid[key(i, j, k)].push_back(int(t));
  }
  long long crossings = 0;
  std::vector<int> seen;
  for (const auto& e : m.edges) {
    const V3<R>& P = x[size_t(e.v[0])];
    const V3<R>& Q = x[size_t(e.v[1])];
    long long a[3], b[3];
    for (int k = 0; k < 3; ++k) { a[k] = cidx(std::min(double(P[k]), double(Q[k])), k); b[k] = cidx(std::max(double(P[k]), double(Q[k])), k); }
    seen.clear();
    for (long long i = a[0]; i <= b[0]; ++i) for (long long j = a[1]; j <= b[1]; ++j) for (long long k = a[2]; k <= b[2]; ++k) {
      auto it = grid.find(key(i, j, k));
      if (it != grid.end()) seen.insert(seen.end(), it->second.begin(), it->second.end());
    }
    std::sort(seen.begin(), seen.end());
    seen.erase(std::unique(seen.begin(), seen.end()), seen.end());
    for (int t : seen) {
      const auto& tri = m.triangles[size_t(t)];
      bool shares = false;
      for (int q = 0; q < 3; ++q) if (tri.v[q] == e.v[0] || tri.v[q] == e.v[1]) shares = true;
      if (shares) continue;
      double A[3], B[3], C[3], p0[3], p1[3];
      for (int k = 0; k < 3; ++k) {
        A[k] = x[size_t(tri.v[0])][k]; B[k] = x[size_t(tri.v[1])][k]; C[k] = x[size_t(tri.v[2])][k];
        p0[k] = P[k]; p1[k] = Q[k];
      }
      double u[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]}, w[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
      double nrm[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
      double s0 = nrm[0] * (p0[0] - A[0]) + nrm[1] * (p0[1] - A[1]) + nrm[2] * (p0[2] - A[2]);
      double s1 = nrm[0] * (p1[0] - A[0]) + nrm[1] * (p1[1] - A[1]) + nrm[2] * (p1[2] - A[2]);
      if (!((s0 > 0 && s1 < 0) || (s0 < 0 && s1 > 0))) continue;
      double tt = s0 / (s0 - s1), X[3];
      for (int k = 0; k < 3; ++k) X[k] = p0[k] + tt * (p1[k] - p0[k]) - A[k];
      double uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2], uw = u[0] * w[0] + u[1] * w[1] + u[2] * w[2], ww = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
      double xu = X[0] * u[0] + X[1] * u[1] + X[2] * u[2], xw = X[0] * w[0] + X[1] * w[1] + X[2] * w[2];
      double den = uu * ww - uw * uw;
      if (!(std::fabs(den) > 0.0)) continue;
      double bv = (ww * xu - uw * xw) / den, bw = (uu * xw - uw * xu) / den;
      if (bv >= 0.0 && bw >= 0.0 && bv + bw <= 1.0) ++crossings;
    }
  }
  return crossings;
}

// Diagnostics of the CORRECTED Newton loop (test infrastructure): when
// enabled, every Newton iteration appends the pair that bounded its time of
// impact and the gradient norm it started from.
struct NewtonTrace {
  bool enabled = false;
  struct Row { int kind = -1; int ids[4] = {-1, -1, -1, -1}; double d0 = 0, l = 0, t = 1, gnorm = 0; int below_half = 0; };
  std::vector<Row> rows;
  Row cur;
  static NewtonTrace& get() { static NewtonTrace t; return t; }
};

template <class R> class CorrectedIntegrator {
 public:
  // Pins are energy terms of the implicit solve (corrected_pin_stiffness): no
  // kinematic pre-move. The conservative time of impact bounds every Newton
  // move, so a step whose pins or free vertices travel several edge lengths
  // advances by small fractions over many iterations; such a step is split
  // into k = ceil(extent / (edge / 2)) sub-steps of dt / k (at most 8),
  // extent = max(largest pin move, dt max |v|), with the pin targets
  // interpolated linearly from where the pinned vertices start.
  static int substeps(const Mesh<R>& mesh, const State<R>& st, const Constraints<R>& C, R dt) {
    const std::vector<V3<R>>& x0 = st.positions_safe.size() == st.positions.size() ? st.positions_safe : st.positions;
    double mv = 0.0;
    for (const auto& pin : C.pins) if (pin.active) mv = std::max(mv, double((pin.target_position - x0[size_t(pin.vertex_idx)]).norm()));
    for (const auto& v : st.velocities) mv = std::max(mv, double(dt) * double(v.norm()));
    double edge = double(max_move(mesh)) / 4.0;
    if (!(edge > 0.0) || !(mv > 0.5 * edge)) return 1;
    return int(std::min(8.0, std::ceil(mv / (0.5 * edge))));
  }

  static void step(Mesh<R>& mesh, State<R>& st, Constraints<R>& C, const SimParams<R>& p, std::vector<RigidBody<R>>* rigids, StepStats<R>* stats = nullptr) {
    StepStats<R> local; StepStats<R>& S = stats ? *stats : local;
    S = StepStats<R>();
    const int k = substeps(mesh, st, C, p.dt);
    S.substeps = k;
    if (k == 1) { step_once(mesh, st, C, p, rigids, S); return; }
    const size_t n = st.positions.size();
    const std::vector<V3<R>>& x0 = st.positions_safe.size() == n ? st.positions_safe : st.positions;
    std::vector<V3<R>> start(C.pins.size());
    for (size_t q = 0; q < C.pins.size(); ++q) start[q] = x0[size_t(C.pins[q].vertex_idx)];
    Constraints<R> Cs = C;
    SimParams<R> ps = p;
    ps.dt = R(double(p.dt) / k);
    for (int j = 1; j <= k; ++j) {
      for (size_t q = 0; q < C.pins.size(); ++q)
        Cs.pins[q].target_position = start[q] + (C.pins[q].target_position - start[q]) * R(double(j) / k);
      StepStats<R> Sj;
      step_once(mesh, st, Cs, ps, rigids, Sj);
      S.newton_iters += Sj.newton_iters; S.pcg_iters += Sj.pcg_iters; S.line_search_fail += Sj.line_search_fail;
      S.contacts = std::max(S.contacts, Sj.contacts); S.pcg_not_converged += Sj.pcg_not_converged; S.strain_active = Sj.strain_active;
      S.beta = Sj.beta;
      S.alphas.insert(S.alphas.end(), Sj.alphas.begin(), Sj.alphas.end());
      S.pcg_per_newton.insert(S.pcg_per_newton.end(), Sj.pcg_per_newton.begin(), Sj.pcg_per_newton.end());
    }
  }

  static void step_once(Mesh<R>& mesh, State<R>& st, Constraints<R>& C, const SimParams<R>& p, std::vector<RigidBody<R>>* rigids,
                        StepStats<R>& S) {
    const size_t n = st.positions.size(); const R dt = p.dt;
    std::vector<char> fixed(n, 0);  // no kinematic vertices: pins are springs of the solve
    // The step starts where the previous one ended (or at the caller's own
    // positions): the position update of State::apply_gravity is an explicit,
    // collision-unchecked move, and the implicit predictor below already
    // carries its velocity (x_target = x_n + dt v with v = v_n + g dt).
    if (st.positions_safe.size() == n) st.positions = st.positions_safe;
    std::vector<V3<R>> x_old = st.positions, x_target(n);
    for (size_t i = 0; i < n; ++i) x_target[i] = x_old[i] + st.velocities[i] * dt;
    R beta = 0; int bi = 0;
    // The step starts where the last one ended, so its first Newton system is
    // always solved: with the gradient test alone, a scene whose forces all lie
    // below pcg_tol (a light cloth starting to fall) would never move.
    bool solve_first = true;
    const Csr<R> H_el = base_elastic(mesh);  // constant: built once per step
    while (beta < p.beta_max && bi < 20) {
      R alpha = inner_newton(mesh, st, x_target, fixed, C, p, rigids, S, solve_first, H_el);
      solve_first = false;
      beta = R(double(beta) + (1.0 - double(beta)) * double(alpha));
      ++bi;
      if (alpha < R(1e-6)) { S.line_search_fail++; break; }
    }
    if (beta > R(1e-6)) inner_newton(mesh, st, x_target, fixed, C, p, rigids, S, false, H_el);
    S.beta = beta;
    // v = (x - x_old) / dt: dividing by beta dt (the reference) turns the
    // error-reduction pass of a step whose line search held beta near zero
    // into an arbitrarily large velocity
    for (size_t i = 0; i < n; ++i) st.velocities[i] = (st.positions[i] - x_old[i]) / dt;
    if (p.velocity_damping > R(0)) { R sc = R(1) - std::clamp(p.velocity_damping, R(0), R(1)); for (auto& v : st.velocities) v = v * sc; }
    st.positions_safe = st.positions;
  }

  static Csr<R> base_elastic(const Mesh<R>& mesh) { std::vector<Triplet<R>> el; corrected_elastic_triplets(mesh, el); return Csr<R>::from_triplets(Index(3 * mesh.vertices.size()), el); }

  static void gradient(const Mesh<R>& mesh, const State<R>& st, const std::vector<V3<R>>& x_target, const std::vector<char>& fixed,
                       const std::vector<ContactPair<R>>& contacts, Constraints<R>& C, const SimParams<R>& p, const Csr<R>& H_el, std::vector<R>& g) {
    const size_t n = st.positions.size(); const R dt = p.dt;
    g.assign(3 * n, R(0));
    for (size_t i = 0; i < n; ++i) { R mf = st.masses[i] / (dt * dt); for (int j = 0; j < 3; ++j) g[3 * i + size_t(j)] += mf * (st.positions[i][j] - x_target[i][j]); }
    std::vector<R> ge; elastic_gradient_at(mesh, st.positions, ge);
    for (size_t i = 0; i < g.size(); ++i) g[i] += ge[i];
    if (p.enable_strain_limiting) { strain_rebuild(mesh, st, p, H_el, C, Lookup::INDEXED); strain_gradient(mesh, st, C, p, g); }
    else C.strain_limits.clear();
    for (const auto& c : contacts) {
      R kb = corrected_contact_stiffness(c, st.masses, H_el, p.min_gap);
      if (!in_domain(c.gap, p.contact_gap_max)) continue;
      V3<R> nrm = normalize_or_default(c.normal, p.contact_normal_epsilon);
      R dV = barrier_gradient(c.gap, p.contact_gap_max, kb);
      Index ids[4] = {c.idx0, c.idx1, c.idx2, c.idx3};
      int cnt = std::max(c.vertex_count, 1);
      for (int i = 0; i < cnt; ++i) {
        if (ids[i] < 0 || c.weights[size_t(i)] == R(0)) continue;
        V3<R> add = nrm * (dV * c.weights[size_t(i)]);
        for (int k = 0; k < 3; ++k) g[size_t(ids[i]) * 3 + size_t(k)] += add[k];
      }
    }
    Csr<R> H_tot = H_el;  // walls take k_bar from the elastic + inertia diagonal block
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nrm = normalize_or_default(w.normal, p.contact_normal_epsilon);
      for (size_t vi = 0; vi < n; ++vi) {
        M3<R> Hb = extract_hessian_block(H_el, Index(vi), Lookup::INDEXED);
        R md = st.masses[vi] / (dt * dt);
        Hb(0, 0) += md; Hb(1, 1) += md; Hb(2, 2) += md;
        R gap = nrm.dot(st.positions[vi]) - w.offset;
        R kb = corrected_wall_stiffness(st.masses[vi], gap, w.normal, Hb, p.min_gap);
        if (!in_domain(gap, p.contact_gap_max)) continue;
        R dV = barrier_gradient(gap, p.contact_gap_max, kb);
        for (int k = 0; k < 3; ++k) g[vi * 3 + size_t(k)] += dV * nrm[k];
      }
    }
    for (const auto& pin : C.pins) {
      if (!pin.active || pin.vertex_idx < 0 || size_t(pin.vertex_idx) >= n) continue;
      size_t vi = size_t(pin.vertex_idx);
      R kp = corrected_pin_stiffness(st.masses[vi], dt, extract_hessian_block(H_el, Index(vi), Lookup::INDEXED)(0, 0));
      for (int k = 0; k < 3; ++k) g[3 * vi + size_t(k)] += kp * (st.positions[vi][k] - pin.target_position[k]);
    }
    for (size_t i = 0; i < n; ++i) if (fixed[i]) for (int k = 0; k < 3; ++k) g[3 * i + size_t(k)] = R(0);
  }

  static Csr<R> assemble(const Mesh<R>& mesh, const State<R>& st, const std::vector<char>& fixed, const std::vector<ContactPair<R>>& contacts,
                         Constraints<R>& C, const SimParams<R>& p, const Csr<R>& H_el) {
    const Index n = Index(st.positions.size()); const R dt = p.dt;
    std::vector<Triplet<R>> tr;
    R dinv = R(1) / (dt * dt);
    for (Index row = 0; row < 3 * n; ++row) { R v = st.masses[size_t(row / 3)] * dinv; if (v != R(0)) tr.push_back({row, row, v}); }
    corrected_elastic_triplets(mesh, tr);
    if (p.membrane_hessian) membrane_correction_triplets(mesh, st.positions, tr);
    if (p.enable_strain_limiting) strain_hessian(mesh, st, C, p, tr);
    for (const auto& c : contacts) {
      R kb = corrected_contact_stiffness(c, st.masses, H_el, p.min_gap);
      if (!in_domain(c.gap, p.contact_gap_max)) continue;
      V3<R> nrm = normalize_or_default(c.normal, p.contact_normal_epsilon);
      R d2V = barrier_hessian(c.gap, p.contact_gap_max, kb);
      Index ids[4] = {c.idx0, c.idx1, c.idx2, c.idx3};
      int cnt = std::max(c.vertex_count, 1);
      for (int i = 0; i < cnt; ++i) for (int j = 0; j < cnt; ++j) {
        if (ids[i] < 0 || ids[j] < 0 || c.weights[size_t(i)] == R(0) || c.weights[size_t(j)] == R(0)) continue;
        V3<R> gi = nrm * c.weights[size_t(i)], gj = nrm * c.weights[size_t(j)];
        for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) {
          R v = d2V * (gi[r] * gj[q]);
          if (std::fabs(v) < p.barrier_tolerance) continue;
          tr.push_back({ids[i] * 3 + r, ids[j] * 3 + q, v});
        }
      }
    }
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nrm = normalize_or_default(w.normal, p.contact_normal_epsilon);
      for (Index vi = 0; vi < n; ++vi) {
        M3<R> Hb = extract_hessian_block(H_el, vi, Lookup::INDEXED);
        R md = st.masses[size_t(vi)] / (dt * dt);
        Hb(0, 0) += md; Hb(1, 1) += md; Hb(2, 2) += md;
        R gap = nrm.dot(st.positions[size_t(vi)]) - w.offset;
        R kb = corrected_wall_stiffness(st.masses[size_t(vi)], gap, w.normal, Hb, p.min_gap);
        if (!in_domain(gap, p.contact_gap_max)) continue;
        R d2V = barrier_hessian(gap, p.contact_gap_max, kb);
        for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) { R v = d2V * nrm[r] * nrm[q]; if (std::fabs(v) >= p.barrier_tolerance) tr.push_back({vi * 3 + r, vi * 3 + q, v}); }
      }
    }
    for (const auto& pin : C.pins) {
      if (!pin.active || pin.vertex_idx < 0 || pin.vertex_idx >= n) continue;
      R kp = corrected_pin_stiffness(st.masses[size_t(pin.vertex_idx)], dt, extract_hessian_block(H_el, pin.vertex_idx, Lookup::INDEXED)(0, 0));
      for (int k = 0; k < 3; ++k) tr.push_back({3 * pin.vertex_idx + k, 3 * pin.vertex_idx + k, kp});
    }
    // kinematic pins: drop every entry touching a fixed vertex, unit diagonal
    std::vector<Triplet<R>> kept; kept.reserve(tr.size());
    for (auto& t : tr) if (!fixed[size_t(t.row / 3)] && !fixed[size_t(t.col / 3)]) kept.push_back(t);
    for (Index i = 0; i < n; ++i) if (fixed[size_t(i)]) for (int k = 0; k < 3; ++k) kept.push_back({3 * i + k, 3 * i + k, R(1)});
    return Csr<R>::from_triplets(3 * n, kept);
  }

  // Incremental potential of the CORRECTED Newton system at positions X, with
  // everything `gradient` evaluates at the state's positions frozen there: the
  // contact pairs and their stiffness, the strain-limit constraints and their
  // stiffness, the wall stiffness. Test infrastructure: its central
  // differences at X = st.positions check `gradient` term by term.
  static double energy(const Mesh<R>& mesh, const State<R>& st, const std::vector<V3<R>>& X, const std::vector<V3<R>>& x_target,
                       const std::vector<ContactPair<R>>& contacts, Constraints<R>& C, const SimParams<R>& p, const Csr<R>& H_el) {
    const size_t n = st.positions.size(); const double dt = double(p.dt);
    double E = 0.0;
    for (size_t i = 0; i < n; ++i) {
      double mf = double(st.masses[i]) / (dt * dt);
      for (int k = 0; k < 3; ++k) { double d = double(X[i][k]) - double(x_target[i][k]); E += 0.5 * mf * d * d; }
    }
    E += elastic_energy_at(mesh, X);
    if (p.enable_strain_limiting) {
      strain_rebuild(mesh, st, p, H_el, C, Lookup::INDEXED);
      R tau = to_fraction(p.strain_tau);
      R eps = p.strain_epsilon > R(0) ? to_fraction(p.strain_epsilon) : tau;
      State<R> sx = st; sx.positions = X;
      for (const auto& sc : C.strain_limits) {
        V3<R> F[2]; strain_F(sx, mesh, size_t(sc.face_idx), F);
        Svd32<R> sv; if (!svd32(F, sv)) continue;
        R gap = (R(1) + tau + eps) - sv.sigma[std::clamp(sc.singular_index, 0, 1)];
        E += double(barrier_energy(gap, eps, sc.stiffness));
      }
    }
    for (const auto& c : contacts) {
      if (c.type != ContactType::POINT_TRIANGLE && c.type != ContactType::EDGE_EDGE) continue;
      R kb = corrected_contact_stiffness(c, st.masses, H_el, p.min_gap);
      R d; V3<R> nm, wp, wq;
      if (c.type == ContactType::POINT_TRIANGLE) narrow_pt(X[size_t(c.idx0)], X[size_t(c.idx1)], X[size_t(c.idx2)], X[size_t(c.idx3)], d, nm, wp, wq);
      else narrow_ee(X[size_t(c.idx0)], X[size_t(c.idx1)], X[size_t(c.idx2)], X[size_t(c.idx3)], d, nm, wp, wq);
      E += double(barrier_energy(d, p.contact_gap_max, kb));
    }
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nrm = normalize_or_default(w.normal, p.contact_normal_epsilon);
      for (size_t vi = 0; vi < n; ++vi) {
        M3<R> Hb = extract_hessian_block(H_el, Index(vi), Lookup::INDEXED);
        R md = st.masses[vi] / (p.dt * p.dt);
        Hb(0, 0) += md; Hb(1, 1) += md; Hb(2, 2) += md;
        R kb = corrected_wall_stiffness(st.masses[vi], nrm.dot(st.positions[vi]) - w.offset, w.normal, Hb, p.min_gap);
        E += double(barrier_energy(nrm.dot(X[vi]) - w.offset, p.contact_gap_max, kb));
      }
    }
    for (const auto& pin : C.pins) {
      if (!pin.active || pin.vertex_idx < 0 || size_t(pin.vertex_idx) >= n) continue;
      size_t vi = size_t(pin.vertex_idx);
      double kp = double(corrected_pin_stiffness(st.masses[vi], p.dt, extract_hessian_block(H_el, Index(vi), Lookup::INDEXED)(0, 0)));
      for (int k = 0; k < 3; ++k) { double d = double(X[vi][k]) - double(pin.target_position[k]); E += 0.5 * kp * d * d; }
    }
    return E;
  }

  // Conservative time of impact along ext (line search of the CORRECTED step).
  static R toi(const Mesh<R>& mesh, const std::vector<V3<R>>& x, const std::vector<V3<R>>& ext, const std::vector<char>& fixed,
               const Constraints<R>& C, const std::vector<RigidBody<R>>* rigids, R eta_min = R(0), R near = R(0)) {
    const size_t n = x.size();
    R t = 1;
    for (const auto& w : C.walls) {
      if (!w.active) continue;
      V3<R> nn = w.normal.normalized();
      for (size_t i = 0; i < n; ++i) {
        if (fixed[i]) continue;
        R dn = nn.dot(ext[i]);
        if (!(dn < R(0))) continue;
        R gap = nn.dot(x[i]) - w.offset;
        t = std::min(t, std::max(gap, R(0)) / (-dn));
      }
    }
    std::vector<V3<R>> x1(n);
    for (size_t i = 0; i < n; ++i) x1[i] = x[i] + ext[i];
    std::vector<std::pair<int, int>> vt, ee;
    candidates(mesh, x, &x1, R(0), vt, ee);
    auto L = [&](int i) { return ext[size_t(i)].norm(); };
    // additive CCD: the distance depends on the relative motion only, so the
    // rate bound comes from the displacements minus the pair's mean
    auto Lrel = [&](int i, const V3<R>& mean) { return (ext[size_t(i)] - mean).norm(); };
    // pairs on the host's cores, each pair's time of impact computed as one
    // thread computes it; the minimum (and the trace) taken in pair order
    auto pt_pair = [&](size_t k, R* d0_out) {
      const auto& pr = vt[k];
      const auto& tri = mesh.triangles[size_t(pr.second)];
      int v = pr.first, a = tri.v[0], b = tri.v[1], c = tri.v[2];
      V3<R> mean = (ext[size_t(v)] + ext[size_t(a)] + ext[size_t(b)] + ext[size_t(c)]) * R(0.25);
      R l = Lrel(v, mean) + std::max(Lrel(a, mean), std::max(Lrel(b, mean), Lrel(c, mean)));
      auto dist = [&](R s) { R d; V3<R> nm, wp, wq; narrow_pt(x[size_t(v)] + ext[size_t(v)] * s, x[size_t(a)] + ext[size_t(a)] * s,
                                                              x[size_t(b)] + ext[size_t(b)] * s, x[size_t(c)] + ext[size_t(c)] * s, d, nm, wp, wq); return d; };
      if (d0_out) *d0_out = dist(R(0));
      return std::make_pair(advance_toi<R>(dist, l, eta_min, near), l);
    };
    auto ee_pair = [&](size_t k, R* d0_out) {
      const auto& pr = ee[k];
      const Edge &e1 = mesh.edges[size_t(pr.first)], &e2 = mesh.edges[size_t(pr.second)];
      int a = e1.v[0], b = e1.v[1], c = e2.v[0], d = e2.v[1];
      V3<R> mean = (ext[size_t(a)] + ext[size_t(b)] + ext[size_t(c)] + ext[size_t(d)]) * R(0.25);
      R l = std::max(Lrel(a, mean), Lrel(b, mean)) + std::max(Lrel(c, mean), Lrel(d, mean));
      auto dist = [&](R s) { R dd; V3<R> nm, wp, wq; narrow_ee(x[size_t(a)] + ext[size_t(a)] * s, x[size_t(b)] + ext[size_t(b)] * s,
                                                               x[size_t(c)] + ext[size_t(c)] * s, x[size_t(d)] + ext[size_t(d)] * s, dd, nm, wp, wq); return dd; };
      if (d0_out) *d0_out = dist(R(0));
      return std::make_pair(advance_toi<R>(dist, l, eta_min, near), l);
    };
    std::vector<R> tvt(vt.size()), tee(ee.size());
    parallel_for((long long)vt.size(), [&](long long k) { tvt[size_t(k)] = pt_pair(size_t(k), nullptr).first; });
    parallel_for((long long)ee.size(), [&](long long k) { tee[size_t(k)] = ee_pair(size_t(k), nullptr).first; });
    auto& trace = NewtonTrace::get();
    for (int kind = 0; kind < 2; ++kind) {
      const std::vector<R>& tv = kind == 0 ? tvt : tee;
      for (size_t k = 0; k < tv.size(); ++k) {
        R tp = tv[k];
        if (trace.enabled) {
          if (tp < R(0.5)) trace.cur.below_half++;
          if (tp < t) {
            R d0 = 0;
            auto res = kind == 0 ? pt_pair(k, &d0) : ee_pair(k, &d0);
            trace.cur.kind = kind; trace.cur.d0 = double(d0); trace.cur.l = double(res.second); trace.cur.t = double(tp);
            if (kind == 0) {
              const auto& tri = mesh.triangles[size_t(vt[k].second)];
              trace.cur.ids[0] = vt[k].first; trace.cur.ids[1] = tri.v[0]; trace.cur.ids[2] = tri.v[1]; trace.cur.ids[3] = tri.v[2];
            } else {
              const Edge &e1 = mesh.edges[size_t(ee[k].first)], &e2 = mesh.edges[size_t(ee[k].second)];
              trace.cur.ids[0] = e1.v[0]; trace.cur.ids[1] = e1.v[1]; trace.cur.ids[2] = e2.v[0]; trace.cur.ids[3] = e2.v[1];
            }
          }
        }
        t = std::min(t, tp);
      }
    }
    if (rigids) {
      for (const auto& body : *rigids) {
        auto wv = body.world_vertices();
        for (size_t v = 0; v < n; ++v) {
          R l = L(int(v));
          if (!(l > R(0))) continue;
          for (const auto& tr : body.tris) {
            AABB<R> tb; tb.expand(wv[size_t(tr.v[0])]); tb.expand(wv[size_t(tr.v[1])]); tb.expand(wv[size_t(tr.v[2])]);
            AABB<R> pb = point_box(x[v]); pb.expand(point_box(x1[v]));
            if (!pb.overlaps(tb)) continue;
            auto dist = [&](R s) { R d; V3<R> nm, wp, wq; narrow_pt(x[v] + ext[v] * s, wv[size_t(tr.v[0])], wv[size_t(tr.v[1])], wv[size_t(tr.v[2])], d, nm, wp, wq); return d; };
            t = std::min(t, advance_toi<R>(dist, l));
          }
        }
      }
    }
    return t;
  }

  static R max_move(const Mesh<R>& mesh) {
    if (mesh.edges.empty()) return std::numeric_limits<R>::max();
    double sum = 0;
    for (const auto& e : mesh.edges) sum += double((mesh.vertices[size_t(e.v[1])] - mesh.vertices[size_t(e.v[0])]).norm());
    return R(4.0 * sum / double(mesh.edges.size()));
  }

  static R inner_newton(const Mesh<R>& mesh, State<R>& st, const std::vector<V3<R>>& x_target, const std::vector<char>& fixed,
                        Constraints<R>& C, const SimParams<R>& p, std::vector<RigidBody<R>>* rigids, StepStats<R>& S, bool solve_first,
                        const Csr<R>& H_el) {
    const size_t n = st.positions.size();
    const R lmax = max_move(mesh);
    for (int it = 0; it < p.max_newton_steps; ++it) {
      auto contacts = detect_corrected(mesh, st.positions, rigids, p.contact_gap_max);
      S.contacts = std::max(S.contacts, int(contacts.size()));
      std::vector<R> g;
      gradient(mesh, st, x_target, fixed, contacts, C, p, H_el, g);
      R gn = 0; for (R e : g) gn = std::max(gn, std::fabs(e));
      if (gn < p.pcg_tol && !(solve_first && it == 0)) return R(1);
      S.newton_iters++;
      if (NewtonTrace::get().enabled) { NewtonTrace::get().cur = NewtonTrace::Row(); NewtonTrace::get().cur.gnorm = double(gn); }
      Csr<R> H = assemble(mesh, st, fixed, contacts, C, p, H_el);
      std::vector<R> d(3 * n, R(0)), ng(3 * n);
      for (size_t i = 0; i < 3 * n; ++i) ng[i] = -g[i];
      auto pr = pcg_solve(H, ng, d, p.pcg_tol, p.pcg_max_iters, true);
      S.pcg_iters += pr.iters; S.pcg_per_newton.push_back(pr.iters);
      if (!pr.converged) S.pcg_not_converged++;
      // extended direction 1.25 d, clipped vertex by vertex to length lmax:
      // no vertex moves more than lmax in one Newton iteration, and a single
      // runaway entry of d does not scale the whole step down
      std::vector<V3<R>> ext(n);
      for (size_t i = 0; i < n; ++i) {
        ext[i] = fixed[i] ? V3<R>() : V3<R>(d[3 * i], d[3 * i + 1], d[3 * i + 2]) * R(1.25);
        R len = ext[i].norm();
        if (len > lmax) ext[i] = ext[i] * (lmax / len);
      }
      R alpha = std::min(R(1), toi(mesh, st.positions, ext, fixed, C, rigids, R(0), R(0)));
      if (NewtonTrace::get().enabled) NewtonTrace::get().rows.push_back(NewtonTrace::get().cur);
      S.alphas.push_back(alpha);
      if (alpha < R(1e-8)) return R(0);
      for (size_t i = 0; i < n; ++i) if (!fixed[i]) st.positions[i] = st.positions[i] + ext[i] * (alpha / R(1.25));
      if (alpha > R(0.99)) return R(1);
    }
    return R(0.5);
  }
};

}  // namespace ando_oracle
