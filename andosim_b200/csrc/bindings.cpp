// bindings.cpp -- the `ando_barrier_core` Python module, a drop-in for the
// reference's pybind11 module (src/py/bindings.cpp:27-633).
//
// Class names, method names, argument order, defaults and error types follow
// the reference so the Blender add-on and the demos load it unchanged. The
// objects hold host mirrors of the mesh and state; Integrator.step and
// Integrator.compute_contacts run on the GPU through the C ABI of
// include/ando_gpu.h. The state lives on the device between steps and is
// copied back only when Python reads it. There is no CPU fallback: without a
// usable B200 the GPU calls raise RuntimeError.
//
// Arrays are returned as float32, the reference's default Real (types.h:12-16).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_set>
#include <cstring>
#include <vector>

#include "../../include/ando_gpu.h"

namespace py = pybind11;

namespace {

using Real = float;
using F32 = py::array_t<float>;
template <class T> using Arr = py::array_t<T, py::array::c_style | py::array::forcecast>;

void check(int32_t rc, const char* what) {
  if (rc != ANDO_OK) throw std::runtime_error(std::string(what) + ": " + ando_status_string(rc) + " (" + ando_last_error() + ")");
}

struct V3 { double x = 0, y = 0, z = 0; };
static_assert(sizeof(V3) == 3 * sizeof(double), "V3 must be three packed doubles (bulk copies of state arrays)");
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double norm(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalized(V3 a) { double n2 = dot(a, a); return n2 > 0 ? mul(a, 1.0 / std::sqrt(n2)) : a; }

// ------------------------------------------------------------------ objects
struct Material {
  Real youngs_modulus = 1e6f, poisson_ratio = 0.3f, density = 1000.0f, thickness = 0.001f, bending_stiffness = 0.0f;
};

struct SimParams {
  Real dt = 0.002f, beta_max = 0.25f;
  int min_newton_steps = 2, max_newton_steps = 8, friction_min_newton_steps = 32;
  Real pcg_tol = 1e-3f;
  int pcg_max_iters = 1000;
  Real contact_gap_max = 0.001f, wall_gap = 0.001f;
  bool enable_ccd = true;
  Real contact_normal_epsilon = 1e-8f, barrier_tolerance = 1e-12f;
  bool enable_friction = false;
  Real friction_mu = 0.1f, friction_epsilon = 1e-5f, friction_tangent_threshold = 1e-6f;
  Real velocity_damping = 0.0f, contact_restitution = 0.0f;
  bool enable_strain_limiting = false;
  Real strain_limit = 0.05f, strain_tau = 0.05f, strain_epsilon = 0.0f, strain_svd_epsilon = 1e-6f;
  Real hessian_epsilon = 1e-8f, min_gap = 1e-8f;
  // GPU-only knobs
  std::string semantics = "reference";
  std::string preconditioner = "block_jacobi";
  int precond_refresh = 1;
  std::string membrane_hessian = "fixed_rotation";   // CORRECTED: or "projected" (ando_params.membrane_hessian)
};

struct Triangle { int32_t v[3] = {-1, -1, -1}; };

// Mesh with its rest state (mesh.cpp:8-98), computed once on the host.
struct Mesh {
  std::vector<V3> vertices;
  std::vector<int32_t> tris;      // 3T
  std::vector<int32_t> edges;     // 2E, first-seen order
  std::vector<double> dm_inv;     // 4T
  std::vector<double> areas;      // T
  Material material;
  uint64_t topo_version = 0, vert_version = 0;
  static uint64_t next_version() { static uint64_t v = 0; return ++v; }

  size_t nv() const { return vertices.size(); }
  size_t nt() const { return tris.size() / 3; }

  void compute_rest_state() {
    // unique edges (mesh.cpp:77-98)
    edges.clear();
    std::unordered_set<uint64_t> seen;
    for (size_t f = 0; f < nt(); ++f)
      for (int i = 0; i < 3; ++i) {
        int32_t a = tris[3 * f + i], b = tris[3 * f + (i + 1) % 3];
        int32_t lo = std::min(a, b), hi = std::max(a, b);
        uint64_t key = (uint64_t(uint32_t(lo)) << 32) | uint64_t(uint32_t(hi));
        if (seen.insert(key).second) { edges.push_back(lo); edges.push_back(hi); }
      }
    dm_inv.assign(4 * nt(), 0.0);
    areas.assign(nt(), 0.0);
    const double eps = 1e-12;
    for (size_t f = 0; f < nt(); ++f) {
      V3 v0 = vertices[tris[3 * f]], v1 = vertices[tris[3 * f + 1]], v2 = vertices[tris[3 * f + 2]];
      V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
      double l1 = dot(e1, e1), l2 = dot(e2, e2);
      if (l1 < eps || l2 < eps) continue;
      V3 n = cross(e1, e2);
      double nl = norm(n);
      if (nl < eps) continue;
      areas[f] = nl * 0.5;
      V3 nu = mul(n, 1.0 / nl), t1 = mul(e1, 1.0 / std::sqrt(l1)), t2 = cross(nu, t1);
      double a = dot(e1, t1), b = dot(e2, t1), c = dot(e1, t2), d = dot(e2, t2);
      double det = a * d - b * c, inv = 1.0 / det;
      dm_inv[4 * f] = d * inv; dm_inv[4 * f + 1] = -b * inv; dm_inv[4 * f + 2] = -c * inv; dm_inv[4 * f + 3] = a * inv;
    }
    topo_version = next_version();
    vert_version = next_version();
  }
};

struct RigidBody {
  std::vector<double> local;      // 3nv
  std::vector<int32_t> tris;      // 3nt
  double mass = 1.0;
  double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, Iinv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  double pos[3] = {0, 0, 0}, R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, lin[3] = {0, 0, 0}, ang[3] = {0, 0, 0};
  double acc_f[3] = {0, 0, 0}, acc_t[3] = {0, 0, 0};

  V3 mv(const double* M, V3 v) const { return {M[0] * v.x + M[1] * v.y + M[2] * v.z, M[3] * v.x + M[4] * v.y + M[5] * v.z, M[6] * v.x + M[7] * v.y + M[8] * v.z}; }
  V3 iworld_inv(V3 v) const {
    V3 t{R[0] * v.x + R[3] * v.y + R[6] * v.z, R[1] * v.x + R[4] * v.y + R[7] * v.z, R[2] * v.x + R[5] * v.y + R[8] * v.z};
    return mv(R, mv(Iinv, t));
  }
  // rigid_body.cpp:11-91
  void initialize(const std::vector<V3>& verts, const std::vector<int32_t>& t, double density) {
    tris = t;
    if (verts.empty()) { local.clear(); mass = 0; std::fill(I, I + 9, 0.0); std::fill(Iinv, Iinv + 9, 0.0); return; }
    V3 c{};
    for (auto& v : verts) c = add(c, v);
    c = mul(c, 1.0 / double(verts.size()));
    local.resize(3 * verts.size());
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (size_t i = 0; i < verts.size(); ++i) {
      V3 l = sub(verts[i], c);
      local[3 * i] = l.x; local[3 * i + 1] = l.y; local[3 * i + 2] = l.z;
      V3 w = add(l, c);
      lo[0] = std::min(lo[0], w.x); lo[1] = std::min(lo[1], w.y); lo[2] = std::min(lo[2], w.z);
      hi[0] = std::max(hi[0], w.x); hi[1] = std::max(hi[1], w.y); hi[2] = std::max(hi[2], w.z);
    }
    pos[0] = c.x; pos[1] = c.y; pos[2] = c.z;
    double Rid[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::copy(Rid, Rid + 9, R);
    std::fill(lin, lin + 3, 0.0); std::fill(ang, ang + 3, 0.0);
    double ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    double vol = std::max(ex, 1e-6) * std::max(ey, 1e-6) * std::max(ez, 1e-6);
    mass = std::max(density * vol, 1e-3);
    std::fill(I, I + 9, 0.0);
    I[0] = (mass / 12.0) * (ey * ey + ez * ez); I[4] = (mass / 12.0) * (ex * ex + ez * ez); I[8] = (mass / 12.0) * (ex * ex + ey * ey);
    for (int k : {0, 4, 8}) if (I[k] < 1e-6) I[k] = 1e-6;
    std::fill(Iinv, Iinv + 9, 0.0);
    Iinv[0] = 1.0 / I[0]; Iinv[4] = 1.0 / I[4]; Iinv[8] = 1.0 / I[8];
    std::fill(acc_f, acc_f + 3, 0.0); std::fill(acc_t, acc_t + 3, 0.0);
  }
  std::vector<V3> world() const {
    std::vector<V3> o(local.size() / 3);
    for (size_t i = 0; i < o.size(); ++i) {
      V3 l{local[3 * i], local[3 * i + 1], local[3 * i + 2]};
      V3 r = mv(R, l);
      o[i] = {pos[0] + r.x, pos[1] + r.y, pos[2] + r.z};
    }
    return o;
  }
  void apply_impulse(V3 p, V3 J) {
    if (mass <= 0) return;
    for (int k = 0; k < 3; ++k) lin[k] += (k == 0 ? J.x : k == 1 ? J.y : J.z) / mass;
    V3 dw = iworld_inv(cross(sub(p, V3{pos[0], pos[1], pos[2]}), J));
    ang[0] += dw.x; ang[1] += dw.y; ang[2] += dw.z;
  }
  // rigid_body.cpp:151-176
  void integrate(double dt) {
    if (mass <= 0) return;
    for (int k = 0; k < 3; ++k) lin[k] += (acc_f[k] / mass) * dt;
    V3 aa = iworld_inv(V3{acc_t[0], acc_t[1], acc_t[2]});
    ang[0] += aa.x * dt; ang[1] += aa.y * dt; ang[2] += aa.z * dt;
    for (int k = 0; k < 3; ++k) pos[k] += lin[k] * dt;
    V3 w{ang[0], ang[1], ang[2]};
    double wn = norm(w);
    if (wn > 1e-8) {
      double th = wn * dt; V3 a = mul(w, 1.0 / wn);
      double c = std::cos(th), s = std::sin(th), t = 1.0 - c;
      double dR[9] = {t * a.x * a.x + c, t * a.x * a.y - s * a.z, t * a.x * a.z + s * a.y,
                      t * a.x * a.y + s * a.z, t * a.y * a.y + c, t * a.y * a.z - s * a.x,
                      t * a.x * a.z - s * a.y, t * a.y * a.z + s * a.x, t * a.z * a.z + c};
      double R2[9];
      for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) R2[3 * r + q] = dR[3 * r] * R[q] + dR[3 * r + 1] * R[3 + q] + dR[3 * r + 2] * R[6 + q];
      std::copy(R2, R2 + 9, R);
    }
    std::fill(acc_f, acc_f + 3, 0.0); std::fill(acc_t, acc_t + 3, 0.0);
  }
  ando_rigid to_abi() const {
    ando_rigid r;
    r.num_vertices = int32_t(local.size() / 3); r.num_triangles = int32_t(tris.size() / 3);
    r.local_vertices = local.data(); r.triangles = tris.data(); r.mass = mass;
    std::copy(Iinv, Iinv + 9, r.inertia_body_inv); std::copy(pos, pos + 3, r.position); std::copy(R, R + 9, r.rotation);
    std::copy(lin, lin + 3, r.linear_velocity); std::copy(ang, ang + 3, r.angular_velocity);
    return r;
  }
  void from_abi(const ando_rigid& r) {
    std::copy(r.position, r.position + 3, pos); std::copy(r.rotation, r.rotation + 9, R);
    std::copy(r.linear_velocity, r.linear_velocity + 3, lin); std::copy(r.angular_velocity, r.angular_velocity + 3, ang);
    std::fill(acc_f, acc_f + 3, 0.0); std::fill(acc_t, acc_t + 3, 0.0);
  }
};

// Simulation state with a device mirror. `dev_x` / `dev_v` / `start_stale`:
// the device copy of the positions / velocities / step start is newer and is
// downloaded only when the host reads that array; `host_dirty`: the host copy
// changed and must be uploaded before the next GPU call.
struct State {
  std::vector<V3> x, v, xp;
  std::vector<V3> start;          // CORRECTED: where the next step starts (ando_state_set_start)
  std::vector<double> m;
  ando_ctx ctx = nullptr;
  uint64_t topo = 0, verts = 0, weights = 0;
  bool dev_x = false, dev_v = false, start_stale = false, host_dirty = true, masses_dirty = true;
  // The contact list the context holds on the device: its id (0: none, or
  // replaced since) and length. compute_contacts stamps the Contact objects it
  // returns with the id and their position, so CollisionValidator can reduce
  // that list on the device instead of downloading the state.
  uint64_t contact_list = 0;
  size_t contact_count = 0;
  static uint64_t next_contact_list() { static uint64_t n = 0; return ++n; }
  // the device holds this state's current positions, velocities and masses
  bool device_current() const { return ctx && !host_dirty && !masses_dirty; }
  ando_step_stats last{};

  State() = default;
  State(const State& o) : x(o.x), v(o.v), xp(o.xp), start(o.start), m(o.m) {}
  ~State() { if (ctx) ando_ctx_destroy(ctx); }

  size_t nv() const { return x.size(); }
  static int& device() { static int d = 0; return d; }
  // Learned-preconditioner weights shared by every state (set_precond_weights);
  // a state loads them into its context when it first steps with them.
  static std::vector<float>& precond_weights() { static std::vector<float> w; return w; }
  static uint64_t& precond_version() { static uint64_t v = 0; return v; }
  void bind_weights() {
    if (weights == precond_version() || precond_weights().empty()) return;
    check(ando_ctx_set_precond_weights(ctx, precond_weights().data(), int32_t(precond_weights().size())), "preconditioner weights");
    weights = precond_version();
  }

  void mark_device_newer() { dev_x = dev_v = start_stale = true; }
  // V3 is three packed doubles, so the host arrays are downloaded into directly.
  static double* raw(std::vector<V3>& a) { return reinterpret_cast<double*>(a.data()); }
  void sync_x() {
    if (!dev_x || !ctx) return;
    x.resize(nv());
    check(ando_state_download(ctx, raw(x), nullptr, int32_t(nv())), "state download");
    dev_x = false;
  }
  void sync_v() {
    if (!dev_v || !ctx) return;
    v.resize(nv());
    check(ando_state_download(ctx, nullptr, raw(v), int32_t(nv())), "state download");
    dev_v = false;
  }
  void sync_start() {
    if (!start_stale || !ctx) return;
    start.resize(nv());
    check(ando_state_get_start(ctx, raw(start), int32_t(nv())), "state start");
    start_stale = false;
  }
  void sync_host() { sync_x(); sync_v(); sync_start(); }
  static std::vector<double> flat(const std::vector<V3>& a) {
    std::vector<double> o(3 * a.size());
    for (size_t i = 0; i < a.size(); ++i) { o[3 * i] = a[i].x; o[3 * i + 1] = a[i].y; o[3 * i + 2] = a[i].z; }
    return o;
  }
  // Make the device hold this mesh and this state.
  void bind(const Mesh& mesh) {
    if (mesh.nv() != nv()) throw std::runtime_error("mesh and state have different vertex counts");
    if (!ctx) check(ando_ctx_create(State::device(), &ctx), "GPU context");
    if (topo != mesh.topo_version) {
      sync_host();
      std::vector<double> mv = flat(mesh.vertices);
      ando_material mt{mesh.material.youngs_modulus, mesh.material.poisson_ratio, mesh.material.density, mesh.material.thickness,
                       mesh.material.bending_stiffness};
      check(ando_mesh_upload(ctx, mv.data(), int32_t(mesh.nv()), mesh.tris.data(), int32_t(mesh.nt()), mesh.areas.data(),
                             mesh.dm_inv.data(), &mt), "mesh upload");
      topo = mesh.topo_version; verts = mesh.vert_version;
      host_dirty = true; masses_dirty = true;
      contact_list = 0;
    } else if (verts != mesh.vert_version) {
      std::vector<double> mv = flat(mesh.vertices);
      check(ando_mesh_set_vertices(ctx, mv.data(), int32_t(mesh.nv())), "mesh vertices");
      verts = mesh.vert_version;
    }
    if (host_dirty || masses_dirty) {
      std::vector<double> fx = flat(x), fv = flat(v), fp = flat(xp);
      check(ando_state_upload(ctx, fx.data(), fv.data(), fp.data(), m.data(), int32_t(nv())), "state upload");
      host_dirty = false; masses_dirty = false;
      contact_list = 0;
      if (start.size() == nv()) {     // the upload made x the start; put the real one back
        std::vector<double> fs = flat(start);
        check(ando_state_set_start(ctx, fs.data(), int32_t(nv())), "state start");
      }
    }
  }
};

struct Pin { int32_t vertex; V3 target; bool active = true; };
struct Wall { V3 normal; double offset, gap; bool active = true; };
struct Constraints {
  std::vector<Pin> pins;
  std::vector<Wall> walls;
};

enum class ContactType { POINT_TRIANGLE = 0, EDGE_EDGE = 1, WALL = 2, RIGID_POINT_TRIANGLE = 3 };
// list / pos: which device contact list this contact was read from (State::contact_list) and where
struct Contact { ando_contact c{}; uint64_t list = 0; int32_t pos = -1; };

// --------------------------------------------------------------- diagnostics
struct EnergyDiagnostics {
  Real kinetic_energy = 0, elastic_energy = 0, barrier_energy = 0, total_energy = 0;
  V3 linear_momentum, angular_momentum;
  Real max_velocity = 0, max_acceleration = 0;
  int num_contacts = 0, num_pins = 0;
  Real energy_drift_percent = 0, energy_drift_absolute = 0;
  void update_drift(Real prev) {
    if (prev > 1e-12f) { energy_drift_absolute = total_energy - prev; energy_drift_percent = (energy_drift_absolute / prev) * 100.0f; }
    else { energy_drift_absolute = 0; energy_drift_percent = 0; }
  }
};

struct CollisionMetrics {
  int num_point_triangle = 0, num_edge_edge = 0, num_wall = 0, num_total_contacts = 0;
  Real min_gap = 0, max_gap = 0, avg_gap = 0;
  int num_penetrations = 0;
  Real max_penetration = 0, avg_penetration = 0;
  bool ccd_enabled = false;
  int num_ccd_contacts = 0, num_broad_phase_contacts = 0;
  Real ccd_effectiveness = 0, max_relative_velocity = 0, avg_relative_velocity = 0;
  bool has_tunneling = false, has_major_penetration = false, is_stable = true;
  // collision_validator.cpp:97-115
  int quality_level() const {
    if (has_tunneling) return 3;
    if (has_major_penetration) return 3;
    if (max_penetration > 0.0001f) return 2;
    if (num_penetrations > 0) return 1;
    return 0;
  }
  const char* quality_description() const {
    switch (quality_level()) {
      case 0: return "Excellent - No penetrations";
      case 1: return "Good - Tiny penetrations (<0.1mm)";
      case 2: return "Warning - Minor penetrations detected";
      case 3: return "Error - Major penetrations or tunneling";
      default: return "Unknown";
    }
  }
};

// Elasticity on mesh.vertices (elasticity.cpp:7-61): energy and gradient.
double elastic_energy(const Mesh& me) {
  double mu = double(me.material.youngs_modulus) / (2.0 * (1.0 + double(me.material.poisson_ratio)));
  double e = 0;
  for (size_t f = 0; f < me.nt(); ++f) {
    V3 v0 = me.vertices[me.tris[3 * f]], v1 = me.vertices[me.tris[3 * f + 1]], v2 = me.vertices[me.tris[3 * f + 2]];
    V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    V3 n = normalized(cross(e1, e2)), t1 = normalized(e1), t2 = cross(n, t1);
    double Ds00 = dot(e1, t1), Ds01 = dot(e2, t1), Ds10 = dot(e1, t2), Ds11 = dot(e2, t2);
    const double* D = &me.dm_inv[4 * f];
    double F00 = Ds00 * D[0] + Ds01 * D[2] - 1.0, F01 = Ds00 * D[1] + Ds01 * D[3], F10 = Ds10 * D[0] + Ds11 * D[2], F11 = Ds10 * D[1] + Ds11 * D[3] - 1.0;
    double k = me.areas[f] * me.material.thickness * mu;
    e += k * (F00 * F00 + F01 * F01 + F10 * F10 + F11 * F11);
  }
  return e;
}
std::vector<double> elastic_gradient(const Mesh& me) {
  double mu = double(me.material.youngs_modulus) / (2.0 * (1.0 + double(me.material.poisson_ratio)));
  std::vector<double> g(3 * me.nv(), 0.0);
  for (size_t f = 0; f < me.nt(); ++f) {
    int i0 = me.tris[3 * f], i1 = me.tris[3 * f + 1], i2 = me.tris[3 * f + 2];
    V3 e1 = sub(me.vertices[i1], me.vertices[i0]), e2 = sub(me.vertices[i2], me.vertices[i0]);
    V3 n = normalized(cross(e1, e2)), t1 = normalized(e1), t2 = cross(n, t1);
    double Ds00 = dot(e1, t1), Ds01 = dot(e2, t1), Ds10 = dot(e1, t2), Ds11 = dot(e2, t2);
    const double* D = &me.dm_inv[4 * f];
    double F00 = Ds00 * D[0] + Ds01 * D[2], F01 = Ds00 * D[1] + Ds01 * D[3], F10 = Ds10 * D[0] + Ds11 * D[2], F11 = Ds10 * D[1] + Ds11 * D[3];
    double tk = 2.0 * me.areas[f] * me.material.thickness * mu;
    double P00 = tk * (F00 - 1), P01 = tk * F01, P10 = tk * F10, P11 = tk * (F11 - 1);
    double H00 = P00 * D[0] + P01 * D[1], H01 = P00 * D[2] + P01 * D[3], H10 = P10 * D[0] + P11 * D[1], H11 = P10 * D[2] + P11 * D[3];
    V3 f1 = add(mul(t1, H00), mul(t2, H10)), f2 = add(mul(t1, H01), mul(t2, H11)), f0 = mul(add(f1, f2), -1.0);
    const V3 fs[3] = {f0, f1, f2};
    const int ids[3] = {i0, i1, i2};
    for (int a = 0; a < 3; ++a) { g[3 * ids[a]] += fs[a].x; g[3 * ids[a] + 1] += fs[a].y; g[3 * ids[a] + 2] += fs[a].z; }
  }
  return g;
}

// Elasticity::compute_hessian (elasticity.cpp:63-91, face_hessian at :135-181):
// per face the 3 x 3 blocks c_ab diag(1, 1, 0) of K = k Dm^-T Dm^-1, each made
// SPD by clamping its eigenvalues at 1e-8 (stiffness.cpp:236-254; the blocks
// are diagonal, so the clamp gives diag(max(c, 1e-8), max(c, 1e-8), 1e-8)).
// 81 (row, col, value) triplets per face, in the reference's order.
std::vector<std::tuple<int, int, float>> elastic_hessian_triplets(const Mesh& me) {
  double mu = double(me.material.youngs_modulus) / (2.0 * (1.0 + double(me.material.poisson_ratio)));
  std::vector<std::tuple<int, int, float>> out;
  out.reserve(81 * me.nt());
  for (size_t f = 0; f < me.nt(); ++f) {
    const double* D = &me.dm_inv[4 * f];
    double k = me.areas[f] * me.material.thickness * mu;
    // K = k Dm^-T Dm^-1 (2 x 2, symmetric)
    double K00 = k * (D[0] * D[0] + D[2] * D[2]), K01 = k * (D[0] * D[1] + D[2] * D[3]), K11 = k * (D[1] * D[1] + D[3] * D[3]);
    const double c[3][3] = {{K00 + K11 + 2.0 * K01, -K00, -K11}, {-K00, K00, -K01}, {-K11, -K01, K11}};
    const int ids[3] = {me.tris[3 * f], me.tris[3 * f + 1], me.tris[3 * f + 2]};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double d = std::max(c[a][b], 1e-8);
        const double blk[3] = {d, d, 1e-8};
        for (int r = 0; r < 3; ++r)
          for (int q = 0; q < 3; ++q) out.emplace_back(3 * ids[a] + r, 3 * ids[b] + q, float(r == q ? blk[r] : 0.0));
      }
  }
  return out;
}

// ------------------------------------------------------------ conversions
std::vector<V3> to_v3(py::object o, const char* what) {
  auto a = Arr<double>::ensure(o);
  if (!a || a.ndim() != 2 || a.shape(1) != 3) throw py::value_error(std::string(what) + " must be an array of shape (N, 3)");
  auto u = a.unchecked<2>();
  std::vector<V3> v(size_t(a.shape(0)));
  for (py::ssize_t i = 0; i < a.shape(0); ++i) v[size_t(i)] = {u(i, 0), u(i, 1), u(i, 2)};
  return v;
}
V3 to_vec3(py::object o, const char* what) {
  auto a = Arr<double>::ensure(o);
  if (!a || a.ndim() != 1 || a.shape(0) != 3) throw py::value_error(what);
  return {a.at(0), a.at(1), a.at(2)};
}
// bindings.cpp:115-149 triangle parsing: (M,3) or flat (3M,), forced to int32.
std::vector<int32_t> to_tris(py::object o, bool setter) {
  py::array arr = py::array::ensure(o);
  if (!arr) throw py::value_error("triangles must be array-like");
  py::array reshaped;
  if (arr.ndim() == 1) {
    if (arr.shape(0) % 3 != 0) throw py::value_error("triangles must contain a multiple of 3 indices");
    reshaped = arr.reshape({arr.shape(0) / 3, py::ssize_t(3)});
  } else if (arr.ndim() == 2) {
    if (arr.shape(1) != 3) throw py::value_error("triangles must have shape (M, 3)");
    reshaped = arr;
  } else {
    throw py::value_error(setter ? "triangles must be 1D or 2D array-like" : "triangles must be a 1D or 2D array");
  }
  auto t = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(reshaped);
  if (!t) throw py::value_error("triangles must be convertible to int32");
  return std::vector<int32_t>(t.data(), t.data() + t.size());
}
F32 v3_array(const std::vector<V3>& v) {
  F32 a({py::ssize_t(v.size()), py::ssize_t(3)});
  auto u = a.mutable_unchecked<2>();
  for (size_t i = 0; i < v.size(); ++i) { u(i, 0) = float(v[i].x); u(i, 1) = float(v[i].y); u(i, 2) = float(v[i].z); }
  return a;
}
py::array_t<double> v3_array64(const std::vector<V3>& v) {
  py::array_t<double> a({py::ssize_t(v.size()), py::ssize_t(3)});
  auto u = a.mutable_unchecked<2>();
  for (size_t i = 0; i < v.size(); ++i) { u(i, 0) = v[i].x; u(i, 1) = v[i].y; u(i, 2) = v[i].z; }
  return a;
}
std::vector<float> vec_f(V3 v) { return {float(v.x), float(v.y), float(v.z)}; }

void mesh_initialize(Mesh& me, std::vector<V3> verts, std::vector<int32_t> tris, const Material& mat) {
  for (int32_t t : tris)
    if (t < 0 || size_t(t) >= verts.size()) throw py::value_error("triangle index out of range");
  me.vertices = std::move(verts);
  me.tris = std::move(tris);
  me.material = mat;
  me.compute_rest_state();
}

void state_initialize(State& s, const Mesh& me) {
  if (me.nv() == 0) throw std::invalid_argument("Mesh must be initialised before creating a state");
  s.x = me.vertices; s.xp = me.vertices; s.start = me.vertices;
  s.v.assign(me.nv(), V3{});
  s.m.assign(me.nv(), 0.0);
  for (size_t f = 0; f < me.nt(); ++f) {
    double fm = me.areas[f] * me.material.thickness * me.material.density;
    for (int a = 0; a < 3; ++a) s.m[me.tris[3 * f + a]] += fm / 3.0;
  }
  s.dev_x = s.dev_v = s.start_stale = false; s.host_dirty = true; s.masses_dirty = true;
}

ando_params to_abi(const SimParams& p) {
  ando_params a;
  a.dt = p.dt; a.beta_max = p.beta_max; a.min_newton_steps = p.min_newton_steps; a.max_newton_steps = p.max_newton_steps;
  a.friction_min_newton_steps = p.friction_min_newton_steps; a.pcg_tol = p.pcg_tol; a.pcg_max_iters = p.pcg_max_iters;
  a.contact_gap_max = p.contact_gap_max; a.wall_gap = p.wall_gap; a.enable_ccd = p.enable_ccd;
  a.contact_normal_epsilon = p.contact_normal_epsilon; a.barrier_tolerance = p.barrier_tolerance;
  a.enable_friction = p.enable_friction; a.friction_mu = p.friction_mu; a.friction_epsilon = p.friction_epsilon;
  a.friction_tangent_threshold = p.friction_tangent_threshold; a.velocity_damping = p.velocity_damping;
  a.contact_restitution = p.contact_restitution; a.enable_strain_limiting = p.enable_strain_limiting;
  a.strain_limit = p.strain_limit; a.strain_tau = p.strain_tau; a.strain_epsilon = p.strain_epsilon;
  a.strain_svd_epsilon = p.strain_svd_epsilon; a.hessian_epsilon = p.hessian_epsilon; a.min_gap = p.min_gap;
  if (p.semantics == "reference") a.semantics = ANDO_SEMANTICS_REFERENCE;
  else if (p.semantics == "corrected") a.semantics = ANDO_SEMANTICS_CORRECTED;
  else throw py::value_error("semantics must be 'reference' or 'corrected'");
  if (p.preconditioner == "block_jacobi") a.precond = ANDO_PRECOND_BLOCK_JACOBI;
  else if (p.preconditioner == "learned") a.precond = ANDO_PRECOND_LEARNED;
  else throw py::value_error("preconditioner must be 'block_jacobi' or 'learned'");
  a.precond_refresh = p.precond_refresh;
  if (p.membrane_hessian == "fixed_rotation") a.membrane_hessian = ANDO_MEMBRANE_FIXED_ROTATION;
  else if (p.membrane_hessian == "projected") a.membrane_hessian = ANDO_MEMBRANE_PROJECTED;
  else throw py::value_error("membrane_hessian must be 'fixed_rotation' or 'projected'");
  return a;
}

std::vector<RigidBody*> rigid_handles(py::object lst) {
  std::vector<RigidBody*> h;
  if (lst.is_none()) return h;
  for (auto it : lst) h.push_back(&it.cast<RigidBody&>());
  return h;
}

std::vector<Contact> compute_contacts(const Mesh& me, State& s, py::object rigid_list, const std::string& semantics, double gap_max) {
  if (semantics != "reference" && semantics != "corrected") throw py::value_error("semantics must be 'reference' or 'corrected'");
  s.bind(me);
  std::vector<RigidBody*> h = rigid_handles(rigid_list);
  std::vector<ando_rigid> ab;
  for (auto* b : h) ab.push_back(b->to_abi());
  const bool corrected = semantics == "corrected";
  auto query = [&](ando_contact* out, int32_t cap, int32_t* n) {
    return corrected ? ando_compute_contacts_corrected(s.ctx, gap_max, ab.data(), int32_t(ab.size()), out, cap, n)
                     : ando_compute_contacts(s.ctx, ab.data(), int32_t(ab.size()), out, cap, n);
  };
  int32_t n = 0;
  std::vector<ando_contact> buf(256);
  int32_t rc = query(buf.data(), int32_t(buf.size()), &n);
  if (rc == ANDO_ERR_CAPACITY) {
    buf.resize(size_t(n));
    rc = query(buf.data(), n, &n);
  }
  check(rc, "compute_contacts");
  const uint64_t id = State::next_contact_list();
  s.contact_list = id;
  s.contact_count = size_t(n);
  std::vector<Contact> out(static_cast<size_t>(n));
  for (int32_t k = 0; k < n; ++k) { out[size_t(k)].c = buf[size_t(k)]; out[size_t(k)].list = id; out[size_t(k)].pos = k; }
  return out;
}

}  // namespace

PYBIND11_MODULE(ando_barrier_core, m) {
  m.doc() = "Ando 2024 Cubic Barrier with Elasticity-Inclusive Dynamic Stiffness (B200 / sm_100a implementation)";
  m.def("version", []() { return std::string("ando_barrier_core v1.0.0"); }, "Get version string");
  m.def("backend", []() { return std::string("cuda-sm_100a"); });
  m.attr("ABI_VERSION") = ando_abi_version();
  m.def("set_device", [](int d) { State::device() = d; }, "CUDA device for states created from now on (default 0)");
  m.def("get_device", []() { return State::device(); });
  m.def("set_precond_weights", [](py::array_t<float, py::array::c_style | py::array::forcecast> w) {
    if (w.ndim() != 1 || w.shape(0) != ando_precond_num_params())
      throw py::value_error("weights must be a flat array of precond_num_params() floats");
    State::precond_weights().assign(w.data(), w.data() + w.shape(0));
    State::precond_version()++;
  }, "Weights of the learned preconditioner (SimParams.preconditioner = 'learned') for every state");
  m.def("precond_num_params", []() { return ando_precond_num_params(); });

  py::class_<Material>(m, "Material")
      .def(py::init<>())
      .def(py::init([](py::kwargs kw) {
        Material mt;
        for (auto it : kw) {
          std::string k = py::cast<std::string>(it.first);
          if (k == "youngs_modulus") mt.youngs_modulus = py::cast<Real>(it.second);
          else if (k == "poisson_ratio") mt.poisson_ratio = py::cast<Real>(it.second);
          else if (k == "density") mt.density = py::cast<Real>(it.second);
          else if (k == "thickness") mt.thickness = py::cast<Real>(it.second);
          else if (k == "bending_stiffness") mt.bending_stiffness = py::cast<Real>(it.second);
          else throw py::attribute_error(("Unknown material property: " + k).c_str());
        }
        return mt;
      }))
      .def_readwrite("youngs_modulus", &Material::youngs_modulus).def_readwrite("poisson_ratio", &Material::poisson_ratio)
      .def_readwrite("density", &Material::density).def_readwrite("thickness", &Material::thickness)
      .def_readwrite("bending_stiffness", &Material::bending_stiffness);

  py::class_<SimParams>(m, "SimParams")
      .def(py::init<>())
      .def_readwrite("dt", &SimParams::dt).def_readwrite("beta_max", &SimParams::beta_max)
      .def_readwrite("min_newton_steps", &SimParams::min_newton_steps).def_readwrite("max_newton_steps", &SimParams::max_newton_steps)
      .def_readwrite("pcg_tol", &SimParams::pcg_tol).def_readwrite("pcg_max_iters", &SimParams::pcg_max_iters)
      .def_readwrite("contact_gap_max", &SimParams::contact_gap_max).def_readwrite("wall_gap", &SimParams::wall_gap)
      .def_readwrite("enable_ccd", &SimParams::enable_ccd).def_readwrite("enable_friction", &SimParams::enable_friction)
      .def_readwrite("friction_mu", &SimParams::friction_mu).def_readwrite("friction_epsilon", &SimParams::friction_epsilon)
      .def_readwrite("velocity_damping", &SimParams::velocity_damping).def_readwrite("contact_restitution", &SimParams::contact_restitution)
      .def_readwrite("enable_strain_limiting", &SimParams::enable_strain_limiting).def_readwrite("strain_limit", &SimParams::strain_limit)
      .def_readwrite("strain_tau", &SimParams::strain_tau)
      // fields the reference keeps unbound, exposed here for completeness
      .def_readwrite("friction_min_newton_steps", &SimParams::friction_min_newton_steps)
      .def_readwrite("contact_normal_epsilon", &SimParams::contact_normal_epsilon).def_readwrite("barrier_tolerance", &SimParams::barrier_tolerance)
      .def_readwrite("friction_tangent_threshold", &SimParams::friction_tangent_threshold)
      .def_readwrite("strain_epsilon", &SimParams::strain_epsilon).def_readwrite("strain_svd_epsilon", &SimParams::strain_svd_epsilon)
      .def_readwrite("hessian_epsilon", &SimParams::hessian_epsilon).def_readwrite("min_gap", &SimParams::min_gap)
      // GPU-only knobs
      .def_readwrite("semantics", &SimParams::semantics).def_readwrite("preconditioner", &SimParams::preconditioner)
      .def_readwrite("membrane_hessian", &SimParams::membrane_hessian)
      .def_readwrite("precond_refresh", &SimParams::precond_refresh);

  py::class_<Triangle>(m, "Triangle")
      .def(py::init<>())
      .def(py::init([](int32_t a, int32_t b, int32_t c) { Triangle t; t.v[0] = a; t.v[1] = b; t.v[2] = c; return t; }))
      .def_property("vertices", [](const Triangle& t) { return std::vector<int32_t>{t.v[0], t.v[1], t.v[2]}; },
                    [](Triangle& t, const std::vector<int32_t>& v) { t.v[0] = v[0]; t.v[1] = v[1]; t.v[2] = v[2]; });

  py::class_<Mesh>(m, "Mesh")
      .def(py::init<>())
      // checkpoint / resume: current vertices, triangles, the rest state as
      // computed at initialisation (kept, not recomputed) and the material
      .def(py::pickle(
          [](const Mesh& me) {
            py::array_t<int32_t> tr(py::ssize_t(me.tris.size())), ed(py::ssize_t(me.edges.size()));
            std::copy(me.tris.begin(), me.tris.end(), tr.mutable_data());
            std::copy(me.edges.begin(), me.edges.end(), ed.mutable_data());
            py::array_t<double> dm(py::ssize_t(me.dm_inv.size())), ar(py::ssize_t(me.areas.size()));
            std::copy(me.dm_inv.begin(), me.dm_inv.end(), dm.mutable_data());
            std::copy(me.areas.begin(), me.areas.end(), ar.mutable_data());
            const Material& mt = me.material;
            return py::make_tuple(v3_array64(me.vertices), tr, ed, dm, ar,
                                  py::make_tuple(mt.youngs_modulus, mt.poisson_ratio, mt.density, mt.thickness, mt.bending_stiffness));
          },
          [](py::tuple t) {
            if (t.size() != 6) throw std::runtime_error("Mesh: bad pickle");
            Mesh me;
            me.vertices = to_v3(t[0], "vertices");
            auto tr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(t[1]);
            auto ed = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(t[2]);
            auto dm = Arr<double>::ensure(t[3]);
            auto ar = Arr<double>::ensure(t[4]);
            if (!tr || !ed || !dm || !ar) throw std::runtime_error("Mesh: bad pickle arrays");
            me.tris.assign(tr.data(), tr.data() + tr.size());
            me.edges.assign(ed.data(), ed.data() + ed.size());
            me.dm_inv.assign(dm.data(), dm.data() + dm.size());
            me.areas.assign(ar.data(), ar.data() + ar.size());
            if (me.tris.size() % 3 || me.dm_inv.size() != 4 * me.nt() || me.areas.size() != me.nt())
              throw std::runtime_error("Mesh: inconsistent pickle");
            for (int32_t q : me.tris) if (q < 0 || size_t(q) >= me.nv()) throw std::runtime_error("Mesh: triangle index out of range");
            py::tuple mt = t[5].cast<py::tuple>();
            me.material.youngs_modulus = mt[0].cast<Real>(); me.material.poisson_ratio = mt[1].cast<Real>();
            me.material.density = mt[2].cast<Real>(); me.material.thickness = mt[3].cast<Real>();
            me.material.bending_stiffness = mt[4].cast<Real>();
            me.topo_version = Mesh::next_version(); me.vert_version = Mesh::next_version();
            return me;
          }))
      .def("initialize", [](Mesh& me, py::object v, py::object t, const Material& mt) {
        mesh_initialize(me, to_v3(v, "vertices"), to_tris(t, false), mt);
      }, py::arg("vertices"), py::arg("triangles"), py::arg("material"), "Initialize mesh from array-like vertex and triangle data")
      .def("num_vertices", &Mesh::nv)
      .def("num_triangles", &Mesh::nt)
      .def("get_vertices", [](const Mesh& me) { return v3_array(me.vertices); })
      .def("set_positions", [](Mesh& me, py::object p) { me.vertices = to_v3(p, "positions"); me.vert_version = Mesh::next_version(); })
      .def_property("vertices", [](const Mesh& me) { return v3_array(me.vertices); },
                    [](Mesh& me, py::object p) {
                      auto v = to_v3(p, "vertices");
                      for (size_t i = 0; i < v.size() && i < me.nv(); ++i) me.vertices[i] = v[i];
                      me.vert_version = Mesh::next_version();
                    })
      .def_property("triangles",
                    [](const Mesh& me) {
                      py::array_t<int32_t> a({py::ssize_t(me.nt()), py::ssize_t(3)});
                      std::copy(me.tris.begin(), me.tris.end(), a.mutable_data());
                      return a;
                    },
                    [](Mesh& me, py::object t) {
                      auto tr = to_tris(t, true);
                      for (int32_t q : tr) if (q < 0 || size_t(q) >= me.nv()) throw py::value_error("triangle index out of range");
                      me.tris = tr;
                      me.compute_rest_state();
                    });

  py::class_<State>(m, "State")
      .def(py::init<>())
      .def("initialize", &state_initialize)
      .def("num_vertices", &State::nv)
      .def("get_positions", [](State& s) { s.sync_x(); return v3_array(s.x); })
      .def("get_velocities", [](State& s) { s.sync_v(); return v3_array(s.v); })
      .def("set_velocities", [](State& s, py::object vel) {
        auto v = to_v3(vel, "velocities");
        s.sync_host();
        for (size_t i = 0; i < v.size() && i < s.nv(); ++i) s.v[i] = v[i];
        s.host_dirty = true;
      })
      .def("get_masses", [](const State& s) {
        F32 a(py::ssize_t(s.nv()));
        for (size_t i = 0; i < s.nv(); ++i) a.mutable_data()[i] = float(s.m[i]);
        return a;
      })
      .def("apply_gravity", [](State& s, py::object g, Real dt) {
        if (s.nv() == 0) throw std::runtime_error("State has not been initialised");
        auto ga = Arr<double>::ensure(g);
        if (!ga || ga.ndim() != 1 || ga.shape(0) != 3) throw py::value_error("Gravity must be a 3D vector");
        double gv[3] = {ga.at(0), ga.at(1), ga.at(2)};
        if (s.ctx && !s.host_dirty) {
          check(ando_apply_gravity(s.ctx, gv, dt), "apply_gravity");
          s.mark_device_newer();
        } else {
          for (size_t i = 0; i < s.nv(); ++i) {
            s.v[i] = add(s.v[i], mul(V3{gv[0], gv[1], gv[2]}, dt));
            s.x[i] = add(s.x[i], mul(s.v[i], dt));
          }
          s.host_dirty = true;
        }
      }, "Apply gravity acceleration to all vertices")
      // FP64 accessors (the device keeps positions and velocities in FP64)
      .def("get_positions64", [](State& s) { s.sync_x(); return v3_array64(s.x); })
      .def("get_velocities64", [](State& s) { s.sync_v(); return v3_array64(s.v); })
      .def("set_positions64", [](State& s, py::object p) {
        auto v = to_v3(p, "positions");
        if (v.size() != s.nv()) throw py::value_error("positions must have one row per vertex");
        s.sync_host(); s.x = v; s.start = v; s.host_dirty = true;
      })
      .def("_stream_handle", [](State& s) -> uintptr_t {
        if (!s.ctx) return 0;
        void* st = nullptr;
        check(ando_ctx_stream(s.ctx, &st), "stream");
        return reinterpret_cast<uintptr_t>(st);
      }, "cudaStream_t of the state's device context (0 before the first GPU call)")
      .def("set_velocities64", [](State& s, py::object p) {
        auto v = to_v3(p, "velocities");
        if (v.size() != s.nv()) throw py::value_error("velocities must have one row per vertex");
        s.sync_host(); s.v = v; s.host_dirty = true;
      })
      // checkpoint / resume (no reference counterpart: the reference saves no
      // solver state): FP64 positions, velocities, previous positions, the
      // CORRECTED step's start and the masses, downloaded if the device is
      // newer. A restored state uploads them on its first GPU call, so the
      // next steps continue the saved run.
      .def(py::pickle(
          [](State& s) {
            s.sync_host();
            py::array_t<double> mass(py::ssize_t(s.nv()));
            std::copy(s.m.begin(), s.m.end(), mass.mutable_data());
            return py::make_tuple(v3_array64(s.x), v3_array64(s.v), v3_array64(s.xp),
                                  v3_array64(s.start.size() == s.nv() ? s.start : s.x), mass);
          },
          [](py::tuple t) {
            if (t.size() != 5) throw std::runtime_error("State: bad pickle");
            State s;
            s.x = to_v3(t[0], "positions"); s.v = to_v3(t[1], "velocities"); s.xp = to_v3(t[2], "positions_prev");
            s.start = to_v3(t[3], "start");
            auto mass = Arr<double>::ensure(t[4]);
            if (!mass || size_t(mass.size()) != s.x.size() || s.v.size() != s.x.size() || s.xp.size() != s.x.size() || s.start.size() != s.x.size())
              throw std::runtime_error("State: inconsistent pickle");
            s.m.assign(mass.data(), mass.data() + mass.size());
            s.dev_x = s.dev_v = s.start_stale = false; s.host_dirty = true; s.masses_dirty = true;
            return s;
          }));

  py::class_<Constraints>(m, "Constraints")
      .def(py::init<>())
      // checkpoint / resume: every pin and wall with its active flag, in order
      .def(py::pickle(
          [](const Constraints& c) {
            py::list pins, walls;
            for (auto& p : c.pins) pins.append(py::make_tuple(p.vertex, p.target.x, p.target.y, p.target.z, p.active));
            for (auto& w : c.walls) walls.append(py::make_tuple(w.normal.x, w.normal.y, w.normal.z, w.offset, w.gap, w.active));
            return py::make_tuple(pins, walls);
          },
          [](py::tuple t) {
            if (t.size() != 2) throw std::runtime_error("Constraints: bad pickle");
            Constraints c;
            for (auto it : t[0].cast<py::list>()) {
              py::tuple q = it.cast<py::tuple>();
              c.pins.push_back({q[0].cast<int32_t>(), V3{q[1].cast<double>(), q[2].cast<double>(), q[3].cast<double>()}, q[4].cast<bool>()});
            }
            for (auto it : t[1].cast<py::list>()) {
              py::tuple q = it.cast<py::tuple>();
              c.walls.push_back({V3{q[0].cast<double>(), q[1].cast<double>(), q[2].cast<double>()}, q[3].cast<double>(), q[4].cast<double>(), q[5].cast<bool>()});
            }
            return c;
          }))
      .def("add_pin", [](Constraints& c, int32_t i, py::object t) { c.pins.push_back({i, to_vec3(t, "pin target must be a 3D vector"), true}); })
      .def("add_wall", [](Constraints& c, py::object n, Real off, Real gap) {
        c.walls.push_back({normalized(to_vec3(n, "wall normal must be a 3D vector")), double(off), double(gap), true});
      }, py::arg("normal"), py::arg("offset"), py::arg("gap"))
      .def("num_active_pins", [](const Constraints& c) { size_t k = 0; for (auto& p : c.pins) k += p.active; return k; })
      .def("num_active_contacts", [](const Constraints& c) { size_t k = 0; for (auto& w : c.walls) k += w.active; return k; })
      .def_property_readonly("_pins", [](const Constraints& c) {
        py::dict d;
        for (auto& p : c.pins) if (p.active) { F32 t(3); t.mutable_data()[0] = float(p.target.x); t.mutable_data()[1] = float(p.target.y); t.mutable_data()[2] = float(p.target.z); d[py::cast(p.vertex)] = t; }
        return d;
      })
      .def_property_readonly("_walls", [](const Constraints& c) {
        py::list l;
        for (auto& w : c.walls) {
          if (!w.active) continue;
          F32 n(3); n.mutable_data()[0] = float(w.normal.x); n.mutable_data()[1] = float(w.normal.y); n.mutable_data()[2] = float(w.normal.z);
          double off = std::round(double(float(w.offset)) * 1e6) / 1e6, gap = std::round(double(float(w.gap)) * 1e6) / 1e6;
          l.append(py::make_tuple(n, off, gap));
        }
        return l;
      });

  py::enum_<ContactType>(m, "ContactType")
      .value("POINT_TRIANGLE", ContactType::POINT_TRIANGLE).value("EDGE_EDGE", ContactType::EDGE_EDGE)
      .value("WALL", ContactType::WALL).value("RIGID_POINT_TRIANGLE", ContactType::RIGID_POINT_TRIANGLE).export_values();

  py::class_<Contact>(m, "Contact")
      .def(py::init<>())
      // not in the reference's binding: a contact built by hand (its fields stay
      // read-only), so a caller can judge its own contact list with
      // CollisionValidator; such a list is always read on the host
      .def(py::init([](ContactType type, int32_t idx0, int32_t idx1, int32_t idx2, int32_t idx3, double gap, py::object normal,
                       int32_t rigid_body_index) {
             Contact c;
             c.c.type = int32_t(type); c.c.idx0 = idx0; c.c.idx1 = idx1; c.c.idx2 = idx2; c.c.idx3 = idx3;
             c.c.rigid_body_index = rigid_body_index; c.c.gap = gap;
             if (!normal.is_none()) {
               V3 n = to_vec3(normal, "normal must be a 3D vector");
               c.c.normal[0] = n.x; c.c.normal[1] = n.y; c.c.normal[2] = n.z;
             }
             return c;
           }),
           py::arg("type"), py::arg("idx0") = -1, py::arg("idx1") = -1, py::arg("idx2") = -1, py::arg("idx3") = -1,
           py::arg("gap") = 0.0, py::arg("normal") = py::none(), py::arg("rigid_body_index") = -1)
      .def_property_readonly("type", [](const Contact& c) { return ContactType(c.c.type); })
      .def_property_readonly("idx0", [](const Contact& c) { return c.c.idx0; })
      .def_property_readonly("idx1", [](const Contact& c) { return c.c.idx1; })
      .def_property_readonly("idx2", [](const Contact& c) { return c.c.idx2; })
      .def_property_readonly("idx3", [](const Contact& c) { return c.c.idx3; })
      .def_property_readonly("rigid_body_index", [](const Contact& c) { return c.c.rigid_body_index; })
      .def_property_readonly("gap", [](const Contact& c) { return float(c.c.gap); })
      .def_property_readonly("normal", [](const Contact& c) { return vec_f({c.c.normal[0], c.c.normal[1], c.c.normal[2]}); })
      .def_property_readonly("witness_p", [](const Contact& c) { return vec_f({c.c.witness_p[0], c.c.witness_p[1], c.c.witness_p[2]}); })
      .def_property_readonly("witness_q", [](const Contact& c) { return vec_f({c.c.witness_q[0], c.c.witness_q[1], c.c.witness_q[2]}); });

  py::class_<RigidBody>(m, "RigidBody")
      .def(py::init<>())
      .def("initialize", [](RigidBody& b, py::object v, py::object t, Real density) {
        auto verts = to_v3(v, "vertices");
        auto tr = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(t);
        if (!tr || tr.ndim() != 2 || tr.shape(1) != 3) throw py::value_error("triangles must have shape (M, 3)");
        b.initialize(verts, std::vector<int32_t>(tr.data(), tr.data() + tr.size()), density);
      })
      .def_property("position", [](const RigidBody& b) { return vec_f({b.pos[0], b.pos[1], b.pos[2]}); },
                    [](RigidBody& b, const std::vector<Real>& p) { for (int k = 0; k < 3; ++k) b.pos[k] = p.at(k); })
      .def_property("linear_velocity", [](const RigidBody& b) { return vec_f({b.lin[0], b.lin[1], b.lin[2]}); },
                    [](RigidBody& b, const std::vector<Real>& v) { for (int k = 0; k < 3; ++k) b.lin[k] = v.at(k); })
      .def_property("angular_velocity", [](const RigidBody& b) { return vec_f({b.ang[0], b.ang[1], b.ang[2]}); },
                    [](RigidBody& b, const std::vector<Real>& v) { for (int k = 0; k < 3; ++k) b.ang[k] = v.at(k); })
      .def_property_readonly("mass", [](const RigidBody& b) { return float(b.mass); })
      .def("world_vertices", [](const RigidBody& b) { return v3_array(b.world()); })
      .def("apply_impulse", [](RigidBody& b, py::object p, py::object j) { b.apply_impulse(to_vec3(p, "point"), to_vec3(j, "impulse")); })
      .def("integrate", [](RigidBody& b, Real dt) { b.integrate(dt); });

  struct Elasticity {};
  py::class_<Elasticity>(m, "Elasticity")
      .def(py::init<>())
      .def_static("compute_energy", [](const Mesh& me, const State&) { return float(elastic_energy(me)); }, "Compute total elastic energy")
      .def_static("compute_gradient", [](const Mesh& me, const State&, py::array_t<Real> out) {
        auto g = elastic_gradient(me);
        auto o = out.mutable_unchecked<1>();
        for (py::ssize_t i = 0; i < o.shape(0); ++i) o(i) = size_t(i) < g.size() ? float(g[size_t(i)]) : 0.0f;
      }, "Compute elastic gradient (forces)")
      // The reference binds its C++ signature (mesh, state, std::vector<Triplet>&); here the
      // (row, col, value) triplets are appended to the list given (a new one if omitted) and returned.
      .def_static("compute_hessian", [](const Mesh& me, const State&, py::object triplets) {
        py::list out = triplets.is_none() ? py::list() : triplets.cast<py::list>();
        for (const auto& t : elastic_hessian_triplets(me)) out.append(py::make_tuple(std::get<0>(t), std::get<1>(t), std::get<2>(t)));
        return out;
      }, py::arg("mesh"), py::arg("state"), py::arg("triplets") = py::none(), "Compute elastic Hessian (explicit assembly)");

  // barrier.cpp:29-65
  m.def("barrier_energy", [](Real g, Real gm, Real k) -> Real {
    if (gm <= 0 || g >= gm) return 0; Real d = gm - g; if (d <= 0) return 0; return Real(0.5) * k * (Real(1) / gm) * d * d * d; });
  m.def("barrier_gradient", [](Real g, Real gm, Real k) -> Real {
    if (gm <= 0 || g >= gm) return 0; Real d = gm - g; return -Real(1.5) * k * (Real(1) / gm) * d * d; });
  m.def("barrier_hessian", [](Real g, Real gm, Real k) -> Real {
    if (gm <= 0 || g >= gm) return 0; Real d = gm - g; return Real(3) * k * (Real(1) / gm) * d; });

  m.def("create_mesh_from_blender", [](py::object v, py::object t, const Material& mt) {
    Mesh me; mesh_initialize(me, to_v3(v, "vertices"), to_tris(t, false), mt); return me;
  }, "Create mesh from numpy arrays (vertices Nx3, triangles Mx3)");

  struct Integrator {};
  py::class_<Integrator>(m, "Integrator")
      .def(py::init<>())
      .def_static("step", [](Mesh& me, State& s, Constraints& c, const SimParams& p, py::object rigid_list) {
        ando_params ap = to_abi(p);
        s.bind(me);
        if (ap.precond == ANDO_PRECOND_LEARNED) s.bind_weights();
        std::vector<ando_pin> pins;
        for (auto& q : c.pins) pins.push_back({q.vertex, q.active ? 1 : 0, {q.target.x, q.target.y, q.target.z}});
        std::vector<ando_wall> walls;
        for (auto& w : c.walls) walls.push_back({{w.normal.x, w.normal.y, w.normal.z}, w.offset, w.gap, w.active ? 1 : 0, 0});
        std::vector<RigidBody*> h = rigid_handles(rigid_list);
        std::vector<ando_rigid> ab;
        for (auto* b : h) ab.push_back(b->to_abi());
        int32_t rc;
        s.contact_list = 0;               // the step replaces the device contact list
        {
          py::gil_scoped_release nogil;
          rc = ando_step(s.ctx, &ap, pins.data(), int32_t(pins.size()), walls.data(), int32_t(walls.size()),
                         ab.data(), int32_t(ab.size()), &s.last);
        }
        check(rc, "Integrator.step");
        s.mark_device_newer();
        for (size_t i = 0; i < h.size(); ++i) h[i]->from_abi(ab[i]);
      }, py::arg("mesh"), py::arg("state"), py::arg("constraints"), py::arg("params"), py::arg("rigid_bodies") = py::none(),
         "Take one simulation step using Newton integrator with beta accumulation")
      // semantics="corrected" (not in the reference's binding) returns the self and rigid contacts
      // within gap_max that the CORRECTED step uses
      .def_static("compute_contacts", [](const Mesh& me, State& s, py::object rigid_list, const std::string& semantics, double gap_max) {
        return compute_contacts(me, s, rigid_list, semantics, gap_max); },
                  py::arg("mesh"), py::arg("state"), py::arg("rigid_bodies") = py::none(), py::arg("semantics") = "reference",
                  py::arg("gap_max") = 1e-3, "Detect all collision contacts for the current mesh/state")
      .def_static("last_step_stats", [](const State& s) {
        py::dict d;
        d["newton_iters"] = s.last.newton_iters; d["pcg_iters"] = s.last.pcg_iters; d["pcg_max_per_newton"] = s.last.pcg_max_per_newton;
        d["pcg_not_converged"] = s.last.pcg_not_converged; d["line_search_fail"] = s.last.line_search_fail; d["contacts"] = s.last.contacts;
        d["strain_active"] = s.last.strain_active; d["beta"] = s.last.beta; d["last_alpha"] = s.last.last_alpha;
        d["device_ms"] = s.last.device_ms; d["precond_fallbacks"] = s.last.precond_fallbacks; d["graph_launched"] = s.last.graph_launched != 0; d["substeps"] = s.last.substeps;
        return d;
      }, py::arg("state"), "Counters of the state's last step");

  py::class_<EnergyDiagnostics>(m, "EnergyDiagnostics")
      .def(py::init<>())
      .def_readonly("kinetic_energy", &EnergyDiagnostics::kinetic_energy).def_readonly("elastic_energy", &EnergyDiagnostics::elastic_energy)
      .def_readonly("barrier_energy", &EnergyDiagnostics::barrier_energy).def_readonly("total_energy", &EnergyDiagnostics::total_energy)
      .def_readonly("energy_drift_percent", &EnergyDiagnostics::energy_drift_percent)
      .def_readonly("energy_drift_absolute", &EnergyDiagnostics::energy_drift_absolute)
      .def_property_readonly("linear_momentum", [](const EnergyDiagnostics& d) { return vec_f(d.linear_momentum); })
      .def_property_readonly("angular_momentum", [](const EnergyDiagnostics& d) { return vec_f(d.angular_momentum); })
      .def_readonly("max_velocity", &EnergyDiagnostics::max_velocity)
      .def_readonly("num_contacts", &EnergyDiagnostics::num_contacts).def_readonly("num_pins", &EnergyDiagnostics::num_pins)
      .def("update_drift", &EnergyDiagnostics::update_drift);

  // energy_tracker.cpp:6-76: reduced on the device when it holds the state
  // (ando_state_moments, no download), else over the host copy
  struct EnergyTracker {};
  auto moments = [](State& s) {
    ando_moments mo{};
    if (s.device_current()) { check(ando_state_moments(s.ctx, &mo), "state moments"); return mo; }
    s.sync_host();
    double v2max = 0;
    for (size_t i = 0; i < s.nv(); ++i) {
      V3 p = mul(s.v[i], s.m[i]), L = cross(s.x[i], p);
      mo.kinetic_energy += 0.5 * s.m[i] * dot(s.v[i], s.v[i]);
      mo.linear_momentum[0] += p.x; mo.linear_momentum[1] += p.y; mo.linear_momentum[2] += p.z;
      mo.angular_momentum[0] += L.x; mo.angular_momentum[1] += L.y; mo.angular_momentum[2] += L.z;
      v2max = std::max(v2max, dot(s.v[i], s.v[i]));
    }
    mo.max_speed = std::sqrt(v2max);
    return mo;
  };
  auto ke = [moments](State& s) { return moments(s).kinetic_energy; };
  auto lm = [moments](State& s) { ando_moments mo = moments(s); return V3{mo.linear_momentum[0], mo.linear_momentum[1], mo.linear_momentum[2]}; };
  auto am = [moments](State& s) { ando_moments mo = moments(s); return V3{mo.angular_momentum[0], mo.angular_momentum[1], mo.angular_momentum[2]}; };
  auto mvel = [moments](State& s) { return moments(s).max_speed; };
  py::class_<EnergyTracker>(m, "EnergyTracker")
      .def(py::init<>())
      .def_static("compute", [moments](const Mesh& me, State& s, const Constraints& c, const SimParams&) {
        EnergyDiagnostics d;
        ando_moments mo = moments(s);
        d.kinetic_energy = float(mo.kinetic_energy); d.elastic_energy = float(elastic_energy(me)); d.barrier_energy = 0;
        d.total_energy = d.kinetic_energy + d.elastic_energy + d.barrier_energy;
        d.linear_momentum = V3{mo.linear_momentum[0], mo.linear_momentum[1], mo.linear_momentum[2]};
        d.angular_momentum = V3{mo.angular_momentum[0], mo.angular_momentum[1], mo.angular_momentum[2]};
        d.max_velocity = float(mo.max_speed);
        int nw = 0; for (auto& w : c.walls) nw += w.active;
        int np = 0; for (auto& p : c.pins) np += p.active;
        d.num_contacts = 0 * nw; d.num_pins = np;
        return d;
      }, py::arg("mesh"), py::arg("state"), py::arg("constraints"), py::arg("params"), "Compute comprehensive energy diagnostics")
      .def_static("compute_kinetic_energy", [ke](State& s) { return float(ke(s)); }, "Compute kinetic energy")
      .def_static("compute_linear_momentum", [lm](State& s) { return vec_f(lm(s)); }, "Compute linear momentum")
      .def_static("compute_angular_momentum", [am](State& s) { return vec_f(am(s)); }, "Compute angular momentum")
      .def_static("compute_max_velocity", [mvel](State& s) { return float(mvel(s)); }, "Compute maximum velocity");

  py::class_<CollisionMetrics>(m, "CollisionMetrics")
      .def(py::init<>())
      .def_readonly("num_point_triangle", &CollisionMetrics::num_point_triangle).def_readonly("num_edge_edge", &CollisionMetrics::num_edge_edge)
      .def_readonly("num_wall", &CollisionMetrics::num_wall).def_readonly("num_total_contacts", &CollisionMetrics::num_total_contacts)
      .def_readonly("min_gap", &CollisionMetrics::min_gap).def_readonly("max_gap", &CollisionMetrics::max_gap)
      .def_readonly("avg_gap", &CollisionMetrics::avg_gap).def_readonly("num_penetrations", &CollisionMetrics::num_penetrations)
      .def_readonly("max_penetration", &CollisionMetrics::max_penetration).def_readonly("avg_penetration", &CollisionMetrics::avg_penetration)
      .def_readonly("ccd_enabled", &CollisionMetrics::ccd_enabled).def_readonly("num_ccd_contacts", &CollisionMetrics::num_ccd_contacts)
      .def_readonly("num_broad_phase_contacts", &CollisionMetrics::num_broad_phase_contacts)
      .def_readonly("ccd_effectiveness", &CollisionMetrics::ccd_effectiveness)
      .def_readonly("max_relative_velocity", &CollisionMetrics::max_relative_velocity)
      .def_readonly("avg_relative_velocity", &CollisionMetrics::avg_relative_velocity)
      .def_readonly("has_tunneling", &CollisionMetrics::has_tunneling).def_readonly("has_major_penetration", &CollisionMetrics::has_major_penetration)
      .def_readonly("is_stable", &CollisionMetrics::is_stable)
      .def("quality_level", &CollisionMetrics::quality_level).def("quality_description", &CollisionMetrics::quality_description);

  // collision_validator.cpp:7-221. A list that compute_contacts returned for
  // this state, unchanged and still the one the device holds, is reduced on
  // the device (ando_collision_metrics: no contact or state download); any
  // other list is read on the host, with the state's velocities downloaded.
  struct CollisionValidator {};
  py::class_<CollisionValidator>(m, "CollisionValidator")
      .def(py::init<>())
      .def_static("compute_metrics", [](const Mesh&, State& s, const std::vector<Contact>& cs, Real gap_max, bool ccd) {
        CollisionMetrics M;
        M.ccd_enabled = ccd;
        M.num_total_contacts = int(cs.size());
        bool on_device = !cs.empty() && s.device_current() && s.contact_list != 0 && cs.size() == s.contact_count;
        for (size_t k = 0; on_device && k < cs.size(); ++k) on_device = cs[k].list == s.contact_list && cs[k].pos == int32_t(k);
        if (on_device) {
          ando_metrics d{};
          check(ando_collision_metrics(s.ctx, double(gap_max), ccd ? 1 : 0, &d), "collision metrics");
          const int n = d.num_total_contacts;
          M.num_point_triangle = d.num_point_triangle; M.num_edge_edge = d.num_edge_edge; M.num_wall = d.num_wall;
          M.min_gap = Real(d.min_gap); M.max_gap = Real(d.max_gap); M.avg_gap = Real(d.sum_gap / n);
          M.num_penetrations = d.num_penetrations;
          M.max_penetration = Real(d.max_penetration);
          if (d.num_penetrations > 0) { M.avg_penetration = Real(d.sum_penetration / d.num_penetrations); M.is_stable = false; }
          M.has_major_penetration = d.num_major_penetrations > 0; M.has_tunneling = d.num_tunneling > 0;
          M.num_ccd_contacts = d.num_ccd_contacts; M.num_broad_phase_contacts = n - d.num_ccd_contacts;
          M.ccd_effectiveness = (ccd && n > 0) ? Real(d.num_ccd_contacts) / Real(n) * 100.0f : 0.0f;
          if (d.num_relative_velocities > 0) {
            M.max_relative_velocity = Real(d.max_relative_velocity);
            M.avg_relative_velocity = Real(d.sum_relative_velocity / d.num_relative_velocities);
          }
          return M;
        }
        if (!cs.empty()) {
          M.min_gap = M.max_gap = float(cs[0].c.gap);
          Real sum_gap = 0, sum_pen = 0;
          M.num_point_triangle = M.num_edge_edge = M.num_wall = 0;
          for (auto& C : cs) {
            if (C.c.type == 0) M.num_point_triangle++; else if (C.c.type == 1) M.num_edge_edge++; else if (C.c.type == 2) M.num_wall++;
            Real g = float(C.c.gap);
            M.min_gap = std::min(M.min_gap, g); M.max_gap = std::max(M.max_gap, g); sum_gap += g;
            if (g < 0) {
              M.num_penetrations++; Real pen = -g; M.max_penetration = std::max(M.max_penetration, pen); sum_pen += pen;
              if (pen > 0.001) M.has_major_penetration = true;
              if (pen > 0.1 * gap_max) M.has_tunneling = true;
            }
          }
          M.avg_gap = sum_gap / M.num_total_contacts;
          if (M.num_penetrations > 0) { M.avg_penetration = sum_pen / M.num_penetrations; M.is_stable = false; }
          for (auto& C : cs) { if (ccd && float(C.c.gap) < gap_max * 0.5) M.num_ccd_contacts++; else M.num_broad_phase_contacts++; }
          M.ccd_effectiveness = (ccd && M.num_total_contacts > 0) ? Real(M.num_ccd_contacts) / Real(M.num_total_contacts) * 100.0f : 0.0f;
          s.sync_host();
          std::vector<Real> rv;
          for (auto& C : cs) {
            V3 n{C.c.normal[0], C.c.normal[1], C.c.normal[2]};
            if (C.c.type == 0) {
              V3 vt = mul(add(add(s.v[C.c.idx1], s.v[C.c.idx2]), s.v[C.c.idx3]), 1.0 / 3.0);
              rv.push_back(float(std::fabs(dot(sub(s.v[C.c.idx0], vt), n))));
            } else if (C.c.type == 1) {
              V3 a = mul(add(s.v[C.c.idx0], s.v[C.c.idx1]), 0.5), b = mul(add(s.v[C.c.idx2], s.v[C.c.idx3]), 0.5);
              rv.push_back(float(std::fabs(dot(sub(a, b), n))));
            } else if (C.c.type == 2) {
              rv.push_back(float(std::fabs(dot(s.v[C.c.idx0], n))));
            }
          }
          if (!rv.empty()) {
            M.max_relative_velocity = *std::max_element(rv.begin(), rv.end());
            Real sv = 0; for (Real x : rv) sv += x; M.avg_relative_velocity = sv / rv.size();
          }
        }
        return M;
      }, py::arg("mesh"), py::arg("state"), py::arg("contacts"), py::arg("gap_max"), py::arg("ccd_enabled"), "Compute comprehensive collision metrics")
      // not in the reference's binding: the discrete check no contact list can give
      .def_static("edge_triangle_crossings", [](const Mesh& me, State& s) {
        s.bind(me);
        int64_t n = 0;
        check(ando_edge_triangle_crossings(s.ctx, &n), "edge_triangle_crossings");
        return n;
      }, py::arg("mesh"), py::arg("state"),
         "Mesh edges whose segment passes through a triangle they share no vertex with (exact test on the GPU)")
      .def_static("has_penetrations", [](const std::vector<Contact>& cs) { for (auto& C : cs) if (C.c.gap < 0) return true; return false; })
      .def_static("max_penetration_depth", [](const std::vector<Contact>& cs) { Real m = 0; for (auto& C : cs) if (C.c.gap < 0) m = std::max(m, float(-C.c.gap)); return m; });

  // adaptive_timestep.cpp:8-151 (flat 3N velocities)
  struct AdaptiveTimestep {};
  auto min_edge = [](const Mesh& me) -> Real {
    if (me.edges.empty()) return 0;
    double best = std::numeric_limits<double>::max(); bool found = false;
    for (size_t e = 0; e < me.edges.size() / 2; ++e) {
      int a = me.edges[2 * e], b = me.edges[2 * e + 1];
      if (a < 0 || b < 0 || size_t(a) >= me.nv() || size_t(b) >= me.nv()) continue;
      V3 d = sub(me.vertices[b], me.vertices[a]);
      double l2 = float(dot(d, d));
      if (!std::isfinite(l2)) continue;
      best = std::min(best, l2); found = true;
    }
    if (!found) return 0;
    Real r = float(std::sqrt(std::max(best, 0.0)));
    return std::isfinite(r) ? r : 0;
  };
  // velocities: the reference's flat 3N array, or a State (its device
  // velocities are reduced on the device, ando_state_moments)
  auto max_vel = [](py::object v) -> Real {
    if (py::isinstance<State>(v)) {
      State& st = v.cast<State&>();
      if (st.device_current()) { ando_moments mo{}; check(ando_state_moments(st.ctx, &mo), "state moments"); return float(mo.max_speed); }
      st.sync_v();
      double mx = 0;
      for (auto& q : st.v) mx = std::max(mx, double(float(q.x * q.x + q.y * q.y + q.z * q.z)));
      return float(std::sqrt(mx));
    }
    auto a = Arr<float>::ensure(v);
    double mx = 0; py::ssize_t n = a.size() / 3;
    for (py::ssize_t i = 0; i < n; ++i) { double x = a.data()[3 * i], y = a.data()[3 * i + 1], z = a.data()[3 * i + 2]; mx = std::max(mx, double(float(x * x + y * y + z * z))); }
    return float(std::sqrt(mx));
  };
  auto cfl = [](Real vmax, Real edge, Real safety) -> Real { if (vmax < 1e-6f) return 1.0f; return safety * edge / vmax; };
  py::class_<AdaptiveTimestep>(m, "AdaptiveTimestep")
      .def(py::init<>())
      .def_static("compute_next_dt", [min_edge, max_vel, cfl](py::object vel, const Mesh& me, double cur, double dmin, double dmax, double safety) {
        Real v = max_vel(vel);
        Real dt;
        if (v < 1e-6f) dt = Real(dmax);
        else {
          Real e = min_edge(me); if (e < 1e-5f) e = 1e-5f;
          Real target = std::clamp(cfl(v, e, Real(safety)), Real(dmin), Real(dmax));
          Real next = target < Real(cur) ? target : std::min(target, Real(cur) * 1.5f);
          dt = std::clamp(next, Real(dmin), Real(dmax));
        }
        return std::clamp(double(dt), dmin, dmax);
      }, py::arg("velocities"), py::arg("mesh"), py::arg("current_dt"), py::arg("dt_min"), py::arg("dt_max"), py::arg("safety") = 0.5,
         "Compute next timestep using CFL condition")
      .def_static("compute_cfl_timestep", cfl, py::arg("max_velocity"), py::arg("min_edge_length"), py::arg("safety") = 0.5)
      .def_static("compute_min_edge_length", min_edge, py::arg("mesh"))
      .def_static("compute_max_velocity", max_vel, py::arg("velocities"));
}
