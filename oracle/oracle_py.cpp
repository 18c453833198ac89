// oracle_py.cpp -- pybind11 binding of the CPU oracle (test infrastructure only).
//
// Builds the module `ando_oracle` with two submodules, `f64` and `f32`, each a
// restatement of the reference's ando_barrier_core surface
// (src/py/bindings.cpp:27-633) in that precision, plus entry points that
// expose intermediate results (gradient, assembled Hessian, PCG, line search,
// broad phase) so the CUDA path can be checked stage by stage.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <chrono>
#include <string>

#include "ando_oracle.hpp"

namespace py = pybind11;
using namespace ando_oracle;

namespace {

template <class R> using Arr = py::array_t<R, py::array::c_style | py::array::forcecast>;

template <class R> std::vector<V3<R>> to_v3(const Arr<R>& a) {
  if (a.ndim() != 2 || a.shape(1) != 3) throw py::value_error("expected an array of shape (N, 3)");
  std::vector<V3<R>> v(size_t(a.shape(0)));
  auto u = a.template unchecked<2>();
  for (py::ssize_t i = 0; i < a.shape(0); ++i) v[size_t(i)] = V3<R>(u(i, 0), u(i, 1), u(i, 2));
  return v;
}
template <class R> py::array_t<R> from_v3(const std::vector<V3<R>>& v) {
  py::array_t<R> a({py::ssize_t(v.size()), py::ssize_t(3)});
  auto u = a.template mutable_unchecked<2>();
  for (size_t i = 0; i < v.size(); ++i) { u(i, 0) = v[i].x; u(i, 1) = v[i].y; u(i, 2) = v[i].z; }
  return a;
}
template <class R> V3<R> vec3(py::object o) {
  auto a = Arr<R>::ensure(o);
  if (!a || a.ndim() != 1 || a.shape(0) != 3) throw py::value_error("expected a 3-vector");
  return V3<R>(a.at(0), a.at(1), a.at(2));
}
std::vector<Triangle> to_tris(py::object o) {
  auto a = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(o);
  if (!a) throw py::value_error("triangles must be array-like");
  if (a.ndim() == 1) { if (a.shape(0) % 3) throw py::value_error("triangles must contain a multiple of 3 indices"); a = a.reshape({a.shape(0) / 3, py::ssize_t(3)}); }
  if (a.ndim() != 2 || a.shape(1) != 3) throw py::value_error("triangles must have shape (M, 3)");
  std::vector<Triangle> t(size_t(a.shape(0)));
  auto u = a.unchecked<2>();
  for (py::ssize_t i = 0; i < a.shape(0); ++i) t[size_t(i)] = Triangle(u(i, 0), u(i, 1), u(i, 2));
  return t;
}
Lookup to_lookup(const std::string& s) { return s == "literal" ? Lookup::LITERAL : Lookup::INDEXED; }
BroadPhase to_broad(const std::string& s) { return s == "intended" ? BroadPhase::INTENDED : BroadPhase::LITERAL; }

template <class R> py::dict csr_dict(const Csr<R>& A) {
  py::dict d;
  d["n"] = A.n;
  d["rowptr"] = py::array_t<int32_t>(py::ssize_t(A.rowptr.size()), A.rowptr.data());
  d["cols"] = py::array_t<int32_t>(py::ssize_t(A.cols.size()), A.cols.data());
  d["vals"] = py::array_t<R>(py::ssize_t(A.vals.size()), A.vals.data());
  return d;
}
template <class R> std::vector<R> vec_of(py::object o) {
  auto a = Arr<R>::ensure(o);
  return std::vector<R>(a.data(), a.data() + a.size());
}
template <class R> Csr<R> csr_from(int n, py::object rows, py::object cols, py::object vals) {
  auto r = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(rows);
  auto c = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(cols);
  auto v = Arr<R>::ensure(vals);
  std::vector<Triplet<R>> t(size_t(v.size()));
  for (py::ssize_t k = 0; k < v.size(); ++k) t[size_t(k)] = {r.at(k), c.at(k), v.at(k)};
  return Csr<R>::from_triplets(n, t);
}

template <class R> void bind(py::module_& m) {
  using MeshT = Mesh<R>; using StateT = State<R>; using ConT = Constraints<R>; using ParT = SimParams<R>;
  using CP = ContactPair<R>; using RB = RigidBody<R>;

  py::class_<Material<R>>(m, "Material")
      .def(py::init<>())
      .def(py::init([](py::kwargs kw) {
        Material<R> mt;
        for (auto it : kw) {
          std::string k = py::cast<std::string>(it.first);
          R v = py::cast<R>(it.second);
          if (k == "youngs_modulus") mt.youngs_modulus = v; else if (k == "poisson_ratio") mt.poisson_ratio = v;
          else if (k == "density") mt.density = v; else if (k == "thickness") mt.thickness = v;
          else if (k == "bending_stiffness") mt.bending_stiffness = v;
          else throw py::attribute_error(("Unknown material property: " + k).c_str());
        }
        return mt;
      }))
      .def_readwrite("youngs_modulus", &Material<R>::youngs_modulus).def_readwrite("poisson_ratio", &Material<R>::poisson_ratio)
      .def_readwrite("density", &Material<R>::density).def_readwrite("thickness", &Material<R>::thickness)
      .def_readwrite("bending_stiffness", &Material<R>::bending_stiffness);

  py::class_<ParT>(m, "SimParams")
      .def(py::init<>())
      .def_readwrite("dt", &ParT::dt).def_readwrite("beta_max", &ParT::beta_max)
      .def_readwrite("min_newton_steps", &ParT::min_newton_steps).def_readwrite("max_newton_steps", &ParT::max_newton_steps)
      .def_readwrite("friction_min_newton_steps", &ParT::friction_min_newton_steps)
      .def_readwrite("pcg_tol", &ParT::pcg_tol).def_readwrite("pcg_max_iters", &ParT::pcg_max_iters)
      .def_readwrite("contact_gap_max", &ParT::contact_gap_max).def_readwrite("wall_gap", &ParT::wall_gap)
      .def_readwrite("enable_ccd", &ParT::enable_ccd).def_readwrite("contact_normal_epsilon", &ParT::contact_normal_epsilon)
      .def_readwrite("barrier_tolerance", &ParT::barrier_tolerance)
      .def_readwrite("enable_friction", &ParT::enable_friction).def_readwrite("friction_mu", &ParT::friction_mu)
      .def_readwrite("friction_epsilon", &ParT::friction_epsilon).def_readwrite("friction_tangent_threshold", &ParT::friction_tangent_threshold)
      .def_readwrite("velocity_damping", &ParT::velocity_damping).def_readwrite("contact_restitution", &ParT::contact_restitution)
      .def_readwrite("enable_strain_limiting", &ParT::enable_strain_limiting).def_readwrite("strain_limit", &ParT::strain_limit)
      .def_readwrite("strain_tau", &ParT::strain_tau).def_readwrite("strain_epsilon", &ParT::strain_epsilon)
      .def_readwrite("strain_svd_epsilon", &ParT::strain_svd_epsilon).def_readwrite("hessian_epsilon", &ParT::hessian_epsilon).def_readwrite("membrane_hessian", &ParT::membrane_hessian)
      .def_readwrite("min_gap", &ParT::min_gap);

  py::class_<MeshT>(m, "Mesh")
      .def(py::init<>())
      .def("initialize", [](MeshT& me, py::object v, py::object t, const Material<R>& mt) {
        auto va = Arr<R>::ensure(v);
        if (!va || va.ndim() != 2 || va.shape(1) != 3) throw py::value_error("vertices must be an array of shape (N, 3)");
        me.initialize(to_v3<R>(va), to_tris(t), mt);
      }, py::arg("vertices"), py::arg("triangles"), py::arg("material"))
      .def("num_vertices", [](const MeshT& me) { return me.vertices.size(); })
      .def("num_triangles", [](const MeshT& me) { return me.triangles.size(); })
      .def("num_edges", [](const MeshT& me) { return me.edges.size(); })
      .def("get_vertices", [](const MeshT& me) { return from_v3(me.vertices); })
      .def("set_positions", [](MeshT& me, Arr<R> p) { me.vertices = to_v3<R>(p); })
      .def_property_readonly("edges", [](const MeshT& me) {
        py::array_t<int32_t> a({py::ssize_t(me.edges.size()), py::ssize_t(2)}); auto u = a.template mutable_unchecked<2>();
        for (size_t i = 0; i < me.edges.size(); ++i) { u(i, 0) = me.edges[i].v[0]; u(i, 1) = me.edges[i].v[1]; }
        return a; })
      .def_property_readonly("rest_areas", [](const MeshT& me) { return py::array_t<R>(py::ssize_t(me.rest_areas.size()), me.rest_areas.data()); })
      .def_property_readonly("Dm_inv", [](const MeshT& me) {
        py::array_t<R> a({py::ssize_t(me.Dm_inv.size()), py::ssize_t(2), py::ssize_t(2)}); auto u = a.template mutable_unchecked<3>();
        for (size_t i = 0; i < me.Dm_inv.size(); ++i) { u(i, 0, 0) = me.Dm_inv[i].a; u(i, 0, 1) = me.Dm_inv[i].b; u(i, 1, 0) = me.Dm_inv[i].c; u(i, 1, 1) = me.Dm_inv[i].d; }
        return a; });

  py::class_<StateT>(m, "State")
      .def(py::init<>())
      .def("initialize", &StateT::initialize)
      .def("num_vertices", [](const StateT& s) { return s.positions.size(); })
      .def("get_positions", [](const StateT& s) { return from_v3(s.positions); })
      .def("set_positions", [](StateT& s, Arr<R> p) { s.positions = to_v3<R>(p); s.positions_safe = s.positions; })
      .def("get_velocities", [](const StateT& s) { return from_v3(s.velocities); })
      .def("set_velocities", [](StateT& s, Arr<R> v) { auto vv = to_v3<R>(v); for (size_t i = 0; i < vv.size() && i < s.velocities.size(); ++i) s.velocities[i] = vv[i]; })
      .def("get_positions_prev", [](const StateT& s) { return from_v3(s.positions_prev); })
      .def("get_masses", [](const StateT& s) { return py::array_t<R>(py::ssize_t(s.masses.size()), s.masses.data()); })
      .def("set_masses", [](StateT& s, Arr<R> mm) { s.masses.assign(mm.data(), mm.data() + mm.size()); })
      .def("apply_gravity", [](StateT& s, py::object g, R dt) { s.apply_gravity(vec3<R>(g), dt); });

  py::class_<ConT>(m, "Constraints")
      .def(py::init<>())
      .def("add_pin", [](ConT& c, Index i, py::object t) { c.add_pin(i, vec3<R>(t)); })
      .def("add_wall", [](ConT& c, py::object n, R off, R gap) { c.add_wall(vec3<R>(n), off, gap); }, py::arg("normal"), py::arg("offset"), py::arg("gap"))
      .def("num_active_pins", &ConT::num_active_pins)
      .def("num_active_walls", &ConT::num_active_walls)
      .def("num_strain_limits", [](const ConT& c) { return c.strain_limits.size(); })
      .def("clear_pins", [](ConT& c) { c.pins.clear(); });

  py::module_ parent = py::module_::import("ando_oracle");
  m.attr("ContactType") = parent.attr("ContactType");
  for (const char* nm : {"POINT_TRIANGLE", "EDGE_EDGE", "WALL", "RIGID_POINT_TRIANGLE"}) m.attr(nm) = parent.attr(nm);

  py::class_<CP>(m, "Contact")
      .def(py::init<>())
      .def_readwrite("type", &CP::type).def_readwrite("idx0", &CP::idx0).def_readwrite("idx1", &CP::idx1)
      .def_readwrite("idx2", &CP::idx2).def_readwrite("idx3", &CP::idx3).def_readwrite("gap", &CP::gap)
      .def_readwrite("vertex_count", &CP::vertex_count).def_readwrite("rigid_body_index", &CP::rigid_body_index)
      .def_property("normal", [](const CP& c) { return std::vector<R>{c.normal.x, c.normal.y, c.normal.z}; }, [](CP& c, py::object o) { c.normal = vec3<R>(o); })
      .def_property("witness_p", [](const CP& c) { return std::vector<R>{c.witness_p.x, c.witness_p.y, c.witness_p.z}; }, [](CP& c, py::object o) { c.witness_p = vec3<R>(o); })
      .def_property("witness_q", [](const CP& c) { return std::vector<R>{c.witness_q.x, c.witness_q.y, c.witness_q.z}; }, [](CP& c, py::object o) { c.witness_q = vec3<R>(o); })
      .def_property("weights", [](const CP& c) { return std::vector<R>(c.weights.begin(), c.weights.end()); },
                    [](CP& c, std::vector<R> w) { for (size_t i = 0; i < 4 && i < w.size(); ++i) c.weights[i] = w[i]; });

  py::class_<RB>(m, "RigidBody")
      .def(py::init<>())
      .def("initialize", [](RB& b, Arr<R> v, py::object t, R density) { b.initialize(to_v3<R>(v), to_tris(t), density); })
      .def_property("position", [](const RB& b) { return std::vector<R>{b.position.x, b.position.y, b.position.z}; }, [](RB& b, std::vector<R> p) { b.position = V3<R>(p[0], p[1], p[2]); })
      .def_property("linear_velocity", [](const RB& b) { return std::vector<R>{b.lin_vel.x, b.lin_vel.y, b.lin_vel.z}; }, [](RB& b, std::vector<R> p) { b.lin_vel = V3<R>(p[0], p[1], p[2]); })
      .def_property("angular_velocity", [](const RB& b) { return std::vector<R>{b.ang_vel.x, b.ang_vel.y, b.ang_vel.z}; }, [](RB& b, std::vector<R> p) { b.ang_vel = V3<R>(p[0], p[1], p[2]); })
      .def_property_readonly("mass", [](const RB& b) { return b.mass; })
      .def("world_vertices", [](const RB& b) { return from_v3(b.world_vertices()); })
      .def("apply_impulse", [](RB& b, py::object p, py::object j) { b.apply_impulse(vec3<R>(p), vec3<R>(j)); })
      .def("integrate", &RB::integrate);

  auto opts = [](const std::string& lookup, const std::string& broad) { Options<R> o; o.lookup = to_lookup(lookup); o.broad = to_broad(broad); return o; };
  auto stats_dict = [](const StepStats<R>& S, double seconds) {
    py::dict d;
    d["newton_iters"] = S.newton_iters; d["pcg_iters"] = S.pcg_iters; d["line_search_fail"] = S.line_search_fail;
    d["contacts"] = S.contacts; d["pcg_not_converged"] = S.pcg_not_converged; d["beta"] = S.beta; d["substeps"] = S.substeps;
    d["alphas"] = S.alphas; d["pcg_per_newton"] = S.pcg_per_newton; d["seconds"] = seconds;
    return d;
  };

  struct IntegratorTag {};
  py::class_<IntegratorTag>(m, "Integrator")
      .def_static("step", [opts, stats_dict](MeshT& me, StateT& s, ConT& c, const ParT& p, py::object rigid, const std::string& lookup,
                                            const std::string& broad, const std::string& semantics) {
        Options<R> o = opts(lookup, broad);
        StepStats<R> S;
        bool corrected = semantics == "corrected";
        auto t0 = std::chrono::steady_clock::now();
        std::vector<RB*> h; std::vector<RB> store;
        if (!rigid.is_none()) for (auto it : rigid) { RB& b = it.cast<RB&>(); h.push_back(&b); store.push_back(b); }
        std::vector<RB>* rp = rigid.is_none() ? nullptr : &store;
        if (corrected) CorrectedIntegrator<R>::step(me, s, c, p, rp, &S);
        else Integrator<R>::step(me, s, c, p, rp, o, &S);
        for (size_t i = 0; i < h.size(); ++i) *h[i] = store[i];
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return stats_dict(S, secs);
      }, py::arg("mesh"), py::arg("state"), py::arg("constraints"), py::arg("params"), py::arg("rigid_bodies") = py::none(),
         py::arg("lookup") = "indexed", py::arg("broad") = "literal", py::arg("semantics") = "reference")
      // CORRECTED stages at the current state: contacts, gradient, Hessian, time of impact
      .def_static("corrected_system", [](const MeshT& me, StateT& s, Arr<R> x_target, py::object fixed_mask, ConT& c, const ParT& p) {
        auto fm = py::array_t<int8_t, py::array::c_style | py::array::forcecast>::ensure(fixed_mask);
        std::vector<char> fixed(fm.data(), fm.data() + fm.size());
        auto contacts = detect_corrected(me, s.positions, (const std::vector<RB>*)nullptr, p.contact_gap_max);
        Csr<R> H_el = CorrectedIntegrator<R>::base_elastic(me);
        std::vector<R> g;
        CorrectedIntegrator<R>::gradient(me, s, to_v3<R>(x_target), fixed, contacts, c, p, H_el, g);
        Csr<R> H = CorrectedIntegrator<R>::assemble(me, s, fixed, contacts, c, p, H_el);
        py::dict d; d["gradient"] = py::array_t<R>(py::ssize_t(g.size()), g.data()); d["hessian"] = csr_dict(H);
        d["contacts"] = contacts;
        return d;
      })
      // frozen-stiffness CORRECTED incremental potential at positions X (contacts, strain limits and walls from the state)
      .def_static("corrected_energy", [](const MeshT& me, StateT& s, Arr<R> X, Arr<R> x_target, ConT& c, const ParT& p) {
        auto contacts = detect_corrected(me, s.positions, (const std::vector<RB>*)nullptr, p.contact_gap_max);
        Csr<R> H_el = CorrectedIntegrator<R>::base_elastic(me);
        return CorrectedIntegrator<R>::energy(me, s, to_v3<R>(X), to_v3<R>(x_target), contacts, c, p, H_el);
      })
      .def_static("corrected_toi", [](const MeshT& me, Arr<R> x, Arr<R> ext, py::object fixed_mask, const ConT& c) {
        auto fm = py::array_t<int8_t, py::array::c_style | py::array::forcecast>::ensure(fixed_mask);
        std::vector<char> fixed(fm.data(), fm.data() + fm.size());
        return CorrectedIntegrator<R>::toi(me, to_v3<R>(x), to_v3<R>(ext), fixed, c, (const std::vector<RB>*)nullptr);
      })
      .def_static("compute_contacts", [opts](const MeshT& me, const StateT& s, py::object rigid, const std::string& broad) {
        Options<R> o = opts("indexed", broad);
        if (rigid.is_none()) return detect_all(me, s, (const std::vector<RB>*)nullptr, o.broad);
        std::vector<RB> store; for (auto it : rigid) store.push_back(it.cast<RB>());
        return detect_all(me, s, &store, o.broad);
      }, py::arg("mesh"), py::arg("state"), py::arg("rigid_bodies") = py::none(), py::arg("broad") = "literal")
      // One Newton gradient at the current state (integrator.cpp:246-396); strain constraints are rebuilt in `constraints`.
      .def_static("gradient", [opts](const MeshT& me, const StateT& s, Arr<R> x_target, const std::vector<CP>& contacts, ConT& c, const ParT& p) {
        std::vector<R> g(s.positions.size() * 3, R(0));
        Integrator<R>::gradient(me, s, to_v3<R>(x_target), contacts, c, p, opts("indexed", "literal"), g);
        return py::array_t<R>(py::ssize_t(g.size()), g.data());
      })
      .def_static("assemble", [opts](const MeshT& me, const StateT& s, const std::vector<CP>& contacts, ConT& c, const ParT& p) {
        return csr_dict(Integrator<R>::assemble(me, s, contacts, c, p, opts("indexed", "literal")));
      })
      .def_static("base_matrices", [](const MeshT& me, const StateT& s, const ParT& p) {
        Csr<R> Ht, He; Integrator<R>::base_matrices(me, s, p, false, Ht, He);
        py::dict d; d["H_total"] = csr_dict(Ht); d["H_elastic"] = csr_dict(He); return d;
      });

  m.def("edge_triangle_crossings", [](const MeshT& me, Arr<R> x, double cell) { return count_edge_triangle_crossings(me, to_v3<R>(x), cell); },
        py::arg("mesh"), py::arg("positions"), py::arg("cell") = 0.01,
        "Number of (edge, triangle) pairs sharing no vertex whose segment passes through the triangle");
  m.def("newton_trace", [](bool enable) {
    auto& tr = NewtonTrace::get();
    py::list out;
    for (const auto& r : tr.rows) {
      py::dict d; d["kind"] = r.kind; d["ids"] = py::make_tuple(r.ids[0], r.ids[1], r.ids[2], r.ids[3]);
      d["d0"] = r.d0; d["l"] = r.l; d["t"] = r.t; d["gnorm"] = r.gnorm; d["below_half"] = r.below_half;
      out.append(d);
    }
    tr.rows.clear(); tr.enabled = enable;
    return out;
  }, "Enable or disable the CORRECTED Newton trace; returns and clears the rows recorded so far");
  m.def("barrier_energy", &barrier_energy<R>);
  m.def("barrier_gradient", &barrier_gradient<R>);
  m.def("barrier_hessian", &barrier_hessian<R>);
  m.def("elastic_gradient", [](const MeshT& me) { std::vector<R> g; elastic_gradient(me, g); return py::array_t<R>(py::ssize_t(g.size()), g.data()); });
  m.def("elastic_energy", [](const MeshT& me) { return elastic_energy(me); });
  // CORRECTED (as-rigid-as-possible) membrane energy and its gradient at positions X
  m.def("arap_energy", [](const MeshT& me, Arr<R> X) { return elastic_energy_at(me, to_v3<R>(X)); });
  m.def("arap_gradient", [](const MeshT& me, Arr<R> X) {
    std::vector<R> g; elastic_gradient_at(me, to_v3<R>(X), g); return py::array_t<R>(py::ssize_t(g.size()), g.data()); });
  // sparse assembly from triplets with duplicates summed (what the reference leaves to setFromTriplets)
  m.def("csr_from_triplets", [](Index n, py::object ro, py::object co, py::object vo) {
    auto r = py::array_t<int64_t, py::array::c_style | py::array::forcecast>::ensure(ro);
    auto c = py::array_t<int64_t, py::array::c_style | py::array::forcecast>::ensure(co);
    auto v = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(vo);
    if (!r || !c || !v || r.size() != c.size() || r.size() != v.size()) throw py::value_error("triplet arrays");
    std::vector<Triplet<R>> t(size_t(r.size()));
    for (py::ssize_t k = 0; k < r.size(); ++k) {
      if (r.data()[k] < 0 || r.data()[k] >= n || c.data()[k] < 0 || c.data()[k] >= n) throw py::value_error("triplet index out of range");
      t[size_t(k)] = {Index(r.data()[k]), Index(c.data()[k]), R(v.data()[k])};
    }
    return csr_dict(Csr<R>::from_triplets(n, t)); });
  // thin SVD of one 3 x 2 matrix (the strain limits' and the membrane's svd32): U (3 x 2), sigma, V (2 x 2)
  m.def("svd32", [](py::object Fo) {
    auto F = py::array_t<double, py::array::c_style | py::array::forcecast>::ensure(Fo);
    if (!F || F.ndim() != 2 || F.shape(0) != 3 || F.shape(1) != 2) throw py::value_error("F must be 3 x 2");
    V3<double> c[2] = {V3<double>(F.at(0, 0), F.at(1, 0), F.at(2, 0)), V3<double>(F.at(0, 1), F.at(1, 1), F.at(2, 1))};
    Svd32<double> s; bool ok = svd32(c, s);
    py::array_t<double> U({py::ssize_t(3), py::ssize_t(2)}), S(2), V({py::ssize_t(2), py::ssize_t(2)});
    auto u = U.mutable_unchecked<2>(); auto v = V.mutable_unchecked<2>();
    for (int r = 0; r < 3; ++r) for (int q = 0; q < 2; ++q) u(r, q) = s.U[q][r];
    for (int r = 0; r < 2; ++r) for (int q = 0; q < 2; ++q) v(r, q) = s.V[r][q];
    S.mutable_data()[0] = s.sigma[0]; S.mutable_data()[1] = s.sigma[1];
    return py::make_tuple(U, S, V, ok); });
  // quadratic bending of the CORRECTED step: energy and gradient at X, and the hinges
  m.def("bending_energy", [](const MeshT& me, Arr<R> X) { std::vector<double> g(3 * me.vertices.size(), 0.0); return bending_at(me, to_v3<R>(X), g); });
  m.def("bending_gradient", [](const MeshT& me, Arr<R> X) {
    std::vector<double> g(3 * me.vertices.size(), 0.0); bending_at(me, to_v3<R>(X), g); return py::array_t<double>(py::ssize_t(g.size()), g.data()); });
  m.def("bending_hinges", [](const MeshT& me) {
    const py::ssize_t n = py::ssize_t(me.hinges.size());
    py::array_t<int32_t> v({n, py::ssize_t(4)}); py::array_t<double> w({n, py::ssize_t(4)}); py::array_t<double> c(n);
    auto vu = v.mutable_unchecked<2>(); auto wu = w.mutable_unchecked<2>(); auto cu = c.mutable_unchecked<1>();
    for (py::ssize_t h = 0; h < n; ++h) {
      for (int a = 0; a < 4; ++a) { vu(h, a) = me.hinges[size_t(h)].v[a]; wu(h, a) = me.hinges[size_t(h)].w[a]; }
      cu(h) = me.hinges[size_t(h)].c;
    }
    return py::make_tuple(v, w, c); });
  m.def("pin_stiffness", [](R mass, R dt, py::object off, py::object H, R min_gap) {
    auto h = Arr<R>::ensure(H); M3<R> Hm; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Hm(i, j) = h.at(i, j);
    return pin_stiffness(mass, dt, vec3<R>(off), Hm, min_gap); });
  m.def("wall_stiffness", [](R mass, R wall_gap, py::object n, py::object H, R min_gap) {
    auto h = Arr<R>::ensure(H); M3<R> Hm; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Hm(i, j) = h.at(i, j);
    return wall_stiffness(mass, wall_gap, vec3<R>(n), Hm, min_gap); });
  m.def("contact_stiffness", [](const CP& c, py::object masses, R dt, int n, py::object rows, py::object cols, py::object vals) {
    return contact_stiffness(c, vec_of<R>(masses), dt, csr_from<R>(n, rows, cols, vals), Lookup::INDEXED); });
  m.def("enforce_spd", [](py::object H) {
    auto h = Arr<R>::ensure(H); M3<R> Hm; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Hm(i, j) = h.at(i, j);
    M3<R> S = enforce_spd(Hm); py::array_t<R> o({3, 3}); auto u = o.template mutable_unchecked<2>();
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) u(i, j) = S(i, j); return o; });
  m.def("narrow_phase_point_triangle", [](py::object p, py::object a, py::object b, py::object c) {
    R d; V3<R> n, wp, wq; narrow_pt(vec3<R>(p), vec3<R>(a), vec3<R>(b), vec3<R>(c), d, n, wp, wq);
    return py::make_tuple(d, std::vector<R>{n.x, n.y, n.z}, std::vector<R>{wp.x, wp.y, wp.z}, std::vector<R>{wq.x, wq.y, wq.z}); });
  m.def("narrow_phase_edge_edge", [](py::object p0, py::object p1, py::object q0, py::object q1) {
    R d; V3<R> n, wp, wq; narrow_ee(vec3<R>(p0), vec3<R>(p1), vec3<R>(q0), vec3<R>(q1), d, n, wp, wq);
    return py::make_tuple(d, std::vector<R>{n.x, n.y, n.z}, std::vector<R>{wp.x, wp.y, wp.z}, std::vector<R>{wq.x, wq.y, wq.z}); });
  m.def("line_search", [](Arr<R> x, py::object dir, const std::vector<CP>& contacts, py::list pins, py::object wn, R woff, R ext) {
    std::vector<Pin<R>> pv;
    for (auto it : pins) { auto tup = it.cast<py::tuple>(); Pin<R> p; p.vertex_idx = tup[0].cast<Index>(); p.target_position = vec3<R>(tup[1]); pv.push_back(p); }
    return line_search(to_v3<R>(x), vec_of<R>(dir), contacts, pv, vec3<R>(wn), woff, ext); },
    py::arg("positions"), py::arg("direction"), py::arg("contacts"), py::arg("pins"), py::arg("wall_normal"), py::arg("wall_offset"), py::arg("extension") = R(1.25));
  m.def("pcg_solve", [](int n, py::object rows, py::object cols, py::object vals, py::object b, R tol, int max_iters) {
    Csr<R> A = csr_from<R>(n, rows, cols, vals);
    std::vector<R> bb = vec_of<R>(b), x(bb.size(), R(0));
    auto res = pcg_solve(A, bb, x, tol, max_iters);
    return py::make_tuple(py::array_t<R>(py::ssize_t(x.size()), x.data()), res.converged, res.iters, res.rel_res); });
  m.def("pcg_solve_csr", [](int n, py::object rowptr, py::object cols, py::object vals, py::object b, R tol, int max_iters) {
    Csr<R> A; A.n = n;
    auto rp = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(rowptr);
    auto cc = py::array_t<int32_t, py::array::c_style | py::array::forcecast>::ensure(cols);
    A.rowptr.assign(rp.data(), rp.data() + rp.size()); A.cols.assign(cc.data(), cc.data() + cc.size()); A.vals = vec_of<R>(vals);
    std::vector<R> bb = vec_of<R>(b), x(bb.size(), R(0));
    auto res = pcg_solve(A, bb, x, tol, max_iters);
    return py::make_tuple(py::array_t<R>(py::ssize_t(x.size()), x.data()), res.converged, res.iters, res.rel_res); });
  m.def("broad_phase", [](const MeshT& me, Arr<R> x, const std::string& mode, R pad) {
    std::vector<std::pair<int, int>> vt, ee; broad_phase(me, to_v3<R>(x), to_broad(mode), vt, ee, pad);
    return py::make_tuple(vt, ee); }, py::arg("mesh"), py::arg("positions"), py::arg("mode"), py::arg("pad") = R(0));
  m.def("bvh_node_count", [](const MeshT& me, Arr<R> x) { return bvh_build(triangle_boxes(me, to_v3<R>(x))).nodes.size(); });
}

}  // namespace

PYBIND11_MODULE(ando_oracle, m) {
  m.doc() = "CPU oracle of the AndoSim implicit step (test infrastructure; FP64 and FP32 restatements).";
  py::enum_<ContactType>(m, "ContactType")
      .value("POINT_TRIANGLE", ContactType::POINT_TRIANGLE).value("EDGE_EDGE", ContactType::EDGE_EDGE)
      .value("WALL", ContactType::WALL).value("RIGID_POINT_TRIANGLE", ContactType::RIGID_POINT_TRIANGLE).export_values();
  auto f64 = m.def_submodule("f64", "FP64 restatement");
  auto f32 = m.def_submodule("f32", "FP32 restatement (the reference's default Real=float build)");
  bind<double>(f64);
  bind<float>(f32);
}
