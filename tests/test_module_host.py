"""Host-side parts of the ando_barrier_core module (no GPU needed)."""
from __future__ import annotations

import numpy as np

from andosim_b200 import scenes
from conftest import oracle_scene


def dense(csr, n):
    H = np.zeros((n, n))
    for r in range(n):
        for k in range(csr["rowptr"][r], csr["rowptr"][r + 1]):
            H[r, csr["cols"][k]] += csr["vals"][k]
    return H


def test_elasticity_compute_hessian_matches_oracle(core, oracle):
    """Elasticity.compute_hessian (bindings.cpp:433-434 -> elasticity.cpp:63-91):
    81 SPD-clamped triplets per face, summing to the oracle's H_elastic."""
    sc = scenes.c1(n=6)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    st = core.State()
    trip = []
    out = core.Elasticity.compute_hessian(m, st, trip)
    assert out is trip and len(trip) == 81 * sc.num_triangles
    n = 3 * sc.num_vertices
    H = np.zeros((n, n))
    for r, c, v in trip:
        H[r, c] += v
    O = oracle.f64
    mo, so, p = oracle_scene(O, sc)
    Ho = dense(O.Integrator.base_matrices(mo, so, p)["H_elastic"], n)
    assert np.abs(H - Ho).max() <= 1e-6 * np.abs(Ho).max()
    assert len(core.Elasticity.compute_hessian(m, st)) == len(trip)


def test_unknown_gpu_knobs_are_refused_before_any_device_call(core):
    """SimParams' GPU-only string fields are checked when a step converts them,
    before a context exists: a typo raises ValueError, never a silent default."""
    import pytest

    sc = scenes.c1(n=4)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    st = core.State()
    st.initialize(m)
    for field, bad in (("semantics", "corected"), ("preconditioner", "jacobi"), ("membrane_hessian", "exact")):
        p = core.SimParams()
        setattr(p, field, bad)
        with pytest.raises(ValueError, match=field):
            core.Integrator.step(m, st, core.Constraints(), p)
    p = core.SimParams()
    assert (p.semantics, p.preconditioner, p.membrane_hessian) == ("reference", "block_jacobi", "fixed_rotation")


def test_module_barrier_functions_meet_the_reference_expectations(core):
    """The module's barrier_energy / gradient / hessian (bindings.cpp:421-442 of
    the reference) against tests/test_barrier_derivatives.cpp:21-236: closed
    forms at g = 5 mm, g_max = 10 mm, k = 1000, central differences, the
    domain edges and the force direction, in the reference's FP32 Real."""
    import pytest

    g, gm, k = 0.005, 0.01, 1000.0
    assert core.barrier_energy(g, gm, k) == pytest.approx(6.25e-3, rel=1e-5)
    assert core.barrier_gradient(g, gm, k) == pytest.approx(-3.75, rel=1e-5)
    assert core.barrier_hessian(g, gm, k) == pytest.approx(1500.0, rel=1e-5)
    assert core.barrier_energy(0.015, gm, k) == 0.0 and core.barrier_energy(gm, gm, k) == 0.0
    assert core.barrier_energy(-0.001, gm, k) > 0.0
    assert core.barrier_gradient(gm, gm, k) == 0.0 and core.barrier_hessian(gm, gm, k) == 0.0
    g1, g2, g3 = (core.barrier_gradient(x, gm, k) for x in (0.002, 0.005, 0.009))
    assert g1 < 0 and g2 < 0 and g3 < 0 and abs(g1) > abs(g2) > abs(g3)
    h = 1e-4                                  # FP32 arithmetic: a larger step than the FP64 oracle's
    for i in range(1, 10):
        x = i / 10.0 * gm
        fd_g = (core.barrier_energy(x + h, gm, k) - core.barrier_energy(x - h, gm, k)) / (2 * h)
        fd_h = (core.barrier_gradient(x + h, gm, k) - core.barrier_gradient(x - h, gm, k)) / (2 * h)
        assert abs(core.barrier_gradient(x, gm, k) - fd_g) / (abs(fd_g) + 1e-10) < 1e-2
        assert abs(core.barrier_hessian(x, gm, k) - fd_h) / (abs(fd_h) + 1e-10) < 1e-2


def test_elasticity_energy_and_gradient_match_oracle(core, oracle):
    """Elasticity.compute_energy / compute_gradient (the reference's binding,
    elasticity.cpp:18-61 on the mesh's own vertices) after Mesh.set_positions
    moved them off the rest shape: the module's host evaluation against the
    FP64 oracle's."""
    sc = scenes.c1(n=6)
    rng = np.random.default_rng(8)
    x = sc.vertices + rng.normal(scale=2e-3, size=sc.vertices.shape)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    m.set_positions(x)
    st = core.State()
    st.initialize(m)
    g = np.zeros(3 * sc.num_vertices, dtype=np.float32)
    core.Elasticity.compute_gradient(m, st, g)
    e = core.Elasticity.compute_energy(m, st)
    O = oracle.f64
    mo, _, _ = oracle_scene(O, sc)
    mo.set_positions(x)
    go = np.asarray(O.elastic_gradient(mo))
    eo = O.elastic_energy(mo)
    assert np.abs(go).max() > 0 and eo > 0
    assert np.abs(g - go).max() <= 1e-5 * np.abs(go).max()
    assert abs(e - eo) <= 1e-5 * eo


def test_energy_tracker_on_the_host_copy(core):
    """EnergyTracker (energy_tracker.cpp:7-76) on a state that has no device
    context yet: kinetic energy, momenta and the largest speed from the host
    arrays, against numpy."""
    sc = scenes.c1(n=5)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    st = core.State()
    st.initialize(m)
    rng = np.random.default_rng(9)
    v = rng.normal(size=sc.vertices.shape)
    st.set_velocities64(v)
    mass = np.asarray(st.get_masses(), dtype=np.float64)
    x = st.get_positions64()
    p = mass[:, None] * v
    ke = 0.5 * (mass * (v ** 2).sum(1)).sum()
    assert abs(core.EnergyTracker.compute_kinetic_energy(st) - ke) <= 1e-6 * ke
    np.testing.assert_allclose(core.EnergyTracker.compute_linear_momentum(st), p.sum(0), rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(core.EnergyTracker.compute_angular_momentum(st), np.cross(x, p).sum(0), rtol=1e-5, atol=1e-7)
    assert abs(core.EnergyTracker.compute_max_velocity(st) - np.linalg.norm(v, axis=1).max()) <= 1e-6 * np.linalg.norm(v, axis=1).max()
    d = core.EnergyTracker.compute(m, st, core.Constraints(), core.SimParams())
    assert abs(d.kinetic_energy - ke) <= 1e-6 * ke and d.total_energy >= d.kinetic_energy
