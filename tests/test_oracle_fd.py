"""Central-difference checks of the oracle's Newton gradients, FP64.

The reference checks its scalar barrier this way (tests/test_barrier_derivatives.cpp:21-236:
central differences, h = 1e-5). These tests extend that pattern to every term of the Newton
gradient the oracle assembles: membrane elasticity, pins, walls, point-triangle and edge-edge
contacts and strain limits. Each term's stiffness is frozen at the state, as the Newton
iteration freezes it, so the gradient must be the exact derivative of the frozen-stiffness
energy (CORRECTED: `Integrator.corrected_energy`; REFERENCE: composed below from the oracle's
own barrier and stiffness functions).

Two reference behaviours are not gradients of any energy and are recorded as such instead:
its membrane force formula away from rest (elasticity.cpp:18-61 drops the rotation of its
edge-aligned frame; REFERENCE only evaluates it at rest, where it is zero), and its contact
terms, which keep the detection-time gap for the whole step (barrier.cpp:67-149).
"""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes
from conftest import oracle_scene

H = 1e-7          # central-difference step (m)
REL = 1e-5        # relative tolerance on the largest gradient entry


def fd_gradient(energy, x):
    g = np.zeros(x.size)
    flat = x.ravel()
    for i in range(flat.size):
        xp = flat.copy(); xp[i] += H
        xm = flat.copy(); xm[i] -= H
        g[i] = (energy(xp.reshape(x.shape)) - energy(xm.reshape(x.shape))) / (2 * H)
    return g


def assert_matches(g, fd, rel=REL):
    scale = np.abs(fd).max()
    assert scale > 0
    err = np.abs(np.asarray(g, dtype=np.float64) - fd).max() / scale
    assert err <= rel, err


def sheet(n=4, size=0.03, z=0.3, shift=(0.0, 0.0)):
    v = scenes.grid_plane(n, size)
    v[:, 0] += shift[0]
    v[:, 1] += shift[1]
    v[:, 2] = z
    return v


def scene(vertices, triangles, params=None, pins=(), walls=()):
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
    p = scenes.cloth_params(**(params or {}))
    return scenes.Scene("fd", vertices, triangles, mat, p, list(pins), list(walls))


def corrected_setup(oracle, sc, x, v):
    O = oracle.f64
    m, s, p = oracle_scene(O, sc)
    s.set_positions(x)
    s.set_velocities(v)
    c = O.Constraints()
    for i, t in sc.pins:
        c.add_pin(int(i), t)
    for n, o, gp in sc.walls:
        c.add_wall(n, o, gp)
    xt = x + p.dt * v
    return O, m, s, p, c, xt


def corrected_check(oracle, sc, x, v, expect_contacts=None):
    O, m, s, p, c, xt = corrected_setup(oracle, sc, x, v)
    res = O.Integrator.corrected_system(m, s, xt, np.zeros(len(x), np.int8), c, p)
    if expect_contacts is not None:
        kinds = {int(ct.type) for ct in res["contacts"]}
        assert kinds >= expect_contacts, kinds
    fd = fd_gradient(lambda X: O.Integrator.corrected_energy(m, s, X, xt, c, p), x)
    assert_matches(res["gradient"], fd)


# ---------------------------------------------------------------- elasticity
def test_arap_gradient_matches_central_differences(oracle):
    O = oracle.f64
    v = sheet(n=3, size=0.02)
    sc = scene(v, scenes.grid_triangles(3, 3))
    m, _, _ = oracle_scene(O, sc)
    x = v + np.random.default_rng(1).normal(scale=3e-3, size=v.shape)
    assert_matches(O.arap_gradient(m, x), fd_gradient(lambda X: O.arap_energy(m, X), x))
    assert np.abs(O.arap_gradient(m, v + np.array([0.1, -0.2, 0.3]))).max() < 1e-9   # rigid motion: no force


def test_arap_constant_hessian_is_the_fixed_rotation_jacobian(oracle):
    """The assembled CORRECTED elastic Hessian 2k (G G^T) (x) I3 is the Jacobian of
    2k (F - R0) G^T with the rotation R0 of the state held fixed; that gradient
    equals the oracle's membrane gradient at the state."""
    O = oracle.f64
    v = sheet(n=3, size=0.02)
    tris = scenes.grid_triangles(3, 3)
    sc = scene(v, tris, params=dict(enable_strain_limiting=False))
    m, s, p = oracle_scene(O, sc)
    x = v + np.random.default_rng(2).normal(scale=2e-3, size=v.shape)
    mu = 1e5 / (2 * 1.3)
    D, A = [], []
    for t in tris:
        E = np.stack([v[t[1]] - v[t[0]], v[t[2]] - v[t[0]]], axis=1)[:2]   # rest edges in the plane
        D.append(np.linalg.inv(E)); A.append(0.5 * abs(np.linalg.det(E)))
    R0 = []
    for t, Di in zip(tris, D):
        F = np.stack([x[t[1]] - x[t[0]], x[t[2]] - x[t[0]]], axis=1) @ Di
        U, _, Vt = np.linalg.svd(F, full_matrices=False)
        R0.append(U @ Vt)

    def fixed_r_gradient(X):
        g = np.zeros_like(X)
        for t, Di, a, R in zip(tris, D, A, R0):
            F = np.stack([X[t[1]] - X[t[0]], X[t[2]] - X[t[0]]], axis=1) @ Di
            G = np.array([[-1.0, -1.0], [1.0, 0.0], [0.0, 1.0]]) @ Di
            P = 2 * a * 1e-3 * mu * (F - R)
            for k in range(3):
                g[t[k]] += P @ G[k]
        return g.ravel()

    assert_matches(O.arap_gradient(m, x), fixed_r_gradient(x))
    s.set_positions(x)
    s.set_velocities(np.zeros_like(x))
    res = O.Integrator.corrected_system(m, s, x, np.zeros(len(x), np.int8), O.Constraints(), p)
    Hd = np.zeros((x.size, x.size))
    hs = res["hessian"]
    for r in range(hs["n"]):
        for k in range(hs["rowptr"][r], hs["rowptr"][r + 1]):
            Hd[r, hs["cols"][k]] += hs["vals"][k]
    Hd -= np.diag(np.repeat(np.asarray(s.get_masses()), 3) / p.dt ** 2)   # inertia term
    J = np.zeros_like(Hd)
    flat = x.ravel()
    for i in range(flat.size):
        xp = flat.copy(); xp[i] += H
        xm = flat.copy(); xm[i] -= H
        J[:, i] = (fixed_r_gradient(xp.reshape(x.shape)) - fixed_r_gradient(xm.reshape(x.shape))) / (2 * H)
    assert np.abs(Hd - J).max() <= 1e-6 * np.abs(J).max()


def test_reference_membrane_force_is_not_conservative_away_from_rest(oracle):
    O = oracle.f64
    v = sheet(n=2, size=0.01)
    sc = scene(v, scenes.grid_triangles(2, 2))
    m, _, _ = oracle_scene(O, sc)
    assert np.abs(O.elastic_gradient(m)).max() == 0.0        # at rest: zero, the only place REFERENCE uses it
    x = v + np.random.default_rng(0).normal(scale=2e-3, size=v.shape)

    def energy(X):
        m.set_positions(X)
        return O.elastic_energy(m)
    fd = fd_gradient(energy, x)
    m.set_positions(x)
    err = np.abs(O.elastic_gradient(m) - fd).max() / np.abs(fd).max()
    assert err > 0.1


# ------------------------------------------------------- CORRECTED Newton gradient
def test_corrected_gradient_inertia_elastic_pins(oracle):
    v = sheet()
    sc = scene(v, scenes.grid_triangles(4, 4), params=dict(enable_strain_limiting=False),
               pins=[(0, v[0] + np.array([0.002, 0.0, 0.001])), (15, v[15] + np.array([-0.001, 0.003, 0.0]))])
    rng = np.random.default_rng(3)
    corrected_check(oracle, sc, v + rng.normal(scale=1e-3, size=v.shape), rng.normal(scale=0.2, size=v.shape))


def test_corrected_gradient_walls(oracle):
    v = sheet(z=0.0004)
    sc = scene(v, scenes.grid_triangles(4, 4), params=dict(enable_strain_limiting=False), walls=[scenes.ground()])
    rng = np.random.default_rng(4)
    x = v.copy()
    x[:, 2] = rng.uniform(1e-4, 9e-4, size=len(x))      # every vertex inside the wall's activation distance
    corrected_check(oracle, sc, x, rng.normal(scale=0.1, size=v.shape))


def test_corrected_gradient_self_contact(oracle):
    h = 0.03 / 3
    a = sheet(z=0.3)
    b = sheet(z=0.3006, shift=(0.37 * h, 0.21 * h))
    tris = np.concatenate([scenes.grid_triangles(4, 4), scenes.grid_triangles(4, 4, offset=16)])
    sc = scene(np.concatenate([a, b]), tris, params=dict(enable_strain_limiting=False))
    rng = np.random.default_rng(5)
    x = sc.vertices + rng.normal(scale=5e-5, size=sc.vertices.shape)
    corrected_check(oracle, sc, x, rng.normal(scale=0.1, size=x.shape), expect_contacts={0, 1})


def test_corrected_gradient_strain_limits(oracle):
    v = sheet()
    sc = scene(v, scenes.grid_triangles(4, 4))
    x = v.copy()
    x[:, 0] *= 1.07                    # 7 % stretch along x: inside the 5 % + 5 % barrier band
    x[:, 1] *= 1.02
    x += np.random.default_rng(6).normal(scale=5e-5, size=x.shape)
    O, m, s, p, c, xt = corrected_setup(oracle, sc, x, np.zeros_like(x))
    O.Integrator.corrected_system(m, s, xt, np.zeros(len(x), np.int8), c, p)
    assert c.num_strain_limits() > 0
    corrected_check(oracle, sc, x, np.zeros_like(x))


# ------------------------------------------------------- REFERENCE Newton gradient
def test_reference_gradient_walls_and_pins(oracle):
    """REFERENCE walls (k = m / wall_gap^2 + n^T H n, stiffness.cpp:146-172) and
    pins (repelling barrier on |x - target|, barrier.cpp:161-215, k frozen at the
    state) against the frozen-stiffness energy built from the oracle's barrier
    and stiffness functions."""
    O = oracle.f64
    v = sheet(n=2, size=0.02, z=0.0005)
    tris = scenes.grid_triangles(2, 2)
    targets = [(0, v[0] + np.array([0.0003, 0.0, 0.0002])), (3, v[3] + np.array([0.0, -0.0004, 0.0]))]
    sc = scene(v, tris, params=dict(enable_strain_limiting=False), pins=targets, walls=[scenes.ground()])
    m, s, p = oracle_scene(O, sc)
    c = O.Constraints()
    for i, t in targets:
        c.add_pin(i, t)
    c.add_wall(np.array([0.0, 0.0, 1.0]), 0.0, 1e-3)
    x = v.copy()
    s.set_positions(x)
    xt = x.copy()
    g = np.asarray(O.Integrator.gradient(m, s, xt, [], c, p))
    He = O.Integrator.base_matrices(m, s, p)["H_total"]
    mass = np.asarray(s.get_masses())

    def block(i):
        Hb = np.zeros((3, 3))
        for r in range(3):
            row = 3 * i + r
            for k in range(He["rowptr"][row], He["rowptr"][row + 1]):
                col = He["cols"][k]
                if col // 3 == i:
                    Hb[r, col % 3] += He["vals"][k]
        return Hb
    kw = [O.wall_stiffness(mass[i], p.wall_gap, [0, 0, 1.0], block(i), p.min_gap) for i in range(len(x))]
    kp = {i: O.pin_stiffness(mass[i], p.dt, x[i] - t, block(i), p.min_gap) for i, t in targets}

    def energy(X):
        e = 0.0
        for i in range(len(X)):
            e += O.barrier_energy(X[i, 2], p.contact_gap_max, kw[i])
        for i, t in targets:
            e += O.barrier_energy(float(np.linalg.norm(X[i] - t)), p.contact_gap_max, kp[i])
        return e
    assert_matches(g, fd_gradient(energy, x))
