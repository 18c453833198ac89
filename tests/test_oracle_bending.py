"""The oracle's quadratic bending term (CORRECTED semantics, bending_stiffness > 0).

The reference declares Material::bending_stiffness (types.h:56) and never reads
it, so the term has no reference values to match; it is pinned here by its
mathematics instead, in FP64:

* the gradient is the central-difference derivative of the energy (the
  pattern of tests/test_barrier_derivatives.cpp:21-236), and the assembled
  CORRECTED Hessian gains exactly the term's constant Hessian;
* the energy and force vanish for every affine map of the flat rest sheet
  (stretching is the membrane's business, rigid motion is free);
* an isometric fold by a dihedral angle t about one interior edge costs
  k_b 3 |e|^2 / A_e (2 sin(t/2))^2, the discrete-shell hinge energy
  k_b 3 |e|^2 / A_e t^2 to second order in t;
* a sheet pinned along one side sags less with bending stiffness than without.
"""
from __future__ import annotations

import numpy as np

from andosim_b200 import scenes
from conftest import oracle_scene
from test_oracle_fd import H, assert_matches, fd_gradient

KB = 2e-4


def bending_scene(n=4, size=0.03, kb=KB, params=None):
    v = scenes.grid_plane(n, size)
    v[:, 2] = 0.3
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=kb)
    return scenes.Scene("bend", v, scenes.grid_triangles(n, n), mat, scenes.cloth_params(**(params or {})), [], [])


def test_hinges_are_the_interior_edges(oracle):
    O = oracle.f64
    n = 5
    m, _, _ = oracle_scene(O, bending_scene(n=n))
    v, w, c = O.bending_hinges(m)
    E = 3 * (n - 1) ** 2 + 2 * (n - 1)
    assert len(v) == E - 4 * (n - 1)                      # every edge but the boundary ones
    np.testing.assert_allclose(w.sum(1), 0.0, atol=1e-12)  # constants are annihilated
    assert (c > 0).all()


def test_bending_gradient_matches_central_differences(oracle):
    O = oracle.f64
    sc = bending_scene()
    m, _, _ = oracle_scene(O, sc)
    x = sc.vertices + np.random.default_rng(3).normal(scale=2e-3, size=sc.vertices.shape)
    assert O.bending_energy(m, x) > 0
    assert_matches(O.bending_gradient(m, x), fd_gradient(lambda X: O.bending_energy(m, X), x))


def test_bending_vanishes_on_affine_maps_of_the_rest_sheet(oracle):
    O = oracle.f64
    sc = bending_scene()
    m, _, _ = oracle_scene(O, sc)
    rng = np.random.default_rng(4)
    A = np.eye(3) + rng.normal(scale=0.2, size=(3, 3))
    x = sc.vertices @ A.T + rng.normal(size=3)
    scale = KB * np.abs(x).max()
    assert np.abs(O.bending_gradient(m, x)).max() < 1e-9 * scale
    assert abs(O.bending_energy(m, x)) < 1e-12 * KB


def test_fold_about_one_edge_is_the_hinge_energy(oracle):
    O = oracle.f64
    sc = bending_scene(n=3, size=0.02)
    m, _, _ = oracle_scene(O, sc)
    v, w, c = O.bending_hinges(m)
    x0 = sc.vertices
    # the interior diagonal edge of the first cell: fold the vertex on one side about it
    h = 0
    i, j, k, l = v[h]
    e = x0[j] - x0[i]
    axis = e / np.linalg.norm(e)
    A = 6.0 / c[h]
    for t in (1e-3, 1e-2, 0.1):
        p = x0[l] - x0[i]
        rot = x0[i] + p * np.cos(t) + np.cross(axis, p) * np.sin(t) + axis * (axis @ p) * (1 - np.cos(t))
        x = x0.copy()
        x[l] = rot
        # only hinges that hold l see the move; restrict the energy to hinge h by
        # subtracting the others' share computed from the stencil itself
        s = (w[:, :, None] * x[v]).sum(1)
        per = 0.5 * KB * c * (s ** 2).sum(1)
        assert abs(per.sum() - O.bending_energy(m, x)) <= 1e-12 * per.sum()
        want = KB * 3 * (e @ e) / A * (2 * np.sin(t / 2)) ** 2
        assert abs(per[h] - want) <= 1e-9 * want, (t, per[h], want)
        assert abs(per[h] / (KB * 3 * (e @ e) / A * t * t) - 1) <= t * t / 12 + 1e-9


def test_corrected_hessian_gains_the_bending_hessian(oracle):
    O = oracle.f64
    params = dict(enable_strain_limiting=False)

    def hessian(kb):
        sc = bending_scene(kb=kb, params=params)
        m, s, p = oracle_scene(O, sc)
        x = sc.vertices + np.random.default_rng(5).normal(scale=1e-3, size=sc.vertices.shape)
        s.set_positions(x)
        s.set_velocities(np.zeros_like(x))
        res = O.Integrator.corrected_system(m, s, x, np.zeros(len(x), np.int8), O.Constraints(), p)
        hs = res["hessian"]
        Hd = np.zeros((x.size, x.size))
        for r in range(hs["n"]):
            for q in range(hs["rowptr"][r], hs["rowptr"][r + 1]):
                Hd[r, hs["cols"][q]] += hs["vals"][q]
        return m, x, Hd, np.asarray(res["gradient"])

    m, x, Hb, gb = hessian(KB)
    _, _, H0, g0 = hessian(0.0)
    Q = Hb - H0
    # the difference is the Jacobian of the bending gradient (central differences; exact for a quadratic)
    J = np.zeros_like(Q)
    flat = x.ravel()
    for i in range(flat.size):
        xp = flat.copy(); xp[i] += H
        xm = flat.copy(); xm[i] -= H
        J[:, i] = (O.bending_gradient(m, xp.reshape(x.shape)) - O.bending_gradient(m, xm.reshape(x.shape))) / (2 * H)
    assert np.abs(Q - J).max() <= 1e-6 * np.abs(J).max()
    np.testing.assert_allclose(gb - g0, O.bending_gradient(m, x), rtol=0, atol=1e-9 * np.abs(gb - g0).max())
    assert np.linalg.eigvalsh(0.5 * (Q + Q.T)).min() > -1e-9 * np.abs(Q).max()   # positive semidefinite


def test_pinned_sheet_sags_less_with_bending(oracle):
    O = oracle.f64

    def lowest(kb):
        n = 8
        sc = bending_scene(n=n, size=0.1, kb=kb)
        m, s, p = oracle_scene(O, sc)
        c = O.Constraints()
        for i in range(n):                      # the y = 0 side clamped (two rows)
            c.add_pin(i, sc.vertices[i])
            c.add_pin(n + i, sc.vertices[n + i])
        for _ in range(10):
            s.apply_gravity(np.array([0.0, 0.0, -9.81]), p.dt)
            O.Integrator.step(m, s, c, p, semantics="corrected")
        return float(np.asarray(s.get_positions())[:, 2].min())

    free, stiff = lowest(0.0), lowest(5e-3)
    assert stiff > free + 1e-3, (free, stiff)
