"""The projected exact membrane Hessian of the oracle (CORRECTED, membrane_hessian = 1).

The constant Hessian 2k (G G^T) (x) I3 of the as-rigid-as-possible membrane
holds the face's rotation fixed, so it resists rotations that cost no energy:
a strip clamped along one side creeps down instead of swinging. The
projected form clamps the eigenvalues of the exact Hessian 2k (I - dR/dF) at
zero per face. Pinned here in FP64:

* where every eigenvalue is already non-negative (faces stretched in both
  directions) it is the central-difference Jacobian of the membrane gradient,
  which the fixed-rotation Hessian is not;
* it is positive semidefinite at rest and under compression;
* the clamped strip swings down with it and creeps without it.
"""
from __future__ import annotations

import numpy as np

from andosim_b200 import scenes
from conftest import oracle_scene
from test_oracle_fd import H


def sheet_scene(n=3, size=0.02):
    v = scenes.grid_plane(n, size)
    v[:, 2] = 0.3
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
    return scenes.Scene("membrane", v, scenes.grid_triangles(n, n), mat, scenes.cloth_params(enable_strain_limiting=False), [], [])


def elastic_hessian(O, sc, x, mode):
    m, s, p = oracle_scene(O, sc)
    p.membrane_hessian = mode
    s.set_positions(x)
    s.set_velocities(np.zeros_like(x))
    res = O.Integrator.corrected_system(m, s, x, np.zeros(len(x), np.int8), O.Constraints(), p)
    hs = res["hessian"]
    Hd = np.zeros((x.size, x.size))
    for r in range(hs["n"]):
        for k in range(hs["rowptr"][r], hs["rowptr"][r + 1]):
            Hd[r, hs["cols"][k]] += hs["vals"][k]
    Hd -= np.diag(np.repeat(np.asarray(s.get_masses()), 3) / p.dt ** 2)    # inertia
    return m, Hd


def test_projected_hessian_is_the_exact_jacobian_when_stretched(oracle):
    O = oracle.f64
    sc = sheet_scene()
    x = sc.vertices.copy()
    x[:, :2] *= 1.08
    x += np.random.default_rng(0).normal(scale=2e-4, size=x.shape)
    m, Hp = elastic_hessian(O, sc, x, 1)
    _, Hf = elastic_hessian(O, sc, x, 0)
    J = np.zeros_like(Hp)
    flat = x.ravel()
    for i in range(flat.size):
        xp = flat.copy(); xp[i] += H
        xm = flat.copy(); xm[i] -= H
        J[:, i] = (O.arap_gradient(m, xp.reshape(x.shape)) - O.arap_gradient(m, xm.reshape(x.shape))) / (2 * H)
    scale = np.abs(J).max()
    assert np.abs(Hp - J).max() <= 1e-6 * scale
    assert np.abs(Hf - J).max() >= 0.1 * scale            # the fixed-rotation form is not the Hessian


def test_projected_hessian_is_positive_semidefinite(oracle):
    O = oracle.f64
    sc = sheet_scene(n=4)
    rng = np.random.default_rng(1)
    for squeeze in (1.0, 0.95, 0.7):
        x = sc.vertices.copy()
        x[:, :2] *= squeeze
        if squeeze != 1.0:
            x += rng.normal(scale=5e-4, size=x.shape)
        _, Hp = elastic_hessian(O, sc, x, 1)
        assert np.abs(Hp - Hp.T).max() <= 1e-9 * np.abs(Hp).max()
        assert np.linalg.eigvalsh(Hp).min() >= -1e-9 * np.abs(Hp).max(), squeeze


def test_clamped_strip_swings_with_the_projected_hessian(oracle):
    O = oracle.f64

    def sag(mode, frames=10):
        n = 8
        v = scenes.grid_plane(n, 0.1)
        v[:, 2] = 0.3
        mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
        sc = scenes.Scene("strip", v, scenes.grid_triangles(n, n), mat, scenes.cloth_params(), [], [])
        m, s, p = oracle_scene(O, sc)
        p.membrane_hessian = mode
        c = O.Constraints()
        for i in range(2 * n):                   # the two rows along y = 0 clamped
            c.add_pin(i, v[i])
        for _ in range(frames):
            s.apply_gravity(np.array([0.0, 0.0, -9.81]), p.dt)
            O.Integrator.step(m, s, c, p, semantics="corrected")
        return 0.3 - float(np.asarray(s.get_positions())[:, 2].min())

    creep, swing = sag(0), sag(1)
    assert creep < 5e-3, creep
    assert swing > 5e-2, swing                   # 8 cm in 10 frames against free fall's 13.6 cm


def test_projected_hessian_with_bending_is_the_exact_jacobian(oracle):
    """With bending on as well, the assembled elastic Hessian (projected membrane
    plus the constant bending Hessian) is the central-difference Jacobian of the
    whole elastic gradient where no membrane eigenvalue is clamped."""
    O = oracle.f64
    v = scenes.grid_plane(4, 0.03)
    v[:, 2] = 0.3
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=2e-4)
    sc = scenes.Scene("membrane_bending", v, scenes.grid_triangles(4, 4), mat, scenes.cloth_params(enable_strain_limiting=False), [], [])
    x = v.copy()
    x[:, :2] *= 1.08                            # every face stretched both ways: nothing clamped
    x += np.random.default_rng(4).normal(scale=2e-4, size=x.shape)
    m, Hp = elastic_hessian(O, sc, x, 1)
    J = np.zeros_like(Hp)
    flat = x.ravel()
    for i in range(flat.size):
        xp = flat.copy(); xp[i] += H
        xm = flat.copy(); xm[i] -= H
        J[:, i] = (O.arap_gradient(m, xp.reshape(x.shape)) - O.arap_gradient(m, xm.reshape(x.shape))) / (2 * H)
    assert np.abs(O.bending_gradient(m, x)).max() > 0
    assert np.abs(Hp - J).max() <= 1e-6 * np.abs(J).max()
