"""The CPU oracle against the reference's own known-answer tests.

Each case re-encodes an assertion of the reference test suite (file:line given
per test) and checks it on the FP32 restatement (the reference's default
Real=float build) and on the FP64 one.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

PRECISIONS = ["f32", "f64"]


def mod_of(oracle, prec):
    return getattr(oracle, prec)


# tests/test_barrier_derivatives.cpp:21-236
@pytest.mark.parametrize("prec", PRECISIONS)
def test_barrier_closed_forms(oracle, prec):
    O = mod_of(oracle, prec)
    g, gm, k = 0.005, 0.01, 1000.0
    assert O.barrier_energy(g, gm, k) == pytest.approx(6.25e-3, rel=1e-5)
    assert O.barrier_gradient(g, gm, k) == pytest.approx(-3.75, rel=1e-5)
    assert O.barrier_hessian(g, gm, k) == pytest.approx(1500.0, rel=1e-5)
    h = 1e-5
    fd_g = (O.barrier_energy(g + h, gm, k) - O.barrier_energy(g - h, gm, k)) / (2 * h)
    fd_h = (O.barrier_gradient(g + h, gm, k) - O.barrier_gradient(g - h, gm, k)) / (2 * h)
    assert abs(O.barrier_gradient(g, gm, k) - fd_g) / abs(fd_g) < 1e-3
    assert abs(O.barrier_hessian(g, gm, k) - fd_h) / abs(fd_h) < 1e-3
    assert O.barrier_energy(0.015, gm, k) == 0.0
    assert O.barrier_energy(gm, gm, k) == 0.0
    assert O.barrier_energy(-0.001, gm, k) > 0.0
    assert O.barrier_gradient(gm, gm, k) == 0.0 and O.barrier_hessian(gm, gm, k) == 0.0
    g1, g2, g3 = (O.barrier_gradient(x, gm, k) for x in (0.002, 0.005, 0.009))
    assert g1 < 0 and g2 < 0 and g3 < 0 and abs(g1) > abs(g2) > abs(g3)
    for i in range(1, 10):
        x = i / 10.0 * gm
        an = O.barrier_gradient(x, gm, k)
        nu = (O.barrier_energy(x + h, gm, k) - O.barrier_energy(x - h, gm, k)) / (2 * h)
        assert abs(an - nu) / (abs(nu) + 1e-10) < 1e-3


# tests/test_basic.cpp:193-218
@pytest.mark.parametrize("prec", PRECISIONS)
def test_point_triangle_distance(oracle, prec):
    O = mod_of(oracle, prec)
    d, n, wp, wq = O.narrow_phase_point_triangle([0.25, 0.25, 0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0])
    assert 0.49 < d < 0.51
    assert n[2] > 0.9


# tests/test_basic.cpp:70-81: 500 + 0.1 / 0.1^2 = 510
@pytest.mark.parametrize("prec", PRECISIONS)
def test_pin_stiffness(oracle, prec):
    O = mod_of(oracle, prec)
    k = O.pin_stiffness(0.1, 0.01, [0.1, 0.0, 0.0], np.eye(3) * 500.0, 1e-6)
    assert abs(k - 510.0) < 1.0


# tests/test_basic.cpp:221-271 (signs of the pin and wall barrier gradients)
@pytest.mark.parametrize("prec", PRECISIONS)
def test_pin_and_wall_gradient_signs(oracle, prec):
    O = mod_of(oracle, prec)
    assert O.barrier_gradient(1.0, 2.0, 1000.0) < 0.0      # pin at gap 1, g_max 2 -> -x direction
    assert O.barrier_gradient(0.5, 1.0, 1000.0) < 0.0      # wall at gap 0.5, g_max 1 -> pushes +z


# tests/test_basic.cpp:274-314: wall line search reduces alpha to (0, 1); halving gives 0.5
@pytest.mark.parametrize("prec", PRECISIONS)
def test_wall_line_search(oracle, prec):
    O = mod_of(oracle, prec)
    x = np.array([[0, 0, 0.1], [1, 0, 0.1], [0.5, 1, 0.1]], dtype=np.float64)
    d = np.zeros(9)
    d[2] = -0.15
    a = O.line_search(x, d, [], [], [0, 0, 1], 0.0, 1.0)
    assert 0.0 < a < 1.0
    assert a == 0.5


# tests/test_basic.cpp:316-375: contact line search must reduce alpha
@pytest.mark.parametrize("prec", PRECISIONS)
def test_contact_line_search(oracle, prec):
    O = mod_of(oracle, prec)
    x = np.array([[0.5, 0.5, 0.5], [0, 0, 0], [1, 0, 0], [0.5, 1, 0]], dtype=np.float64)
    d = np.zeros(12)
    d[2] = -1.0
    c = O.Contact()
    c.type = O.POINT_TRIANGLE
    c.idx0, c.idx1, c.idx2, c.idx3 = 0, 1, 2, 3
    c.gap = 0.5
    c.normal = [0, 0, 1]
    a = O.line_search(x, d, [c], [], [0, 0, 0], 0.0, 1.0)
    assert a < 1.0
    # alpha = 1 is rejected (sample t = 0.5 touches the triangle); at alpha = 0.5
    # only the last sample t = 1 touches, and ccd_point_triangle then returns
    # t = 1.0, which `toi < 1.0` (line_search.cpp:192) reads as no collision.
    assert a == 0.5


# tests/test_basic.cpp:377-419: PCG on a 9x9 SPD system
@pytest.mark.parametrize("prec", PRECISIONS)
def test_pcg_9x9(oracle, prec):
    O = mod_of(oracle, prec)
    rows = list(range(9)) + [0, 1, 3, 4]
    cols = list(range(9)) + [1, 0, 4, 3]
    vals = [2.0] * 9 + [0.5, 0.5, 0.3, 0.3]
    x, conv, iters, rel = O.pcg_solve(9, rows, cols, vals, np.ones(9), 1e-6, 100)
    assert conv
    A = np.zeros((9, 9))
    for r, c_, v in zip(rows, cols, vals):
        A[r, c_] += v
    assert np.linalg.norm(np.ones(9) - A @ x) < 1e-3


# tests/test_basic.cpp:164-191: the BVH is non-empty; with >= 2 triangles its
# leaves carry no primitive (collision.cpp:81-86), so no self-contact candidate exists
@pytest.mark.parametrize("prec", PRECISIONS)
def test_bvh_literal_leaf_defect(oracle, prec):
    O = mod_of(oracle, prec)
    m = O.Mesh()
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=np.float64)
    m.initialize(v, np.array([[0, 1, 2], [0, 2, 3]]), O.Material())
    assert O.bvh_node_count(m, v) > 0
    # a vertex hovering over the quad: the intended query finds it, the literal one does not
    v2 = np.vstack([v, [[0.5, 0.5, 5e-5]]])
    m2 = O.Mesh()
    m2.initialize(v2, np.array([[0, 1, 2], [0, 2, 3]]), O.Material())
    vt_lit, ee_lit = O.broad_phase(m2, v2, "literal")
    vt_int, ee_int = O.broad_phase(m2, v2, "intended")
    assert vt_lit == [] and ee_lit == []
    assert (4, 0) in vt_int and (4, 1) in vt_int


# tests/test_hybrid.cpp:12-70: one step against a rigid plate. The cloth starts
# 20 mm above the plate and ends ~15 mm above it, outside the 10 mm detection
# threshold of rigid contacts (collision.cpp:571), so no contact is made and the
# test's first assert (rigid body gains velocity, :61-62) fails against the
# reference itself; the second (cloth v_z > -0.5, :64-66) holds. (Started
# closer, the barrier throws the cloth past 10 mm within the step, so the
# end-of-step coupling pass still finds no contact.)
@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("height,couples", [(0.02, False), (0.0005, False)])
def test_hybrid_rigid_response(oracle, prec, height, couples):
    O = mod_of(oracle, prec)
    m = O.Mesh()
    verts = np.array([[0.0, 0.0, height], [0.01, 0.0, height], [0.0, 0.01, height]])
    mat = O.Material(youngs_modulus=1e5, thickness=0.001)
    m.initialize(verts, np.array([[0, 1, 2]]), mat)
    s = O.State()
    s.initialize(m)
    vel = np.zeros((3, 3))
    vel[0] = [0, 0, -0.5]
    s.set_velocities(vel)
    body = O.RigidBody()
    body.initialize(np.array([[-0.05, -0.05, 0.0], [0.05, -0.05, 0.0], [-0.05, 0.05, 0.0]]), np.array([[0, 1, 2]]), 1000.0)
    p = O.SimParams()
    p.dt = 0.01
    p.contact_gap_max = 0.05
    p.beta_max = 0.25
    p.pcg_tol = 1e-4
    p.max_newton_steps = 5
    O.Integrator.step(m, s, O.Constraints(), p, [body])
    assert (np.linalg.norm(body.linear_velocity) > 1e-6) == couples
    assert s.get_velocities()[0, 2] > -0.5


# tests/test_basic.cpp:19-68,83-129 expect a non-zero contact stiffness from a
# ContactPair whose weights were never set; the reference itself returns 0 there
# (stiffness.cpp:96-104 skips zero weights), so those asserts fail against it.
@pytest.mark.parametrize("prec", PRECISIONS)
def test_stale_contact_stiffness_expectation_is_zero(oracle, prec):
    O = mod_of(oracle, prec)
    c = O.Contact()
    c.type = O.POINT_TRIANGLE
    c.idx0, c.idx1, c.idx2, c.idx3 = 0, 1, 2, 3
    c.normal = [0, 0, 1]
    c.gap = 0.001
    rows = [3 * v + j for v in range(4) for j in range(3)]
    vals = [d for d in (900.0, 100.0, 200.0, 300.0) for _ in range(3)]
    k = O.contact_stiffness(c, [0.1, 0.2, 0.3, 0.4], 0.01, 12, rows, rows, vals)
    assert k == 0.0
    # with the weights detection assigns (collision.cpp:505-511) it is m w^2/dt^2 + Wn^T H Wn
    c.weights = [1.0, -1 / 3, -1 / 3, -1 / 3]
    c.vertex_count = 4
    k = O.contact_stiffness(c, [0.1, 0.2, 0.3, 0.4], 0.01, 12, rows, rows, vals)
    w = np.array([1.0, -1 / 3, -1 / 3, -1 / 3])
    expect = (np.array([0.1, 0.2, 0.3, 0.4]) * w * w).sum() / 1e-4 + (w * w * np.array([900, 100, 200, 300.0])).sum()
    assert k == pytest.approx(expect, rel=1e-5)


# Elasticity::face_hessian (elasticity.cpp:135-181) blocks are c*diag(1,1,0) and
# enforce_spd clamps them to diag(max(c,1e-8), max(c,1e-8), 1e-8) exactly.
@pytest.mark.parametrize("prec", PRECISIONS)
def test_enforce_spd_of_face_blocks(oracle, prec):
    O = mod_of(oracle, prec)
    for c in (3.5, -2.0, 0.0, 1e-9):
        S = O.enforce_spd(np.diag([c, c, 0.0]))
        e = max(c, 1e-8)
        np.testing.assert_array_equal(S, np.diag([e, e, 1e-8]).astype(S.dtype))
    A = np.array([[2.0, 0.5, 0.0], [0.5, -1.0, 0.2], [0.0, 0.2, 0.5]])
    S = O.enforce_spd(A)
    w, Q = np.linalg.eigh(A)
    ref = Q @ np.diag(np.maximum(w, 1e-8)) @ Q.T
    np.testing.assert_allclose(S, ref, rtol=1e-5, atol=1e-6)
