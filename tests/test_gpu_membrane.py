"""The projected exact membrane Hessian on the GPU (CORRECTED,
membrane_hessian = projected) against the FP64 oracle.

The oracle's form is pinned on the CPU (tests/test_oracle_membrane.py: the
exact Jacobian where no eigenvalue is clamped, positive semidefinite
everywhere, a clamped strip that swings). Here the device's Newton system
matches the oracle's at stretched, compressed and pinned states, and a
clamped strip's 8-frame free run stays within 1e-4 of the extent of the FP64
oracle run while it swings down.
"""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes
from test_gpu_corrected import corrected_parity

pytestmark = pytest.mark.gpu

PROJECTED = dict(membrane_hessian=1)


@pytest.mark.parametrize("squeeze", [1.08, 0.93])
def test_projected_system_matches_oracle(oracle, abi, squeeze):
    sc = scenes.c1(n=16)
    rng = np.random.default_rng(5)
    x = sc.vertices.copy()
    x[:, :2] *= squeeze
    x[:, 2] += rng.normal(scale=3e-3, size=len(x))
    v = rng.normal(scale=0.2, size=x.shape)
    corrected_parity(oracle, abi, sc, x, v, params=dict(PROJECTED, enable_strain_limiting=False))


def test_projected_system_with_strain_and_contact(oracle, abi):
    from test_gpu_corrected import two_sheets

    sc = two_sheets()
    res = corrected_parity(oracle, abi, sc, sc.vertices.copy(), np.zeros_like(sc.vertices), params=PROJECTED, expect_contacts=True)
    assert {int(c.type) for c in res["contacts"]} >= {0, 1}


def strip():
    n = 12
    v = scenes.grid_plane(n, 0.2)
    v[:, 2] = 0.5
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3)
    pins = [(i, v[i].copy()) for i in range(2 * n)]       # the two rows along y = 0 clamped
    return scenes.Scene("strip", v, scenes.grid_triangles(n, n), mat, scenes.cloth_params(pcg_tol=1e-5), pins, [scenes.ground()])


def test_projected_free_run_matches_fp64(oracle, abi):
    sc = strip()
    frames = 8
    O = oracle.f64
    om = O.Mesh()
    om.initialize(sc.vertices, sc.triangles, O.Material(**sc.material))
    os_ = O.State()
    os_.initialize(om)
    op = O.SimParams()
    p = abi.make_params(dict(sc.params, **PROJECTED), semantics="corrected")
    for k in ("dt", "beta_max", "max_newton_steps", "pcg_tol", "pcg_max_iters", "contact_gap_max", "wall_gap",
              "enable_strain_limiting", "strain_limit", "strain_tau"):
        setattr(op, k, getattr(p, k))
    op.membrane_hessian = 1
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    worst = 0.0
    for f in range(frames):
        c = O.Constraints()
        for i, t in sc.pins:
            c.add_pin(int(i), t)
        for n, o, g in sc.walls:
            c.add_wall(n, o, g)
        os_.apply_gravity(sc.gravity, op.dt)
        O.Integrator.step(om, os_, c, op, None, "indexed", "literal", "corrected")
        S.apply_gravity(sc.gravity, p.dt)
        st = S.step(p, sc.pins, sc.walls)
        assert st["line_search_fail"] == 0, f
        x, _ = S.download()
        worst = max(worst, float(np.abs(x - np.asarray(os_.get_positions(), dtype=np.float64)).max()) / ext)
    S.close()
    assert worst <= 1e-4, worst
    assert 0.5 - float(x[:, 2].min()) > 0.04                # the strip swung down (the fixed-rotation form: 1 cm in 12 frames)
