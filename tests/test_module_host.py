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
