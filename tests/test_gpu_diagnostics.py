"""Device-side diagnostics against host computations of the same quantities.

* ando_edge_triangle_crossings: the exact FP64 segment-triangle test over an
  LBVH of the triangles gives the oracle's grid-based count, pair for pair in
  number, on meshes that do and do not intersect themselves.
* ando_collision_metrics: CollisionValidator's counts, gap extremes and
  relative normal velocities (collision_validator.cpp:7-221) over the contact
  list still on the device, against the same formulas in numpy over the
  downloaded contacts and velocities.
* ando_state_moments: EnergyTracker's kinetic energy, momenta and largest
  speed (energy_tracker.cpp:7-42) against numpy over the downloaded state.
* The module routes CollisionValidator / EnergyTracker / AdaptiveTimestep
  through these reductions when the device holds the state, and gives the
  host formulas' answers.
"""
from __future__ import annotations

import numpy as np
import pytest

from andosim_b200 import scenes

pytestmark = pytest.mark.gpu


def two_sheets(n=24, spacing=5e-4, noise=0.0, seed=0):
    """Two n x n sheets over [0, 1]^2, the upper one `spacing` above the lower,
    each vertex lifted by uniform noise of amplitude `noise`."""
    rng = np.random.default_rng(seed)
    va, vb = scenes.grid_plane(n, 1.0), scenes.grid_plane(n, 1.0)
    va[:, 2] = 0.5 + noise * rng.uniform(-1, 1, len(va))
    vb[:, 2] = 0.5 + spacing + noise * rng.uniform(-1, 1, len(vb))
    v = np.vstack([va, vb])
    t = np.vstack([scenes.grid_triangles(n, n), scenes.grid_triangles(n, n, offset=n * n)]).astype(np.int32)
    return v, t


def oracle_crossings(oracle, v, t, x):
    O = oracle.f64
    om = O.Mesh()
    om.initialize(v, t, O.Material())
    e = np.linalg.norm(v[t[:, 1]] - v[t[:, 0]], axis=1).mean()
    return O.edge_triangle_crossings(om, x, 2.0 * e)


@pytest.mark.parametrize("case", ["flat", "tilted", "noisy", "noisy_dense"])
def test_edge_triangle_crossings_match_oracle(oracle, abi, case):
    if case == "flat":            # two parallel sheets 0.5 mm apart: none
        v, t = two_sheets()
    elif case == "tilted":        # a sheet tilted through the other along x = 0.5
        v, t = two_sheets(n=30)
        half = len(v) // 2
        v[half:, 2] = 0.5 + (v[half:, 0] - 0.5) * 0.2
    elif case == "noisy":         # crumpled sheets through each other
        v, t = two_sheets(n=32, spacing=2e-3, noise=4e-3, seed=3)
    else:                         # two crumpled sheets on one grid: crossings almost everywhere
        v, t = two_sheets(n=48, spacing=0.0, noise=2e-2, seed=5)
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=0.0)
    S = abi.Scene(v, t, mat)
    S.upload(v, np.zeros_like(v), v, None)
    got = S.edge_triangle_crossings()
    again = S.edge_triangle_crossings()
    S.close()
    want = oracle_crossings(oracle, v, t, v)
    assert got == want == again, (got, want, again)
    if case == "flat":
        assert want == 0
    else:
        assert want > 0


def contact_scene(abi, seed=1):
    v, t = two_sheets(n=24, spacing=5e-4, noise=1e-4, seed=seed)
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=0.0)
    S = abi.Scene(v, t, mat)
    rng = np.random.default_rng(seed)
    vel = rng.normal(scale=0.3, size=v.shape)
    masses = rng.uniform(1e-5, 3e-5, len(v))
    S.upload(v, vel, v, masses)
    return S, v, vel, masses


def numpy_metrics(contacts, vel, gap_max, ccd):
    g = np.array([np.float32(c.gap) for c in contacts], dtype=np.float64)
    types = np.array([c.type for c in contacts])
    pen = -g[g < 0]
    rv = []
    for c in contacts:
        n = np.array(c.normal[:])
        if c.type == 0:
            rel = vel[c.idx0] - (vel[c.idx1] + vel[c.idx2] + vel[c.idx3]) * (1.0 / 3.0)
        elif c.type == 1:
            rel = (vel[c.idx0] + vel[c.idx1]) * 0.5 - (vel[c.idx2] + vel[c.idx3]) * 0.5
        elif c.type == 2:
            rel = vel[c.idx0]
        else:
            continue
        rv.append(float(np.float32(abs(rel @ n))))
    gm = float(np.float32(gap_max))
    return dict(num_total_contacts=len(g), num_point_triangle=int((types == 0).sum()), num_edge_edge=int((types == 1).sum()),
                num_wall=int((types == 2).sum()), num_penetrations=len(pen), num_major_penetrations=int((pen > 0.001).sum()),
                num_tunneling=int((pen > 0.1 * gm).sum()), num_ccd_contacts=int(ccd) * int((g < gm * 0.5).sum()),
                num_relative_velocities=len(rv), min_gap=g.min(), max_gap=g.max(), sum_gap=g.sum(),
                max_penetration=pen.max() if len(pen) else 0.0, sum_penetration=pen.sum(),
                max_relative_velocity=max(rv), sum_relative_velocity=sum(rv))


@pytest.mark.parametrize("ccd", [True, False])
def test_collision_metrics_match_host(abi, ccd):
    S, v, vel, masses = contact_scene(abi)
    gap_max = 1e-3
    contacts = S.contacts(semantics="corrected", gap_max=gap_max)
    assert len(contacts) > 100
    assert {c.type for c in contacts} >= {0, 1}
    got = S.collision_metrics(gap_max, ccd)
    S.close()
    want = numpy_metrics(contacts, vel, gap_max, ccd)
    for k, w in want.items():
        if k.startswith("num_") or k in ("min_gap", "max_gap", "max_penetration", "max_relative_velocity"):
            assert got[k] == w, (k, got[k], w)                 # counts and extremes exactly
        else:
            assert abs(got[k] - w) <= 1e-12 * max(1.0, abs(w)) * len(contacts), (k, got[k], w)


def test_collision_metrics_empty_list(abi):
    v, t = two_sheets(n=8, spacing=0.1)
    S = abi.Scene(v, t, dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=0.0))
    S.upload(v, np.zeros_like(v), v, None)
    assert S.contacts(semantics="corrected", gap_max=1e-3) == []
    got = S.collision_metrics(1e-3, True)
    S.close()
    assert all(val == 0 for val in got.values())


def test_state_moments_match_host(abi):
    S, v, vel, masses = contact_scene(abi, seed=2)
    got = S.moments()
    S.close()
    p = masses[:, None] * vel
    assert abs(got["kinetic_energy"] - 0.5 * (masses * (vel ** 2).sum(1)).sum()) <= 1e-12 * got["kinetic_energy"] * len(v)
    np.testing.assert_allclose(got["linear_momentum"], p.sum(0), rtol=0, atol=1e-15 * np.abs(p).sum())
    L = np.cross(v, p)
    np.testing.assert_allclose(got["angular_momentum"], L.sum(0), rtol=0, atol=1e-15 * np.abs(L).sum())
    assert got["max_speed"] == np.sqrt((vel ** 2).sum(1).max())


def test_module_validator_and_tracker_use_device_state(core):
    """After CORRECTED steps of two sheets in contact, the module's validator,
    energy tracker and adaptive time step (device reductions) agree with the
    same calls on a host-side copy of the contact list and velocities."""
    v, t = two_sheets(n=20, spacing=8e-4, noise=1e-4, seed=4)
    m = core.Mesh()
    m.initialize(v, t, core.Material(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3))
    st = core.State()
    st.initialize(m)
    p = core.SimParams()
    p.semantics = "corrected"
    p.dt = 1.0 / 60.0
    c = core.Constraints()
    c.add_wall(np.array([0.0, 0.0, 1.0]), 0.0, 1e-3)
    for _ in range(3):
        st.apply_gravity(np.array([0.0, 0.0, -9.81]), p.dt)
        core.Integrator.step(m, st, c, p)
    gap = float(p.contact_gap_max)
    contacts = core.Integrator.compute_contacts(m, st, None, "corrected", gap)
    assert len(contacts) > 0
    dev = core.CollisionValidator.compute_metrics(m, st, contacts, gap, True)
    host = core.CollisionValidator.compute_metrics(m, st, list(reversed(contacts)), gap, True)   # another list: host path
    for k in ("num_point_triangle", "num_edge_edge", "num_wall", "num_total_contacts", "num_penetrations",
              "num_ccd_contacts", "num_broad_phase_contacts", "has_tunneling", "has_major_penetration", "is_stable"):
        assert getattr(dev, k) == getattr(host, k), k
    for k in ("min_gap", "max_gap", "max_penetration", "max_relative_velocity"):
        assert getattr(dev, k) == getattr(host, k), k
    for k in ("avg_gap", "avg_penetration", "avg_relative_velocity", "ccd_effectiveness"):
        assert abs(getattr(dev, k) - getattr(host, k)) <= 1e-5 * max(abs(getattr(host, k)), 1e-12), k
    assert core.CollisionValidator.edge_triangle_crossings(m, st) == 0
    ke_dev = core.EnergyTracker.compute_kinetic_energy(st)
    vmax_dev = core.AdaptiveTimestep.compute_max_velocity(st)
    dt_dev = core.AdaptiveTimestep.compute_next_dt(st, m, p.dt, 1e-4, 1.0 / 30.0, 0.5)
    vel = st.get_velocities64() if hasattr(st, "get_velocities64") else np.asarray(st.get_velocities(), dtype=np.float64)
    masses = np.asarray(st.get_masses(), dtype=np.float64)
    assert abs(ke_dev - 0.5 * (masses * (vel ** 2).sum(1)).sum()) <= 1e-5 * ke_dev
    flat = np.asarray(st.get_velocities(), dtype=np.float32).ravel()
    assert abs(vmax_dev - core.AdaptiveTimestep.compute_max_velocity(flat)) <= 1e-6 * vmax_dev
    assert abs(dt_dev - core.AdaptiveTimestep.compute_next_dt(flat, m, p.dt, 1e-4, 1.0 / 30.0, 0.5)) <= 1e-6 * dt_dev
