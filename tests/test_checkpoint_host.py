"""Checkpoint / resume of the module's objects without a GPU.

The reference saves no solver state (its add-on bakes shape keys and its demos
export OBJ frames). Here Mesh, State and Constraints pickle: a run can be
stopped at frame k and restarted from the file. On the host side that means
every field comes back bit for bit; the GPU test (test_gpu_checkpoint.py)
checks that the restored objects continue the run with the same bits.
"""
from __future__ import annotations

import pickle

import numpy as np

from andosim_b200 import scenes


def test_mesh_state_constraints_round_trip(core):
    sc = scenes.c1(n=9)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material, bending_stiffness=2e-3))
    st = core.State()
    st.initialize(m)
    rng = np.random.default_rng(0)
    st.set_positions64(sc.vertices + rng.normal(scale=1e-3, size=sc.vertices.shape))
    st.set_velocities64(rng.normal(size=sc.vertices.shape))
    c = core.Constraints()
    for i, t in sc.pins:
        c.add_pin(int(i), t)
    c.add_wall(np.array([0.0, 0.3, 1.0]), 0.01, 1e-3)
    m2, st2, c2 = pickle.loads(pickle.dumps((m, st, c)))
    assert np.array_equal(m2.get_vertices(), m.get_vertices())
    assert m2.num_triangles() == m.num_triangles()
    np.testing.assert_array_equal(st2.get_positions64(), st.get_positions64())
    np.testing.assert_array_equal(st2.get_velocities64(), st.get_velocities64())
    np.testing.assert_array_equal(st2.get_masses(), st.get_masses())
    assert c2.num_active_pins() == c.num_active_pins() == len(sc.pins)
    assert sorted(c2._pins) == sorted(c._pins)
    for k in c._pins:
        np.testing.assert_array_equal(c2._pins[k], c._pins[k])
    assert len(c2._walls) == 1
    np.testing.assert_array_equal(c2._walls[0][0], c._walls[0][0])
    assert c2._walls[0][1:] == c._walls[0][1:]


def test_corrupt_state_pickle_is_rejected(core):
    import pytest

    sc = scenes.c1(n=5)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    st = core.State()
    st.initialize(m)
    state = st.__getstate__()
    bad = (state[0], state[1][:-1], state[2], state[3], state[4])     # one velocity row missing
    s2 = core.State.__new__(core.State)
    with pytest.raises(RuntimeError, match="inconsistent"):
        s2.__setstate__(bad)


def test_npz_checkpoint_round_trip(core, tmp_path):
    """andosim_b200.checkpoint writes the pickled arrays as a plain .npz and
    rebuilds objects equal field for field."""
    from andosim_b200 import checkpoint

    sc = scenes.c1(n=7)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material, bending_stiffness=1e-3))
    st = core.State()
    st.initialize(m)
    rng = np.random.default_rng(2)
    st.set_positions64(sc.vertices + rng.normal(scale=1e-3, size=sc.vertices.shape))
    st.set_velocities64(rng.normal(size=sc.vertices.shape))
    c = core.Constraints()
    for i, t in sc.pins:
        c.add_pin(int(i), t)
    c.add_wall(np.array([0.0, 0.0, 1.0]), 0.0, 1e-3)
    path = checkpoint.save(tmp_path / "run.npz", m, st, c, frame=42, workload="c1")
    assert checkpoint.restart_frame(path) == 42
    m2, st2, c2, frame, meta = checkpoint.load(path, core)
    assert frame == 42 and meta == {"workload": "c1"}
    with np.load(path, allow_pickle=False) as z:           # plain arrays, no pickled objects
        assert z["positions"].dtype == np.float64 and z["pins"].shape == (len(sc.pins), 5)
    np.testing.assert_array_equal(m2.get_vertices(), m.get_vertices())
    np.testing.assert_array_equal(st2.get_positions64(), st.get_positions64())
    np.testing.assert_array_equal(st2.get_velocities64(), st.get_velocities64())
    np.testing.assert_array_equal(st2.get_masses(), st.get_masses())
    assert sorted(c2._pins) == sorted(c._pins) and len(c2._walls) == 1
    assert m2.__getstate__()[5] == m.__getstate__()[5]      # material, bending stiffness included
