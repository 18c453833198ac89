"""Checkpoint / resume and the solver-dump format on the GPU.

* A run pickled at frame 5 (Mesh, State, Constraints) and restored into
  fresh objects continues with the same bits as the run that never stopped,
  in both semantics.
* A CORRECTED step's Newton system written with andosim_b200.dump reads back
  unchanged, and its solution solves it.
* The device's system at the state of tests/golden/sheets_bending.npz (the
  FP64 oracle's, written by tests/golden/make_systems.py) matches the fixture
  within the parity tolerance: same pattern, same blocks inside and outside
  it, same gradient.
"""
from __future__ import annotations

import pickle
import sys
from pathlib import Path

import numpy as np
import pytest

from andosim_b200 import dump, scenes
from test_gpu_corrected import two_sheets

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def frames(core, sc, m, st, p, first, count):
    for f in range(first, first + count):
        c = core.Constraints()
        for i, t in sc.pins_at(f):
            c.add_pin(int(i), t)
        for n, o, g in sc.walls:
            c.add_wall(n, o, g)
        st.apply_gravity(sc.gravity, p.dt)
        core.Integrator.step(m, st, c, p)


@pytest.mark.parametrize("semantics", ["reference", "corrected"])
def test_resume_continues_the_run_bit_for_bit(core, semantics):
    sc = scenes.c1(n=16)
    m = core.Mesh()
    m.initialize(sc.vertices, sc.triangles, core.Material(**sc.material))
    st = core.State()
    st.initialize(m)
    p = core.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)
    p.semantics = semantics
    frames(core, sc, m, st, p, 0, 5)
    blob = pickle.dumps((m, st))
    frames(core, sc, m, st, p, 5, 4)
    m2, st2 = pickle.loads(blob)
    frames(core, sc, m2, st2, p, 5, 4)
    np.testing.assert_array_equal(st2.get_positions64(), st.get_positions64())
    np.testing.assert_array_equal(st2.get_velocities64(), st.get_velocities64())
    assert np.abs(st.get_positions64() - sc.vertices).max() > 1e-3      # the run moved


def test_dump_round_trip_and_solution(abi, tmp_path):
    sc = two_sheets(n=10, gap=0.0006)
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.keep_system()
    S.upload(sc.vertices, np.zeros_like(sc.vertices), sc.vertices, None)
    p = abi.make_params(dict(sc.params, pcg_tol=1e-6), semantics="corrected")
    S.apply_gravity(sc.gravity, p.dt)
    S.step(p, sc.pins_at(0), sc.walls)
    live = dump.system_arrays(S)
    path = dump.save_system(dump.frame_path(tmp_path, "two_sheets", 0, 0), S, workload="two_sheets", frame=0)
    S.close()
    back = dump.load_system(path)
    assert back["meta"] == {"workload": "two_sheets", "frame": 0}
    for k in dump.KEYS:
        np.testing.assert_array_equal(back[k], live[k], err_msg=k)
    assert len(back["extra_rows"]) > 0
    A = dump.dense(back)
    b = back["rhs"].astype(np.float64)
    x = back["solution"].astype(np.float64)
    assert np.abs(A @ x - b).max() <= 1e-3 * np.abs(b).max()


def test_device_system_matches_the_oracle_fixture(abi):
    sys.path.insert(0, str(GOLDEN))
    import make_systems

    fx = dump.load_system(GOLDEN / "sheets_bending.npz")
    st = np.load(GOLDEN / "sheets_bending_state.npz")
    sc, _, _ = make_systems.sheets_bending()
    x, v = st["x"], st["v"]
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.keep_system()
    S.upload(x, v, sc.vertices, None)
    S.eval_system(abi.make_params(sc.params, semantics="corrected"), sc.pins_at(0), sc.walls)
    got = dump.system_arrays(S)
    S.close()
    np.testing.assert_array_equal(got["rowptr"], fx["rowptr"])
    np.testing.assert_array_equal(got["cols"], fx["cols"])
    g_o = fx["gradient"]
    assert np.abs(got["gradient"] - g_o).max() <= 1e-5 * np.abs(g_o).max()
    H_g, H_o = dump.dense(got), dump.dense(fx)
    hs = np.abs(H_o).max()
    err = np.abs(H_g - H_o)
    assert (err <= 1e-5 * np.abs(H_o) + 1e-7 * hs).all(), float((err / (np.abs(H_o) + 1e-7 * hs)).max())
