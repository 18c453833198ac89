"""Generate the solver-dump regression fixtures from the FP64 oracle.

    python tests/golden/make_systems.py

Each fixture is one Newton system in the dump format of andosim_b200.dump
(BSR over the static pattern plus the contact blocks outside it, right-hand
side -g, FP64 gradient), evaluated by the oracle's CORRECTED stages at a
seeded state:

* sheets_bending.npz: two 6 x 6 sheets 0.6 mm apart over the ground, bending
  stiffness 1e-3, velocities seeded: point-triangle and edge-edge contacts
  (blocks outside the pattern), hinge pairs of the bending term, the wall.

The oracle is test infrastructure; this script runs it on the CPU and writes
the fixtures that tests/test_dump_fixtures.py (CPU, against the oracle) and
tests/test_gpu_checkpoint.py (GPU, against the device's system) read.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from andosim_b200 import dump, scenes  # noqa: E402


def sheets_bending():
    n, gap, h = 6, 0.0006, 0.5 / 5
    a = scenes.grid_plane(n, 0.5)
    b = scenes.grid_plane(n, 0.5)
    b[:, 0] += 0.37 * h
    b[:, 1] += 0.21 * h
    a[:, 2] = 0.3
    b[:, 2] = 0.3 + gap
    v = np.concatenate([a, b])
    t = np.concatenate([scenes.grid_triangles(n, n), scenes.grid_triangles(n, n, offset=n * n)]).astype(np.int32)
    mat = dict(youngs_modulus=1e5, poisson_ratio=0.3, density=200.0, thickness=1e-3, bending_stiffness=1e-3)
    sc = scenes.Scene("sheets_bending", v, t, mat, scenes.cloth_params(), [], [scenes.ground()])
    rng = np.random.default_rng(11)
    x = v + rng.normal(scale=5e-5, size=v.shape)
    vel = rng.normal(scale=0.05, size=v.shape)
    return sc, x, vel


def static_pattern(V, tris, hinges):
    """Self blocks, face pairs and the two vertices opposite each interior edge (the device's pattern)."""
    adj = [{i} for i in range(V)]
    for f in tris:
        for a in f:
            adj[a].update(int(q) for q in f)
    for h in hinges:
        adj[h[2]].add(int(h[3]))
        adj[h[3]].add(int(h[2]))
    rowptr = np.zeros(V + 1, np.int32)
    cols = []
    for i in range(V):
        r = sorted(adj[i])
        cols += r
        rowptr[i + 1] = len(cols)
    return rowptr, np.asarray(cols, np.int32)


def oracle_system(O, sc, x, vel):
    from conftest import oracle_constraints, oracle_scene

    m, s, p = oracle_scene(O, sc)
    s.set_positions(x)
    s.set_velocities(vel)
    res = O.Integrator.corrected_system(m, s, x + p.dt * vel, np.zeros(len(x), np.int8), oracle_constraints(O, sc), p)
    hinges = O.bending_hinges(m)[0]
    V = len(x)
    rowptr, cols = static_pattern(V, sc.triangles, hinges)
    hs = res["hessian"]
    blocks = {}
    for r in range(hs["n"]):
        for k in range(hs["rowptr"][r], hs["rowptr"][r + 1]):
            c = hs["cols"][k]
            blk = blocks.setdefault((r // 3, c // 3), np.zeros((3, 3)))
            blk[r % 3, c % 3] += hs["vals"][k]
    vals = np.zeros((len(cols), 3, 3))
    for i in range(V):
        for k in range(rowptr[i], rowptr[i + 1]):
            vals[k] = blocks.pop((i, int(cols[k])), np.zeros((3, 3)))
    extra = sorted(blocks)
    g = np.asarray(res["gradient"], np.float64)
    return dict(rowptr=rowptr, cols=cols, vals=vals.astype(np.float32),
                extra_rows=np.asarray([r for r, _ in extra], np.int32), extra_cols=np.asarray([c for _, c in extra], np.int32),
                extra_vals=np.asarray([blocks[k] for k in extra], np.float32).reshape(-1, 3, 3),
                rhs=(-g).astype(np.float32), solution=np.zeros(3 * V, np.float32), gradient=g)


def main():
    from oracle.build import load

    O = load().f64
    sc, x, vel = sheets_bending()
    arrays = oracle_system(O, sc, x, vel)
    np.savez_compressed(HERE / "sheets_bending_state.npz", x=x, v=vel)
    out = dump.save_arrays(HERE / "sheets_bending.npz", arrays, workload=sc.name, semantics="corrected", source="FP64 oracle",
                           state="sheets_bending_state.npz")
    print(out, len(arrays["cols"]), "pattern blocks,", len(arrays["extra_rows"]), "extra blocks")


if __name__ == "__main__":
    main()
