"""Checkpoints of a simulation run as ``.npz`` files.

A checkpoint holds what restarting a run at frame k needs, as plain arrays
(no pickled Python objects, so any numpy reader can open it):

* the mesh: current vertices (FP64), triangles, its rest state as computed at
  initialisation (edges, inverse rest shapes, rest areas) and the material;
* the state: positions, velocities, previous positions, the start of the next
  CORRECTED step (FP64) and the masses;
* the constraints: pins (vertex, target, active) and walls (normal, offset,
  gap, active);
* ``frame`` and a JSON ``meta`` string.

The arrays are the ones the module's objects pickle to (``__getstate__``),
so ``load`` rebuilds objects that continue the saved run with the same bits
(the device state is uploaded on the restored state's first step).
"""
from __future__ import annotations

import json
from pathlib import Path
from typing import Optional, Tuple

import numpy as np

FORMAT = 1


def save(path, mesh, state, constraints, frame: int = 0, **meta) -> Path:
    """Write mesh, state and constraints (module objects) to `path` (``.npz``)."""
    mv, tris, edges, dm_inv, areas, material = mesh.__getstate__()
    x, v, xp, start, masses = state.__getstate__()
    pins, walls = constraints.__getstate__()
    pa = np.asarray([(p[0], p[1], p[2], p[3], float(p[4])) for p in pins], dtype=np.float64).reshape(-1, 5)
    wa = np.asarray([(w[0], w[1], w[2], w[3], w[4], float(w[5])) for w in walls], dtype=np.float64).reshape(-1, 6)
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(p, format=np.int64(FORMAT), frame=np.int64(frame), meta=np.array(json.dumps(meta)),
                        mesh_vertices=mv, mesh_triangles=tris, mesh_edges=edges, mesh_dm_inv=dm_inv, mesh_areas=areas,
                        material=np.asarray(material, dtype=np.float64),
                        positions=x, velocities=v, positions_prev=xp, step_start=start, masses=masses,
                        pins=pa, walls=wa)
    return p


def load(path, core=None) -> Tuple[object, object, object, int, dict]:
    """(mesh, state, constraints, frame, meta) from a checkpoint written by `save`."""
    if core is None:
        from . import ando_barrier_core as core
    with np.load(Path(path), allow_pickle=False) as z:
        if int(z["format"]) != FORMAT:
            raise ValueError(f"{path}: checkpoint format {int(z['format'])}, expected {FORMAT}")
        mesh = core.Mesh.__new__(core.Mesh)
        mesh.__setstate__((z["mesh_vertices"], z["mesh_triangles"], z["mesh_edges"], z["mesh_dm_inv"], z["mesh_areas"],
                           tuple(float(q) for q in z["material"])))
        state = core.State.__new__(core.State)
        state.__setstate__((z["positions"], z["velocities"], z["positions_prev"], z["step_start"], z["masses"]))
        pins = [(int(r[0]), float(r[1]), float(r[2]), float(r[3]), bool(r[4])) for r in z["pins"]]
        walls = [(float(r[0]), float(r[1]), float(r[2]), float(r[3]), float(r[4]), bool(r[5])) for r in z["walls"]]
        constraints = core.Constraints.__new__(core.Constraints)
        constraints.__setstate__((pins, walls))
        frame = int(z["frame"])
        meta = json.loads(str(z["meta"]))
    if state.get_positions64().shape[0] != mesh.num_vertices():
        raise ValueError(f"{path}: state and mesh have different vertex counts")
    return mesh, state, constraints, frame, meta


def restart_frame(path) -> Optional[int]:
    """The frame a checkpoint was written at, without building the objects."""
    with np.load(Path(path), allow_pickle=False) as z:
        return int(z["frame"])
