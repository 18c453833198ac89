"""Newton systems as ``.npz`` files: the solver-dump format.

One file holds one Newton system of a step as the device assembled it:

* ``rowptr`` (V+1, int32), ``cols`` (nnzb, int32, sorted per row) and
  ``vals`` (nnzb, 3, 3, float32, row-major blocks): the static BSR pattern
  (self blocks, face pairs and, with bending, the vertices opposite each
  interior edge) with the system's values;
* ``extra_rows``, ``extra_cols`` (int32) and ``extra_vals`` (n, 3, 3,
  float32): contact blocks between vertices outside that pattern (their sum
  with ``vals`` is the whole matrix);
* ``rhs`` (3V, float32, the PCG right-hand side -g), ``solution`` (3V,
  float32, the PCG direction of the step, zero before a solve) and
  ``gradient`` (3V, float64);
* ``meta``: a JSON string (workload, seed, frame, semantics, tolerance ...).

The training pipeline writes one file per collected system
(``learned.collect(..., dump_dir=...)``, ``train_precond --dump DIR``), and the
same files serve as regression fixtures: ``load_system`` gives back the
arrays, ``dense`` the matrix of a small system, and
``ando_pcg_solve_noalloc`` solves the pattern part on the device.
"""
from __future__ import annotations

import json
from pathlib import Path
from typing import Optional

import numpy as np

from . import abi

KEYS = ("rowptr", "cols", "vals", "extra_rows", "extra_cols", "extra_vals", "rhs", "solution", "gradient")


def system_arrays(scene: abi.Scene) -> dict:
    """The last Newton system of `scene` (after ``step`` or ``eval_system``;
    CORRECTED semantics needs ``scene.keep_system()`` before it)."""
    rowptr, cols, vals, rhs, sol = scene.last_system()
    xr, xc, xv = scene.last_contact_blocks()
    return dict(rowptr=np.asarray(rowptr, np.int32), cols=np.asarray(cols, np.int32),
                vals=np.asarray(vals, np.float32).reshape(-1, 3, 3), extra_rows=np.asarray(xr, np.int32),
                extra_cols=np.asarray(xc, np.int32), extra_vals=np.asarray(xv, np.float32).reshape(-1, 3, 3),
                rhs=np.asarray(rhs, np.float32).ravel(), solution=np.asarray(sol, np.float32).ravel(),
                gradient=np.asarray(scene.last_gradient(), np.float64).ravel())


def save_system(path, scene: abi.Scene, **meta) -> Path:
    """Write the last Newton system of `scene` to `path` (``.npz``)."""
    return save_arrays(path, system_arrays(scene), **meta)


def save_arrays(path, arrays: dict, **meta) -> Path:
    p = Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    missing = [k for k in KEYS if k not in arrays]
    if missing:
        raise ValueError(f"system arrays lack {missing}")
    np.savez_compressed(p, meta=np.array(json.dumps(meta)), **{k: arrays[k] for k in KEYS})
    return p


def load_system(path) -> dict:
    """The arrays of a dumped system, checked for consistency; ``meta`` as a dict."""
    with np.load(Path(path), allow_pickle=False) as z:
        out = {k: z[k] for k in KEYS}
        out["meta"] = json.loads(str(z["meta"])) if "meta" in z.files else {}
    V = len(out["rowptr"]) - 1
    nnzb = len(out["cols"])
    if V < 0 or out["rowptr"][0] != 0 or out["rowptr"][-1] != nnzb or np.any(np.diff(out["rowptr"]) < 0):
        raise ValueError(f"{path}: bad row pointer")
    if out["vals"].shape != (nnzb, 3, 3) or out["rhs"].shape != (3 * V,) or out["solution"].shape != (3 * V,):
        raise ValueError(f"{path}: array shapes do not match {V} rows and {nnzb} blocks")
    if nnzb and (out["cols"].min() < 0 or out["cols"].max() >= V):
        raise ValueError(f"{path}: column index out of range")
    n = len(out["extra_rows"])
    if out["extra_cols"].shape != (n,) or out["extra_vals"].shape != (n, 3, 3):
        raise ValueError(f"{path}: extra blocks do not match")
    return out


def dense(system: dict, with_extra: bool = True, dtype=np.float64) -> np.ndarray:
    """The system matrix as a dense (3V, 3V) array (small systems only)."""
    V = len(system["rowptr"]) - 1
    A = np.zeros((3 * V, 3 * V), dtype=dtype)
    rp, cols, vals = system["rowptr"], system["cols"], system["vals"]
    for r in range(V):
        for k in range(rp[r], rp[r + 1]):
            c = cols[k]
            A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += vals[k]
    if with_extra:
        for r, c, b in zip(system["extra_rows"], system["extra_cols"], system["extra_vals"]):
            A[3 * r:3 * r + 3, 3 * c:3 * c + 3] += b
    return A


def frame_path(directory, workload: str, seed: int, frame: int, newton: Optional[int] = None) -> Path:
    """File name of a dumped system: <workload>_s<seed>_f<frame>[_n<newton>].npz."""
    tail = f"_n{newton}" if newton is not None else ""
    return Path(directory) / f"{workload}_s{seed}_f{frame:04d}{tail}.npz"
