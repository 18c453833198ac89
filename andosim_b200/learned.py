"""Training pipeline of the learned preconditioner (host side).

The solver dumps its own training data: for chosen frames of a scene run in
CORRECTED semantics, ``ando_eval_system`` evaluates the frame's first Newton
system on the device and ``ando_trainer_add_system`` keeps its block-scaled
form A^ together with probe residuals of a block-Jacobi solve. Training runs on
the device through the library's forward, backward and Adam kernels
(``ando_trainer_step``); this module only sequences those calls and stores the
resulting weights (a flat float32 vector, ``ando_precond_num_params()`` long).
"""
from __future__ import annotations

import time
from pathlib import Path
from typing import Iterable, List, Optional, Sequence

import numpy as np

from . import abi, dump, scenes

WEIGHTS_DIR = Path(__file__).resolve().parent / "weights"
DEFAULT_WEIGHTS = WEIGHTS_DIR / "precond_c4.npy"


def load_weights(path: Optional[Path] = None) -> np.ndarray:
    """Trained weights shipped with the package (or `path`)."""
    w = np.load(path or DEFAULT_WEIGHTS).astype(np.float32)
    if w.shape != (abi.precond_num_params(),):
        raise ValueError(f"{path or DEFAULT_WEIGHTS}: expected {abi.precond_num_params()} weights, got {w.shape}")
    return w


def save_weights(w: np.ndarray, path: Optional[Path] = None) -> Path:
    p = Path(path or DEFAULT_WEIGHTS)
    p.parent.mkdir(parents=True, exist_ok=True)
    np.save(p, np.asarray(w, dtype=np.float32))
    return p


def collect(trainer: abi.Trainer, sc: scenes.Scene, frames: Iterable[int], device: int = 0, max_probes: int = 6,
            tol: float = 1e-6, params: Optional[dict] = None, dump_dir: Optional[Path] = None, seed: int = -1) -> int:
    """Step `sc` in CORRECTED semantics with block Jacobi and add the first
    Newton system of every frame in `frames` to the trainer. Returns how many
    systems were added (frames whose system had already converged add none).
    With `dump_dir` every evaluated system is also written there as an
    ``.npz`` file (andosim_b200.dump)."""
    frames = sorted(set(frames))
    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=device)
    p = abi.make_params(dict(sc.params, **(params or {})), semantics="corrected")
    if dump_dir is not None:
        S.keep_system()
    added = 0
    try:
        for f in range(frames[-1] + 1):
            S.apply_gravity(sc.gravity, p.dt)
            if f in frames:
                S.eval_system(p, sc.pins_at(f), sc.walls)
                if dump_dir is not None:
                    dump.save_system(dump.frame_path(dump_dir, sc.name, seed, f), S, workload=sc.name, seed=seed, frame=f,
                                     semantics="corrected", newton_iteration=0, pcg_tol=float(p.pcg_tol))
                try:
                    trainer.add_system(S, max_probes=max_probes, tol=tol)
                    added += 1
                except abi.AbiError as e:
                    if "already converged" not in str(e) and "no usable probe" not in str(e):
                        raise
            S.step(p, sc.pins_at(f), sc.walls)
    finally:
        S.close()
    return added


def train(trainer: abi.Trainer, steps: int, lr: float = 1e-3, lr_final: Optional[float] = None, log_every: int = 0) -> List[float]:
    """`steps` Adam steps cycling over the trainer's systems, cosine-decayed
    learning rate from `lr` to `lr_final` (default lr / 10). Returns the losses."""
    lr_final = lr / 10 if lr_final is None else lr_final
    losses = []
    t0 = time.time()
    for k in range(steps):
        c = 0.5 * (1 + np.cos(np.pi * k / max(steps - 1, 1)))
        losses.append(trainer.step(lr_final + (lr - lr_final) * c))
        if log_every and (k + 1) % log_every == 0:
            print(f"step {k + 1}/{steps} loss {np.mean(losses[-log_every:]):.5f} ({time.time() - t0:.1f} s)", flush=True)
    return losses


def mean_loss(trainer: abi.Trainer) -> float:
    return float(np.mean([trainer.loss(i) for i in range(len(trainer))]))


def c4_training_set(trainer: abi.Trainer, seeds: Sequence[int], n: int, frames: Iterable[int], device: int = 0,
                    dump_dir: Optional[Path] = None) -> int:
    """Systems of the two-curtain workload (scenes.c4) for several seeds."""
    total = 0
    for sd in seeds:
        total += collect(trainer, scenes.c4(seed=sd, n=n), frames, device=device, dump_dir=dump_dir, seed=sd)
    return total
