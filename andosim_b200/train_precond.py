"""Train the learned preconditioner on the two-curtain workload and evaluate it.

    python -m andosim_b200.train_precond [--sets 256:0-14:1,64:0-239:4] [--train-seeds 0-7]
        [--eval-seeds 8-11] [--steps 3000] [--out PATH] [--report PATH] [--evaluate WEIGHTS] [--dump DIR]

Training data are the solver's own dumps: the first Newton system of the
chosen frames of CORRECTED-semantics runs of scenes.c4 for the training seeds,
each with probe residuals of a block-Jacobi solve. `--sets` lists
grid:first-last:every triples (several resolutions train one network: its
inputs are scale-free). Evaluation steps the held-out seeds over the same
frame ranges with block Jacobi and with the trained network (device timing,
PCG iterations per Newton step, fallbacks, and the final position difference
between the two runs).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path

import numpy as np

from . import abi, learned, scenes


def seeds(spec: str):
    out = []
    for part in spec.split(","):
        if "-" in part:
            a, b = part.split("-")
            out.extend(range(int(a), int(b) + 1))
        elif part:
            out.append(int(part))
    return out


def evaluate(sc, weights, frames: int, precond: str, refresh: int = 1, device: int = 0):
    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=device)
    if weights is not None:
        S.set_precond_weights(weights)
    p = abi.make_params(sc.params, semantics="corrected", precond=precond, precond_refresh=refresh)
    it = nw = fb = 0
    ms = 0.0
    for f in range(frames):
        S.apply_gravity(sc.gravity, p.dt)
        st = S.step(p, sc.pins_at(f), sc.walls)
        it += st["pcg_iters"]; nw += st["newton_iters"]; fb += st["precond_fallbacks"]; ms += st["device_ms"]
    x, _ = S.download()
    S.close()
    return dict(pcg_iters=it, newton_iters=nw, pcg_per_newton=it / max(nw, 1), fallbacks=fb, device_ms=ms,
                frames_per_s=frames / (ms * 1e-3) if ms > 0 else None), x


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sets", default="256:0-14:1,64:0-239:4")
    ap.add_argument("--train-seeds", default="0-7")
    ap.add_argument("--eval-seeds", default="8-11")
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--init-seed", type=int, default=0)
    ap.add_argument("--refresh", type=int, default=1)
    ap.add_argument("--out", default=str(learned.DEFAULT_WEIGHTS))
    ap.add_argument("--report", default=None)
    ap.add_argument("--dump", default=None, help="also write every training system as .npz into this directory")
    ap.add_argument("--evaluate", default=None,
                    help="weights (.npy) to evaluate on the held-out seeds instead of training new ones")
    a = ap.parse_args(argv)

    sets = []
    for spec in a.sets.split(","):
        n, fr, ev = spec.split(":")
        f0, f1 = fr.split("-")
        sets.append((int(n), int(f0), int(f1), int(ev)))
    if a.evaluate:
        w = learned.load_weights(a.evaluate)
        report = dict(sets=a.sets, weights=a.evaluate, eval=[])
        run_eval(a, sets, w, report)
        return
    t0 = time.time()
    trainer = abi.Trainer(abi.precond_init_weights(a.init_seed))
    n_sys = sum(learned.c4_training_set(trainer, seeds(a.train_seeds), n, range(f0, f1 + 1, ev), dump_dir=a.dump)
                for n, f0, f1, ev in sets)
    t_collect = time.time() - t0
    loss0 = learned.mean_loss(trainer)
    t1 = time.time()
    losses = learned.train(trainer, a.steps, lr=a.lr, log_every=max(a.steps // 10, 1))
    t_train = time.time() - t1
    loss1 = learned.mean_loss(trainer)
    w = trainer.weights()
    trainer.close()
    out = learned.save_weights(w, a.out)
    report = dict(sets=a.sets, train_seeds=seeds(a.train_seeds), systems=n_sys, collect_s=t_collect, train_steps=a.steps,
                  train_s=t_train, loss_before=loss0, loss_after=loss1, weights=str(out), eval=[])
    print(json.dumps({k: v for k, v in report.items() if k != "eval"}), flush=True)
    run_eval(a, sets, w, report)


def run_eval(a, sets, w, report):
    for n, f0, f1, _ in sets:
        for sd in seeds(a.eval_seeds):
            sc = scenes.c4(seed=sd, n=n)
            rj, xj = evaluate(sc, None, f1 + 1, "block_jacobi")
            rl, xl = evaluate(sc, w, f1 + 1, "learned", a.refresh)
            ext = float(np.ptp(sc.vertices, axis=0).max())
            row = dict(n=n, frames=f1 + 1, seed=sd, jacobi=rj, learned=rl, pos_diff_rel=float(np.abs(xl - xj).max() / ext),
                       iter_ratio=rl["pcg_per_newton"] / max(rj["pcg_per_newton"], 1e-30))
            report["eval"].append(row)
            print(json.dumps(row), flush=True)
    if a.report:
        Path(a.report).write_text(json.dumps(report, indent=1))


if __name__ == "__main__":
    main()
