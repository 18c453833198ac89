#!/usr/bin/env python
"""Benchmark of the implicit cloth step on B200.

Workload: two 2 m x 2 m curtains of 256 x 256 vertices (131,072 vertices,
260,100 triangles), 3 mm apart, top rows pinned and driven +-0.3 m along x at
0.5 Hz in opposite phase, ground plane at z = 0 (synthetic, seeded), stepped
with the reference's semantics and block-Jacobi PCG. One bench step = one
frame: State.apply_gravity + Integrator.step, as the reference demos drive it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line on rank 0. `value` is frames/s over all ranks with the
state resident on the device, timed with CUDA events on the library's stream
(L2 flushed before every timed frame); `e2e` is the same metric through the
`ando_barrier_core` Python API with the per-frame host<->device copies inside
the timed region. With N > 1 every rank runs an independent replica (the step
has no exchange between scenes), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "frames/s, PCG iters/Newton: learned vs Jacobi PCG, 1×B200, ≤1e-4 pos err"
WORKLOAD = "c4_curtains_2x256x256"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=240)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256, help="curtain grid side")
    ap.add_argument("--cpu-frames", type=int, default=1, help="frames of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--corrected-steps", type=int, default=60, help="frames of the CORRECTED-semantics measurement (0: skip)")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_setup(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = False
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
        pg = True
    return rank, world, local, pg


def dist_max(x, pg):
    if not pg:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg:
        import torch.distributed as dist

        dist.barrier()


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"ando_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        try:
            self.path.unlink()
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------- ours
def algorithmic_bytes(V, T, nnzb, prof):
    """Algorithmic bytes per phase over the timed region.

    assembly  : 24 V + 72 nnzb per launch (x and g read once, the cached 36-B
                constant block read and the 36-B value block written per slot)
    PCG       : 40 nnzb + 160 V per iteration (block SpMV + fused vector updates)
                plus 48 V per launch (x, r, z initialisation)
    gradient  : 212 V per launch (x, x_hat, per-step constants and mass read,
                g, rhs and the diagonal terms written)
    strain    : 53 T + 24 V per launch (indices, rest data, positions, flags)
    """
    pl = prof["phase_launches"]
    out = {}
    out["assemble"] = (24 * V + 72 * nnzb) * pl["assemble"]
    out["pcg"] = (40 * nnzb + 160 * V) * prof["pcg_iterations"] + 48 * V * pl["pcg"]
    # the gradient phase counts the gradient kernel and the 1-thread check kernel
    out["gradient"] = 212 * V * (pl["gradient"] // 2 if pl["gradient"] else 0)
    out["strain"] = (53 * T + 24 * V) * (pl["strain"] // 2 if pl["strain"] else 0)
    return out


def run_ours(args, rank, world, local, pg):
    import torch

    from andosim_b200 import abi, scenes
    from andosim_b200.build import build

    if rank == 0:
        build()
    barrier(pg)
    torch.cuda.set_device(local)
    sc = scenes.c4(seed=rank, n=args.n)
    V, T = sc.num_vertices, sc.num_triangles
    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    params = abi.make_params(sc.params)
    stream = torch.cuda.ExternalStream(S.stream(), device=torch.device("cuda", local))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = ClockSampler(local)

    frame = 0

    def do_frame(f, pins=None):
        S.apply_gravity(sc.gravity, params.dt)
        return S.step(params, sc.pins_at(f) if pins is None else pins, sc.walls)

    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)

    def timed(n, first):
        stats, ms = [], 0.0
        for k in range(n):
            pins = abi.pin_array(sc.pins_at(first + k))     # the scene's driven pin targets, built untimed
            with torch.cuda.stream(stream):
                flush.zero_()          # evict L2 (256 MB > 126 MB) before every timed frame
                ev_a.record(stream)
            stats.append(do_frame(first + k, pins))
            ev_b.record(stream)
            ev_b.synchronize()
            ms += ev_a.elapsed_time(ev_b)
        return stats, ms

    for _ in range(args.warmup):
        do_frame(frame)
        frame += 1
    torch.cuda.synchronize()
    barrier(pg)
    clocks.start()
    # headline pass: profiler off, so each frame is one whole-frame CUDA graph launch
    S.profile_enable(False)                 # also resets the launch counters
    stats, total_ms = timed(args.steps, frame)
    frame += args.steps
    launches = int(S.profile()["launches"])
    graph_frames = sum(int(s["graph_launched"]) for s in stats)
    torch.cuda.synchronize()
    total_ms = dist_max(total_ms, pg)
    barrier(pg)
    # phase breakdown: a separate pass with per-phase CUDA events (host-driven loop)
    prof_frames = min(args.steps, 120)
    S.profile_enable(True)
    _, prof_total_ms = timed(prof_frames, frame)
    frame += prof_frames
    prof = S.profile()
    S.profile_enable(False)
    barrier(pg)

    # end to end through the Python API: host buffers, copies inside the timed region
    from andosim_b200 import ando_barrier_core as abc

    abc.set_device(local)
    m = abc.Mesh()
    m.initialize(sc.vertices, sc.triangles, abc.Material(**sc.material))
    st = abc.State()
    st.initialize(m)
    p = abc.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)

    def api_frame(f):
        c = abc.Constraints()
        for i, t in sc.pins_at(f):
            c.add_pin(int(i), t)
        for n, o, g in sc.walls:
            c.add_wall(n, o, g)
        st.apply_gravity(sc.gravity, p.dt)
        abc.Integrator.step(m, st, c, p)
        return st.get_positions()

    for f in range(args.warmup):
        api_frame(f)
    e2e_stream = torch.cuda.ExternalStream(st._stream_handle(), device=torch.device("cuda", local))
    e2e_ms = 0.0
    for f in range(args.steps):
        with torch.cuda.stream(e2e_stream):
            flush.zero_()
            ev_a.record(e2e_stream)
        pos = api_frame(args.warmup + f)
        ev_b.record(e2e_stream)
        ev_b.synchronize()
        e2e_ms += ev_a.elapsed_time(ev_b)
    e2e_ms = dist_max(e2e_ms, pg)
    clock_info = clocks.stop()
    n_pins = len(sc.pins_at(0))
    h2d = n_pins * (4 + 24) + len(sc.walls) * 48          # pins and walls uploaded each step
    d2h = 2 * 24 * V                                      # positions and velocities (FP64) read back

    # roofline of the dominant phase
    nnzb = 0
    try:
        rowptr, cols, vals, rhs, sol = S.last_system()
        nnzb = int(len(cols))
    except Exception:
        pass
    ab = algorithmic_bytes(V, T, nnzb, prof)
    peaks = json.loads(PEAKS_FILE.read_text()) if PEAKS_FILE.exists() else {}
    hbm = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    phase_ms = prof["phase_ms"]
    # dominant kernel phase among those with an algorithmic byte count
    dom = max(ab, key=lambda k: phase_ms.get(k, 0.0))
    dom_bytes = ab.get(dom)
    roof = None
    if dom_bytes is not None and phase_ms[dom] > 0:
        dom_launches = max(1, prof["phase_launches"][dom] // (2 if dom in ("gradient", "strain") else 1))
        achieved = dom_bytes / (phase_ms[dom] * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "traffic": None, "peak_source": "measured" if peaks else "fallback",
                "bytes_per_launch": dom_bytes // dom_launches, "launches": dom_launches,
                "avg_launch_us": round(phase_ms[dom] * 1e3 / dom_launches, 2)}
    newton = sum(s["newton_iters"] for s in stats)
    pcg = sum(s["pcg_iters"] for s in stats)
    fps = args.steps * world / (total_ms * 1e-3)
    out = {
        "metric": METRIC, "value": round(fps, 2), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 BSR/PCG vectors, f64 positions/gradient/dots",
        "data": "synthetic (seeded curtains, scenes.c4)",
        "config": {"workload": WORKLOAD, "vertices": V, "triangles": T, "bsr_blocks": nnzb, "semantics": "REFERENCE",
                   "preconditioner": "block_jacobi", "frames_timed_per_gpu": args.steps, "l2": "flushed before every timed frame",
                   "parallelism": f"replicas x{world}"},
        "newton_iters_per_frame": round(newton / args.steps, 3),
        "pcg_iters_per_newton": round(pcg / newton, 3) if newton else 0.0,
        "newton_iters_per_s": round(newton * world / (total_ms * 1e-3), 1),
        "graph_frames": graph_frames,
        "profiled_pass": {"frames": prof_frames, "ms_per_frame": round(prof_total_ms / prof_frames, 4),
                          "phase_ms_per_frame": {k: round(v / prof_frames, 5) for k, v in phase_ms.items()}},
        "gpu_launches": launches,
        "e2e": {"value": round(args.steps * world / (e2e_ms * 1e-3), 2), "unit": "frames/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roof,
        "clocks": clock_info,
    }
    S.close()
    if args.corrected_steps > 0:
        out["corrected"] = run_corrected(args, sc, local, flush, pg)
    return out, sc


def run_corrected(args, sc, local, flush, pg, precond="block_jacobi"):
    """The same workload in CORRECTED semantics (elasticity on the current
    positions, kinematic pins, working self contact, time-of-impact line
    search): a real PCG solve every Newton iteration."""
    import torch

    from andosim_b200 import abi

    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    params = abi.make_params(sc.params, semantics="corrected", precond=precond)
    stream = torch.cuda.ExternalStream(S.stream(), device=torch.device("cuda", local))
    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)
    for f in range(args.warmup):
        S.apply_gravity(sc.gravity, params.dt)
        S.step(params, sc.pins_at(f), sc.walls)
    S.profile_enable(True)
    total_ms, stats = 0.0, []
    for k in range(args.corrected_steps):
        f = args.warmup + k
        pins = abi.pin_array(sc.pins_at(f))
        with torch.cuda.stream(stream):
            flush.zero_()
            ev_a.record(stream)
        S.apply_gravity(sc.gravity, params.dt)
        stats.append(S.step(params, pins, sc.walls))
        ev_b.record(stream)
        ev_b.synchronize()
        total_ms += ev_a.elapsed_time(ev_b)
    prof = S.profile()
    S.close()
    total_ms = dist_max(total_ms, pg)
    newton = sum(s["newton_iters"] for s in stats)
    pcg = sum(s["pcg_iters"] for s in stats)
    nnzb = 0
    V = sc.num_vertices
    pcg_ms = prof["phase_ms"]["pcg"]
    pcg_iters = prof["pcg_iterations"]
    return {
        "semantics": "CORRECTED", "preconditioner": precond, "frames": args.corrected_steps,
        "frames_per_s": round(args.corrected_steps / (total_ms * 1e-3), 2),
        "ms_per_frame": round(total_ms / args.corrected_steps, 3),
        "newton_iters_per_frame": round(newton / args.corrected_steps, 3),
        "pcg_iters_per_newton": round(pcg / newton, 2) if newton else 0.0,
        "newton_iters_per_s": round(newton / (total_ms * 1e-3), 1),
        "pcg_us_per_iteration": round(pcg_ms * 1e3 / pcg_iters, 2) if pcg_iters else None,
        "phase_ms_per_frame": {k: round(v / args.corrected_steps, 4) for k, v in prof["phase_ms"].items()},
        "contacts_max": max(s["contacts"] for s in stats) if stats else 0,
        "gpu_launches": int(prof["launches"]),
    }


# ----------------------------------------------------------- CPU baseline
def oracle_frames(sc, frames, prec="f32", lookup="indexed"):
    """Time `frames` oracle steps of scene `sc` (single thread). Returns seconds per frame."""
    from oracle.build import load

    O = getattr(load(), prec)
    m = O.Mesh()
    m.initialize(sc.vertices, sc.triangles, O.Material(**sc.material))
    s = O.State()
    s.initialize(m)
    p = O.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)
    secs = 0.0
    for f in range(frames):
        c = O.Constraints()
        for i, t in sc.pins_at(f):
            c.add_pin(int(i), t)
        for n, o, g in sc.walls:
            c.add_wall(n, o, g)
        s.apply_gravity(sc.gravity, p.dt)
        t0 = time.perf_counter()
        O.Integrator.step(m, s, c, p, None, lookup)
        secs += time.perf_counter() - t0
    return secs / frames


def cpu_baseline(sc, frames):
    spf = oracle_frames(sc, frames)
    return {"value": round(1.0 / spf, 4), "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": f"{frames} frame(s) of {WORKLOAD} ({sc.num_vertices} vertices) through the FP32 oracle "
                      f"(C++ restatement of the reference, INDEXED block lookup, one thread)"}


def run_reference(args, rank, world, pg):
    """The reference's CPU path (oracle port; the reference itself does not build here) on the same workload."""
    if rank != 0:
        return None
    from andosim_b200 import scenes

    sc = scenes.c4(seed=0, n=args.n)
    spf = oracle_frames(sc, max(1, min(args.steps, 3)))
    base = {"value": round(1.0 / spf, 4), "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": f"{max(1, min(args.steps, 3))} frame(s) of {WORKLOAD} through the FP32 oracle "
                      "(C++ restatement of the reference, INDEXED block lookup, one thread; the reference "
                      "is single-threaded)"}
    return {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(spf * 1e3, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded curtains, scenes.c4)",
            "config": {"workload": WORKLOAD, "vertices": sc.num_vertices, "semantics": "REFERENCE"},
            "cpu_baseline": base, "e2e": {"value": base["value"], "unit": "frames/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world, pg)
        else:
            out, sc = run_ours(args, rank, world, local, pg)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                out["cpu_baseline"] = cpu_baseline(sc, args.cpu_frames)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if pg:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
