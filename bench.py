#!/usr/bin/env python
"""Benchmark of the implicit cloth step on B200.

Workload: two 2 m x 2 m curtains of 256 x 256 vertices (131,072 vertices,
260,100 triangles), 3 mm apart, top rows pinned and driven +-0.3 m along x at
0.5 Hz in opposite phase, ground plane at z = 0, Newton/PCG tolerance 1e-4
(synthetic, seeded). One bench step = one frame: State.apply_gravity +
Integrator.step, as the reference demos drive it.

Headline (`value`): frames/s of the CORRECTED step (the step the reference
intends: as-rigid-as-possible membrane forces on the current positions, pins
as springs of the implicit solve, contact stiffness from the current gap,
working self contact, conservative time-of-impact line search, sub-steps for
fast drives) with the learned preconditioner, next to the same frames with
block-Jacobi PCG (`jacobi`, each frame stepped from the same state), with PCG
iterations per Newton step for both. `reference_semantics` times the
reference's own step (REFERENCE semantics, block Jacobi, whole frame as one
CUDA graph); `cpu_baseline` and `fp64_step_error` step the oracle from the
GPU's state at the first timed frame; `--impl reference` runs the oracle on
the same workload, semantics and frames.

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
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256, help="curtain grid side")
    ap.add_argument("--reference-budget", type=float, default=150.0,
                    help="seconds of timed frames the CPU reference arm may spend (it times the frames that fit)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-steps", type=int, default=240, help="frames of the REFERENCE-semantics measurement (0: skip)")
    ap.add_argument("--full-n", type=int, default=64, help="curtain grid of the full-length CORRECTED comparison (0: skip)")
    ap.add_argument("--full-steps", type=int, default=240, help="frames of the full-length CORRECTED comparison")
    ap.add_argument("--refresh", type=int, default=8,
                    help="Newton iterations between evaluations of the preconditioner network (8: about once per frame; in "
                         "between, S is rebuilt from each Newton system with the last coefficients)")
    ap.add_argument("--pcg-shape", type=int, default=-1,
                    help="learned scaled-PCG launch candidate of the timed contexts (-1: autotune on the first solve; "
                         "a fixed candidate reproduces one shape, e.g. under a profiler)")
    ap.add_argument("--weights", default=None, help="learned preconditioner weights (.npy); default: the shipped C4 weights")
    ap.add_argument("--c3-frames", type=int, default=60, help="timed frames of the batched 64-scene comparison (0: skip)")
    ap.add_argument("--c2-frames", type=int, default=200, help="frames of the four-sheet stack (0: skip)")
    ap.add_argument("--seeds", type=int, default=3, help="seeds of the curtain workload in the paired learned/Jacobi window")
    ap.add_argument("--c5-frames", type=int, default=0, help="frames of the tablecloth over the box (0: skip)")
    ap.add_argument("--heldout-frames", type=int, default=300,
                    help="frames of the full-length learned runs of the curtains on the held-out seeds (0: skip)")
    ap.add_argument("--heldout-seeds", default="8,9,10,11", help="held-out curtain seeds (the shipped weights trained on 0-7)")
    ap.add_argument("--c5-n", type=int, default=512, help="tablecloth grid side")
    return ap.parse_args()


# ---------------------------------------------------------------- distributed
def dist_setup(n_gpus, backend=None):
    """One process per GPU (RANK / WORLD_SIZE / LOCAL_RANK from torchrun). The
    ranks run independent replicas (seeded by rank); the only collectives are
    the barriers around timed regions and the max over ranks of each time.
    NCCL on GPUs; gloo when given (the CPU tests of this logic)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = False
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        backend = backend or "nccl"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
        pg = True
    return rank, world, local, pg


def dist_max(x, pg):
    """Max of x over the ranks (the job's time is its slowest rank's)."""
    if not pg:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
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
def pcg_bytes(V, nnzb, prof):
    """Algorithmic bytes of the scaled PCG over the profiled frames.

    Per block-Jacobi iteration (CG on the scaled system, identity diagonal):
      phase A  40 nnzb (scaled BSR values + column) + 40 per contact block
               outside the mesh pattern, 12 V each for z, p_old (gathered
               once), p_new and Ap
      phase B  12 V p, 24 V x^ read+write (FP64), 12 V Ap, 24 V r read+write,
               24 V L (FP32, residual norm)
      = 40 nnzb + 40 n_extra + 144 V
    A learned iteration adds the second product z = S r on the mesh pattern,
    applied as S_ij = coef_ij A^_ij plus S's diagonal blocks:
      + 44 nnzb (A^ values, column, coefficient) + 36 V (diagonal blocks)
      + 24 V (r2, z written) + 12 V (Ap gathered)
    plus 48 V per launch (initialisation and d = L^-T x^)."""
    it = prof["pcg_iterations"]
    lit = prof["pcg_learned_iterations"]
    return (40 * nnzb + 144 * V) * it + 40 * prof["pcg_extra_block_iterations"] + (44 * nnzb + 72 * V) * lit \
        + 48 * V * prof["phase_launches"]["pcg"]


def assembly_bytes(V, nnzb, learned=True):
    """Algorithmic bytes of one CORRECTED assembly, k_diag_factor + k_assemble_scaled_slice.
      k_diag_factor, per vertex: the FP64 diagonal terms (72) and gradient (24) in; L^-1 (FP64, 48),
        L (FP32, 24), b^ (12) and the factor flag (1) out                                   = 181 V
      k_assemble_scaled_slice, per block slot: the FP64 elastic pair (16), its row, column and SELL
        position (12) in, the scaled FP32 block out in SELL order (36)                      = 64 nnzb
        per vertex: the row's and the column's L^-1 (48 each, each read once) and the diagonal terms
        (72) again                                                                          = 168 V
      learned preconditioner: the scaled block again in CSR order for the network's features = 36 nnzb"""
    return 349 * V + (100 if learned else 64) * nnzb


# DRAM bytes (read + write) per launch of the kernel on this workload, from one ncu capture (the summaries
# under profiles/ give the command): the PCG's matrix and vectors come from DRAM once per launch and from L2
# for every later iteration; the assembly's figure is k_diag_factor plus k_assemble_scaled_slice (44.9 + 27.9 MB).
PCG_TRAFFIC = 53_985_536
ASSEMBLY_TRAFFIC = 72_798_720


class Timer:
    """CUDA-event timing of frames on the library's stream, L2 flushed before each."""

    def __init__(self, torch, stream, flush):
        self.torch, self.stream, self.flush = torch, stream, flush
        self.a = torch.cuda.Event(enable_timing=True)
        self.b = torch.cuda.Event(enable_timing=True)

    def frame(self, fn):
        with self.torch.cuda.stream(self.stream):
            self.flush.zero_()          # evict L2 (256 MB > 126 MB) before every timed frame
            self.a.record(self.stream)
        r = fn()
        self.b.record(self.stream)
        self.b.synchronize()
        return r, self.a.elapsed_time(self.b)


def corrected_run(args, sc, local, flush, pg, precond, weights, profile=False, frames=None):
    """`frames` CORRECTED frames after `warmup` untimed ones, device-resident
    (the profiled pass: per-phase CUDA events)."""
    import torch

    from andosim_b200 import abi

    frames = args.steps if frames is None else frames
    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    if weights is not None:
        S.set_precond_weights(weights)
    if args.pcg_shape >= 0:
        S.select_pcg_shape(True, args.pcg_shape)
    params = abi.make_params(sc.params, semantics="corrected", precond=precond, precond_refresh=args.refresh)
    tm = Timer(torch, torch.cuda.ExternalStream(S.stream(), device=torch.device("cuda", local)), flush)
    for f in range(args.warmup):
        S.apply_gravity(sc.gravity, params.dt)
        S.step(params, sc.pins_at(f), sc.walls)
    S.profile_enable(profile)
    total_ms, stats = 0.0, []
    for k in range(frames):
        pins = abi.pin_array(sc.pins_at(args.warmup + k))

        def one():
            S.apply_gravity(sc.gravity, params.dt)
            return S.step(params, pins, sc.walls)
        st, ms = tm.frame(one)
        stats.append(st)
        total_ms += ms
    prof = S.profile()
    nnzb = S.system_size()[1]
    shape = S.pcg_shape(precond == "learned")
    S.close()
    newton = sum(s["newton_iters"] for s in stats)
    pcg = sum(s["pcg_iters"] for s in stats)
    return {"preconditioner": precond, "frames": frames, "ms_per_frame": round(total_ms / frames, 3),
            "pcg_iters_per_newton": round(pcg / newton, 2) if newton else 0.0,
            "phase_ms_per_frame": {k: round(v / frames, 4) for k, v in prof["phase_ms"].items()},
            "pcg_us_per_iteration": round(prof["phase_ms"]["pcg"] * 1e3 / prof["pcg_iterations"], 2) if prof["pcg_iterations"] else None,
            "pcg_launch_shape": {q: shape[q] for q in ("tpb", "grid", "unroll", "candidates")},
            "_prof": prof, "_nnzb": nnzb}


def paired_run(args, sc, local, flush, pg, weights, steps=None, raw=False):
    """The learned-preconditioner trajectory, timed frame by frame; before each
    learned frame a block-Jacobi frame is timed from the same state and then
    undone, so both preconditioners solve exactly the same Newton systems of
    the first iteration and the comparison does not depend on where two
    contact-rich trajectories drift apart."""
    import torch

    from andosim_b200 import abi

    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    S.set_precond_weights(weights)
    if args.pcg_shape >= 0:
        S.select_pcg_shape(True, args.pcg_shape)
    pl = abi.make_params(sc.params, semantics="corrected", precond="learned", precond_refresh=args.refresh)
    pj = abi.make_params(sc.params, semantics="corrected", precond="block_jacobi")
    tm = Timer(torch, torch.cuda.ExternalStream(S.stream(), device=torch.device("cuda", local)), flush)
    for f in range(args.warmup):
        S.apply_gravity(sc.gravity, pl.dt)
        S.step(pl, sc.pins_at(f), sc.walls)
    torch.cuda.synchronize()
    barrier(pg)
    S.profile_enable(False)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    res = {"learned": dict(ms=0.0, stats=[], launches=0), "block_jacobi": dict(ms=0.0, stats=[], launches=0)}
    diffs = []
    steps = args.steps if steps is None else steps
    for k in range(steps):
        pins = abi.pin_array(sc.pins_at(args.warmup + k))
        x0, v0 = S.download()
        outs = {}
        for name, p in (("block_jacobi", pj), ("learned", pl)):
            if name == "learned":
                S.upload(x0, v0)
            n0 = S.profile()["launches"]

            def one():
                S.apply_gravity(sc.gravity, p.dt)
                return S.step(p, pins, sc.walls)
            st, ms = tm.frame(one)
            r = res[name]
            r["ms"] += ms
            r["stats"].append(st)
            r["launches"] += S.profile()["launches"] - n0
            outs[name] = S.download()[0]
        diffs.append(float(np.abs(outs["learned"] - outs["block_jacobi"]).max() / ext))
    crossings = S.edge_triangle_crossings()       # untimed: the window's end state, exact test on the GPU
    S.close()
    if raw:
        return res, diffs, steps, crossings
    out = summarize_pair(args, res, diffs, steps, pg)
    out["edge_triangle_crossings_end"] = crossings
    return out


def summarize_pair(args, res, diffs, steps, pg):
    """Per-arm frames/s and iteration counts of paired frames (summed over scenes)."""
    out = {}
    for name, r in res.items():
        ms = dist_max(r["ms"], pg)
        stats = r["stats"]
        newton = sum(s["newton_iters"] for s in stats)
        pcg = sum(s["pcg_iters"] for s in stats)
        out[name] = {"frames": steps, "total_ms": ms, "frames_per_s": round(steps / (ms * 1e-3), 2),
                     "ms_per_frame": round(ms / steps, 3), "newton_iters_per_frame": round(newton / steps, 3),
                     "pcg_iters_per_newton": round(pcg / newton, 2) if newton else 0.0,
                     "newton_iters_per_s": round(newton / (ms * 1e-3), 1),
                     "precond_fallbacks": sum(s["precond_fallbacks"] for s in stats),
                     "line_search_fail": sum(s["line_search_fail"] for s in stats),
                     "substeps": sum(s["substeps"] for s in stats),
                     "contacts_max": max(s["contacts"] for s in stats) if stats else 0,
                     "gpu_launches": int(r["launches"])}
    out["learned"]["refresh"] = args.refresh
    out["step_position_diff_rel_extent"] = {"max": max(diffs) if diffs else 0.0, "median": float(np.median(diffs)) if diffs else 0.0}
    return out


def reference_semantics_run(args, sc, local, flush, pg):
    """The reference's own step (REFERENCE semantics, block Jacobi): each frame one whole-frame CUDA graph."""
    import torch

    from andosim_b200 import abi

    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    params = abi.make_params(sc.params)
    tm = Timer(torch, torch.cuda.ExternalStream(S.stream(), device=torch.device("cuda", local)), flush)
    for f in range(args.warmup):
        S.apply_gravity(sc.gravity, params.dt)
        S.step(params, sc.pins_at(f), sc.walls)
    S.profile_enable(False)
    total_ms, stats = 0.0, []
    for k in range(args.reference_steps):
        pins = abi.pin_array(sc.pins_at(args.warmup + k))

        def one():
            S.apply_gravity(sc.gravity, params.dt)
            return S.step(params, pins, sc.walls)
        st, ms = tm.frame(one)
        stats.append(st)
        total_ms += ms
    launches = int(S.profile()["launches"])
    S.close()
    total_ms = dist_max(total_ms, pg)
    newton = sum(s["newton_iters"] for s in stats)
    pcg = sum(s["pcg_iters"] for s in stats)
    return {"semantics": "REFERENCE", "preconditioner": "block_jacobi", "frames": args.reference_steps,
            "frames_per_s": round(args.reference_steps / (total_ms * 1e-3), 2),
            "ms_per_frame": round(total_ms / args.reference_steps, 4),
            "newton_iters_per_frame": round(newton / args.reference_steps, 3),
            "pcg_iters_per_newton": round(pcg / newton, 3) if newton else 0.0,
            "graph_frames": sum(int(s["graph_launched"]) for s in stats), "gpu_launches": launches}


def e2e_run(args, scs, local, flush, pg, weights):
    """Frames/s through the ando_barrier_core API (host arrays in, positions out every frame), over the
    same seeds and frames as the device-resident number: frames 0..W-1 untimed, W..W+K-1 timed."""
    import torch

    from andosim_b200 import ando_barrier_core as abc

    abc.set_device(local)
    abc.set_precond_weights(weights)
    e2e_ms, frames = 0.0, 0
    for sc in scs:
        m = abc.Mesh()
        m.initialize(sc.vertices, sc.triangles, abc.Material(**sc.material))
        st = abc.State()
        st.initialize(m)
        p = abc.SimParams()
        for k, v in sc.params.items():
            setattr(p, k, v)
        p.semantics = "corrected"
        p.preconditioner = "learned"
        p.precond_refresh = args.refresh

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
        tm = Timer(torch, torch.cuda.ExternalStream(st._stream_handle(), device=torch.device("cuda", local)), flush)
        for f in range(args.steps):
            _, ms = tm.frame(lambda: api_frame(args.warmup + f))
            e2e_ms += ms
            frames += 1
        del st, m
    e2e_ms = dist_max(e2e_ms, pg)
    sc = scs[0]
    n_pins = len(sc.pins_at(0))
    return {"value": round(frames * int(os.environ.get("WORLD_SIZE", "1")) / (e2e_ms * 1e-3), 2), "unit": "frames/s",
            "frames": frames, "h2d_bytes_per_step": n_pins * (4 + 24) + len(sc.walls) * 48,   # pins and walls uploaded each step
            "d2h_bytes_per_step": 24 * sc.num_vertices}                                      # positions (FP64) read back


def c3_run(args, local, seed=0):
    """The batched workload: 64 uneven cloths (16..128 per side, 1-4 corner pins,
    log-uniform E), CORRECTED step with block Jacobi. Scene by scene (one host
    thread, one scene at a time) against ando_step_batch (the scenes' contexts
    stepping concurrently on their own streams). Each call returns when its
    scenes' steps are done; the wall time of whole frames is measured with the
    device idle on both sides. Both sets start from the same state and must end
    with the same bits."""
    import torch

    from andosim_b200 import abi, scenes

    scs = scenes.c3(seed=seed, scenes=64)
    params = [abi.make_params(sc.params, semantics="corrected") for sc in scs]
    sets = {m: [abi.Scene(sc.vertices, sc.triangles, sc.material, device=local) for sc in scs] for m in ("sequential", "batched")}
    times = {m: 0.0 for m in sets}
    newton = {m: 0 for m in sets}
    warm = 2
    for f in range(warm + args.c3_frames):
        for mode, S in sets.items():
            for s_, sc, p in zip(S, scs, params):
                s_.apply_gravity(sc.gravity, p.dt)
            torch.cuda.synchronize(local)
            t0 = time.perf_counter()
            if mode == "sequential":
                st = [s_.step(p, sc.pins_at(f), sc.walls) for s_, sc, p in zip(S, scs, params)]
            else:
                st = abi.step_batch(S, params, [sc.pins_at(f) for sc in scs], [sc.walls for sc in scs], threads=16)
            torch.cuda.synchronize(local)
            if f >= warm:
                times[mode] += time.perf_counter() - t0
                newton[mode] += sum(x["newton_iters"] for x in st)
    same = True
    for a, b in zip(sets["sequential"], sets["batched"]):
        xa, va = a.download()
        xb, vb = b.download()
        same = same and bool(np.array_equal(xa, xb) and np.array_equal(va, vb))
    for S in sets.values():
        for s_ in S:
            s_.close()
    nf = max(args.c3_frames, 1)
    out = {"workload": "c3_64_scenes_16_to_128", "vertices": int(sum(sc.num_vertices for sc in scs)), "frames": args.c3_frames,
           "semantics": "CORRECTED", "preconditioner": "block_jacobi", "timing": "host wall clock around whole batch frames, device idle before and after",
           "identical_results": same}
    for mode in sets:
        out[mode] = {"scene_frames_per_s": round(64 * nf / max(times[mode], 1e-9), 1), "ms_per_batch_frame": round(1e3 * times[mode] / nf, 3),
                     "newton_iters_per_frame": round(newton[mode] / (64 * nf), 3)}
    out["speedup"] = round(times["sequential"] / max(times["batched"], 1e-9), 3)
    return out


def c2_run(args, local, pg, seed=0):
    """The four-sheet stack (4 x 96 x 96, 200 frames: drop, land, stack), CORRECTED with block Jacobi,
    device-resident; contacts judged every 20 frames by the module's CollisionValidator on the CORRECTED
    contact set (reduced on the device), the exact edge-triangle crossing count and the lowest vertex
    height."""
    import torch

    from andosim_b200 import abi, ando_barrier_core as abc, scenes

    sc = scenes.c2(seed=seed, frames=args.c2_frames)
    abc.set_device(local)
    m = abc.Mesh()
    m.initialize(sc.vertices, sc.triangles, abc.Material(**sc.material))
    st = abc.State()
    st.initialize(m)
    p = abc.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)
    p.semantics = "corrected"
    ms, newton, pcg, contacts, penetrations, zmin, fails, crossings = 0.0, 0, 0, 0, 0, 1e9, 0, 0
    c = abc.Constraints()
    for n, o, g in sc.walls:
        c.add_wall(n, o, g)
    for f in range(args.c2_frames):
        st.apply_gravity(sc.gravity, p.dt)
        abc.Integrator.step(m, st, c, p)
        s_ = abc.Integrator.last_step_stats(st)
        ms += s_["device_ms"]; newton += s_["newton_iters"]; pcg += s_["pcg_iters"]; fails += s_["line_search_fail"]
        if f % 20 == 19 or f == args.c2_frames - 1:
            cs = abc.Integrator.compute_contacts(m, st, None, "corrected", float(p.contact_gap_max))
            contacts = max(contacts, len(cs))
            met = abc.CollisionValidator.compute_metrics(m, st, cs, float(p.contact_gap_max), True)
            penetrations += int(met.num_penetrations)
            crossings += int(abc.CollisionValidator.edge_triangle_crossings(m, st))
            zmin = min(zmin, float(st.get_positions64()[:, 2].min()))
    ms = dist_max(ms, pg)
    return {"workload": "c2_stack_4x96x96", "vertices": sc.num_vertices, "frames": args.c2_frames, "semantics": "CORRECTED",
            "preconditioner": "block_jacobi", "frames_per_s": round(args.c2_frames / (ms * 1e-3), 2),
            "newton_iters_per_frame": round(newton / args.c2_frames, 2), "pcg_iters_per_newton": round(pcg / max(newton, 1), 2),
            "line_search_fail": fails, "contacts_max": contacts, "validator_penetrations": penetrations,
            "edge_triangle_crossings": crossings, "z_min": zmin,
            "timing": "CUDA events of each step (device_ms), positions stay on the device",
            "waves": "2 mm (the configured 2 cm waves on sheets 5 mm apart start the stack self-intersecting)"}


def heldout_run(args, local, flush, pg, weights):
    """The configured evaluation of the curtains: each held-out seed run for the full number of frames
    with the learned preconditioner (refresh as in the timed window), device-resident; per seed the
    frames/s, Newton and PCG counts, fallbacks, line-search failures, frames at the Newton cap, and
    every 30 frames the exact edge-triangle crossing count (untimed)."""
    import torch

    from andosim_b200 import abi, scenes

    out = []
    for seed in [int(q) for q in args.heldout_seeds.split(",") if q.strip()]:
        sc = scenes.c4(seed=seed, n=args.n, frames=args.heldout_frames)
        S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
        S.set_precond_weights(weights)
        p = abi.make_params(sc.params, semantics="corrected", precond="learned", precond_refresh=args.refresh)
        ms, newton, pcg, fb, fails, capped, crossings = 0.0, 0, 0, 0, 0, 0, 0
        for f in range(args.heldout_frames):
            S.apply_gravity(sc.gravity, p.dt)
            st = S.step(p, sc.pins_at(f), sc.walls)
            ms += st["device_ms"]; newton += st["newton_iters"]; pcg += st["pcg_iters"]
            fb += st["precond_fallbacks"]; fails += st["line_search_fail"]
            capped += int(st["newton_iters"] >= p.max_newton_steps * max(1, st["substeps"]))
            if f % 30 == 29:
                crossings += S.edge_triangle_crossings()
        S.close()
        ms = dist_max(ms, pg)
        out.append({"seed": seed, "frames": args.heldout_frames, "frames_per_s": round(args.heldout_frames / (ms * 1e-3), 2),
                    "newton_iters_per_frame": round(newton / args.heldout_frames, 2),
                    "pcg_iters_per_newton": round(pcg / max(newton, 1), 2), "precond_fallbacks": fb,
                    "line_search_fail": fails, "frames_at_newton_cap": capped, "edge_triangle_crossings": crossings})
    return {"workload": f"c4_curtains_2x{args.n}x{args.n}", "preconditioner": "learned", "precond_refresh": args.refresh, "seeds": out,
            "timing": "step device time (CUDA events inside ando_step), L2 not flushed, crossings checked every 30 frames"}


def c5_run(args, local, pg, seed=0):
    """The tablecloth (n x n over a 3 m square) draped over the 12-triangle box (density 1e6, static in
    effect) on the ground, one edge row pulled at 1 m/s after frame 60: CORRECTED with block Jacobi
    through the module API, device-resident. Reported as measured: frames/s, Newton and PCG counts,
    frames that end at the Newton cap (the strain-limit limitation of the pull), line-search
    failures, and every 40 frames the exact edge-triangle crossing count, the validator's
    penetrations on the CORRECTED contact set and the lowest vertex above the ground."""
    from andosim_b200 import ando_barrier_core as abc, scenes

    sc = scenes.c5(seed=seed, n=args.c5_n, frames=args.c5_frames)
    abc.set_device(local)
    m = abc.Mesh()
    m.initialize(sc.vertices, sc.triangles, abc.Material(**sc.material))
    st = abc.State()
    st.initialize(m)
    p = abc.SimParams()
    for k, v in sc.params.items():
        setattr(p, k, v)
    p.semantics = "corrected"
    box = abc.RigidBody()
    rg = sc.rigids[0]
    box.initialize(rg.vertices, rg.triangles, rg.density)
    ms, newton, pcg, fails, capped, crossings, penetrations, zmin, contacts = 0.0, 0, 0, 0, 0, 0, 0, 1e9, 0
    for f in range(args.c5_frames):
        c = abc.Constraints()
        for i, t in sc.pins_at(f):
            c.add_pin(int(i), t)
        for n, o, g in sc.walls:
            c.add_wall(n, o, g)
        st.apply_gravity(sc.gravity, p.dt)
        abc.Integrator.step(m, st, c, p, [box])
        s_ = abc.Integrator.last_step_stats(st)
        ms += s_["device_ms"]; newton += s_["newton_iters"]; pcg += s_["pcg_iters"]; fails += s_["line_search_fail"]
        contacts = max(contacts, s_["contacts"])
        capped += int(s_["newton_iters"] >= p.max_newton_steps * max(1, s_["substeps"]))
        if f % 40 == 39 or f == args.c5_frames - 1:
            cs = abc.Integrator.compute_contacts(m, st, [box], "corrected", float(p.contact_gap_max))
            met = abc.CollisionValidator.compute_metrics(m, st, cs, float(p.contact_gap_max), True)
            penetrations += int(met.num_penetrations)
            crossings += int(abc.CollisionValidator.edge_triangle_crossings(m, st))
            zmin = min(zmin, float(st.get_positions64()[:, 2].min()))
    ms = dist_max(ms, pg)
    return {"workload": f"c5_tablecloth_{args.c5_n}x{args.c5_n}_box", "vertices": sc.num_vertices, "frames": args.c5_frames,
            "semantics": "CORRECTED", "preconditioner": "block_jacobi", "frames_per_s": round(args.c5_frames / (ms * 1e-3), 2),
            "newton_iters_per_frame": round(newton / args.c5_frames, 2), "pcg_iters_per_newton": round(pcg / max(newton, 1), 2),
            "frames_at_newton_cap": capped, "line_search_fail": fails, "contacts_max": contacts,
            "validator_penetrations": penetrations, "edge_triangle_crossings": crossings, "z_min": zmin,
            "timing": "CUDA events of each step (device_ms), positions stay on the device"}


def run_ours(args, rank, world, local, pg):
    import torch

    from andosim_b200 import learned, scenes
    from andosim_b200.build import build

    if rank == 0:
        build()
    barrier(pg)
    torch.cuda.set_device(local)
    scs = [scenes.c4(seed=rank + world * k, n=args.n) for k in range(max(args.seeds, 1))]
    sc = scs[0]
    V, T = sc.num_vertices, sc.num_triangles
    weights = learned.load_weights(Path(args.weights) if args.weights else None)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = ClockSampler(local)
    clocks.start()
    # the paired window over several seeds of the workload: one trajectory's
    # iteration counts depend on which hard Newton systems its frames contain
    res, diffs, nframes, crossings = None, [], 0, []
    for sck in scs:
        r, d, n, cr = paired_run(args, sck, local, flush, pg, weights, raw=True)
        crossings.append(cr)
        if res is None:
            res = r
        else:
            for name in res:
                res[name]["ms"] += r[name]["ms"]
                res[name]["stats"] += r[name]["stats"]
                res[name]["launches"] += r[name]["launches"]
        diffs += d
        nframes += n
    pair = summarize_pair(args, res, diffs, nframes, pg)
    clock_info = clocks.stop()
    lrn, jac = pair["learned"], pair["block_jacobi"]
    # phase breakdown and rooflines: a separate profiled pass (per-phase CUDA events)
    lp = corrected_run(args, sc, local, flush, pg, "learned", weights, profile=True, frames=args.steps)
    full = None
    if args.full_n > 0:
        scf = scenes.c4(seed=rank, n=args.full_n)
        pf = paired_run(args, scf, local, flush, pg, weights, steps=args.full_steps)
        full = {"workload": f"c4_curtains_2x{args.full_n}x{args.full_n}", "frames": args.full_steps,
                "learned": {k: v for k, v in pf["learned"].items() if k != "total_ms"},
                "jacobi": {k: v for k, v in pf["block_jacobi"].items() if k != "total_ms"},
                "frames_per_s_ratio": round(pf["learned"]["frames_per_s"] / pf["block_jacobi"]["frames_per_s"], 3),
                "pcg_iters_per_newton_ratio": round(pf["learned"]["pcg_iters_per_newton"] / max(pf["block_jacobi"]["pcg_iters_per_newton"], 1e-9), 3),
                "step_position_diff_rel_extent": pf["step_position_diff_rel_extent"],
                "edge_triangle_crossings_end": pf["edge_triangle_crossings_end"]}
    prof, nnzb = lp.pop("_prof"), lp.pop("_nnzb")
    peaks = json.loads(PEAKS_FILE.read_text()) if PEAKS_FILE.exists() else {}
    hbm = float(peaks.get("hbm_gbs", FALLBACK_HBM_GBS))
    source = "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks else "fallback"
    pcg_ms = prof["phase_ms"]["pcg"]
    launches = max(1, prof["phase_launches"]["pcg"])
    pb = pcg_bytes(V, nnzb, prof)
    roof = None
    if pcg_ms > 0:
        achieved = pb / (pcg_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": "k_pcg_scaled (learned and block-Jacobi launches)", "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": PCG_TRAFFIC,
                "peak_source": source, "bytes_per_launch": int(pb // launches),
                "launches": int(launches), "avg_launch_us": round(pcg_ms * 1e3 / launches, 2),
                "pcg_iterations": int(prof["pcg_iterations"]), "share_of_frame": round(pcg_ms / max(sum(prof["phase_ms"].values()), 1e-9), 3)}
    asm_ms = prof["phase_ms"]["assemble"]
    asm_n = max(1, prof["newton_iterations"])
    roof_asm = None
    if asm_ms > 0:
        ab = assembly_bytes(V, nnzb) * asm_n
        achieved = ab / (asm_ms * 1e-3) / 1e9
        roof_asm = {"bound": "hbm", "kernel": "k_diag_factor + k_assemble_scaled_slice (+ k_extra_merge)", "achieved": round(achieved, 1),
                    "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": ASSEMBLY_TRAFFIC, "peak_source": source,
                    "bytes_per_newton_iteration": int(assembly_bytes(V, nnzb)), "newton_iterations": int(asm_n),
                    "avg_us_per_newton_iteration": round(asm_ms * 1e3 / asm_n, 2)}
    ms_l = lrn.pop("total_ms")
    jac.pop("total_ms")
    out = {
        "metric": METRIC, "value": round(nframes * world / (ms_l * 1e-3), 2), "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_l / nframes, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 BSR/PCG vectors, f64 positions/gradient/dots",
        "data": "synthetic (seeded curtains, scenes.c4)",
        "config": {"workload": WORKLOAD, "vertices": V, "triangles": T, "bsr_blocks": nnzb, "semantics": "CORRECTED",
                   "preconditioner": "learned", "precond_refresh": args.refresh, "pcg_tol": sc.params["pcg_tol"],
                   "frames_timed_per_gpu": nframes,
                   "frames": f"{args.warmup}-{args.warmup + args.steps - 1} of seeds " + ",".join(str(rank + world * k) for k in range(len(scs))),
                   "l2": "flushed before every timed frame", "parallelism": f"replicas x{world}"},
        "pcg_iters_per_newton": lrn["pcg_iters_per_newton"],
        "newton_iters_per_frame": lrn["newton_iters_per_frame"],
        "newton_iters_per_s": round(lrn["newton_iters_per_s"] * world, 1),
        "learned": lrn, "jacobi": jac,
        "learned_vs_jacobi": {"frames_per_s_ratio": round(lrn["frames_per_s"] / jac["frames_per_s"], 3),
                              "pcg_iters_per_newton_ratio": round(lrn["pcg_iters_per_newton"] / max(jac["pcg_iters_per_newton"], 1e-9), 3),
                              "paired": "each frame both preconditioners step from the same state",
                              "step_position_diff_rel_extent": pair["step_position_diff_rel_extent"]},
        "edge_triangle_crossings": {"end_of_window_per_seed": crossings,
                                    "check": "mesh edges through a triangle they share no vertex with, exact FP64 test on the GPU "
                                             "(ando_edge_triangle_crossings), untimed"},
        "profiled_pass": lp,
        "full_length": full,
        "gpu_launches": lrn["gpu_launches"],
        "roofline": roof,
        "roofline_assembly": roof_asm,
        "clocks": clock_info,
    }
    if args.reference_steps > 0:
        out["reference_semantics"] = reference_semantics_run(args, sc, local, flush, pg)
    out["e2e"] = e2e_run(args, scs, local, flush, pg, weights)
    if args.c3_frames > 0:
        out["c3_batched"] = c3_run(args, local, seed=rank)
    if args.c2_frames > 0:
        out["c2_stack"] = c2_run(args, local, pg, seed=rank)
    if args.c5_frames > 0:
        out["c5_tablecloth"] = c5_run(args, local, pg, seed=rank)
    if args.heldout_frames > 0 and args.heldout_seeds:
        out["heldout_full_length"] = heldout_run(args, local, flush, pg, weights)
    return out, sc, weights


# ----------------------------------------------------------- CPU baseline
def oracle_state(O, sc, x, v):
    """Oracle objects for scene `sc` at positions x and velocities v (FP64 arrays)."""
    m = O.Mesh()
    m.initialize(sc.vertices, sc.triangles, O.Material(**sc.material))
    s = O.State()
    s.initialize(m)
    s.set_positions(x)
    s.set_velocities(v)
    p = O.SimParams()
    for k, val in sc.params.items():
        setattr(p, k, val)
    return m, s, p


def oracle_step(O, sc, m, s, p, frame):
    c = O.Constraints()
    for i, t in sc.pins_at(frame):
        c.add_pin(int(i), t)
    for n, o, g in sc.walls:
        c.add_wall(n, o, g)
    s.apply_gravity(sc.gravity, p.dt)
    t0 = time.perf_counter()
    st = O.Integrator.step(m, s, c, p, None, "indexed", "literal", "corrected")
    return time.perf_counter() - t0, st


def cpu_baseline(args, sc, local, weights):
    """CPU baseline and per-frame FP64 error, from the GPU's own state at the first timed frame.

    The GPU runs frames 0..W-1 (learned), then steps frame W from that state with each preconditioner;
    the oracle steps the same frame from the same state in FP32 (timed: the reference's default
    Real = float build, CORRECTED semantics, block-Jacobi PCG) and in FP64 (the all-FP64 reference
    run the position error is quoted against)."""
    from andosim_b200 import abi
    from oracle.build import load

    ora = load()
    S = abi.Scene(sc.vertices, sc.triangles, sc.material, device=local)
    S.set_precond_weights(weights)
    pl = abi.make_params(sc.params, semantics="corrected", precond="learned", precond_refresh=args.refresh)
    pj = abi.make_params(sc.params, semantics="corrected", precond="block_jacobi")
    W = args.warmup
    for f in range(W):
        S.apply_gravity(sc.gravity, pl.dt)
        S.step(pl, sc.pins_at(f), sc.walls)
    x0, v0 = S.download()
    gpu = {}
    for name, p in (("learned", pl), ("block_jacobi", pj)):
        S.upload(x0, v0)
        S.apply_gravity(sc.gravity, p.dt)
        S.step(p, sc.pins_at(W), sc.walls)
        gpu[name] = S.download()[0]
    S.close()
    m, s, p = oracle_state(ora.f64, sc, x0, v0)
    sec64, _ = oracle_step(ora.f64, sc, m, s, p, W)
    x64 = np.asarray(s.get_positions(), dtype=np.float64)
    m, s, p = oracle_state(ora.f32, sc, x0, v0)
    sec32, st32 = oracle_step(ora.f32, sc, m, s, p, W)
    ext = float(np.ptp(sc.vertices, axis=0).max())
    threads = int(os.environ.get("ANDO_ORACLE_THREADS", "0")) or (os.cpu_count() or 1)
    base = {"value": round(1.0 / sec32, 4), "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"frame {W} of seed 0 of {WORKLOAD} ({sc.num_vertices} vertices; the first timed frame), stepped by the "
                      f"FP32 oracle (C++ restatement of the reference, CORRECTED semantics, block-Jacobi PCG) from the GPU's "
                      f"own state at that frame; sparse products, PCG vector updates, broad-phase queries and "
                      f"time-of-impact pairs on {threads} threads, the rest on one",
            "newton_iters": int(st32["newton_iters"]), "substeps": int(st32["substeps"])}
    err = {"frame": W, "seed": 0, "unit": "max |x_gpu - x_fp64| / extent, one step from the same state",
           "learned": float(np.abs(gpu["learned"] - x64).max() / ext),
           "block_jacobi": float(np.abs(gpu["block_jacobi"] - x64).max() / ext), "fp64_oracle_seconds": round(sec64, 2)}
    return base, err


def run_reference(args, rank, world, pg):
    """The reference's CPU path on the same workload and semantics: the oracle (a C++ restatement of the
    reference; the reference itself does not build here) stepping the curtain workload in CORRECTED
    semantics with block-Jacobi PCG, seed 0, frames 0..W-1 untimed and frames W.. timed until K frames
    or the time budget (--reference-budget) is reached; `steps` is the number of frames actually timed.
    Rank 0 only; the other ranks do no work."""
    if rank != 0:
        return None
    from andosim_b200 import scenes
    from oracle.build import load

    O = load().f32
    sc = scenes.c4(seed=0, n=args.n)
    m, s, p = oracle_state(O, sc, sc.vertices, np.zeros_like(sc.vertices))
    for f in range(args.warmup):
        oracle_step(O, sc, m, s, p, f)
    secs, frames, newton = 0.0, 0, 0
    while frames < args.steps and (frames == 0 or secs < args.reference_budget):
        dt, st = oracle_step(O, sc, m, s, p, args.warmup + frames)
        secs += dt
        frames += 1
        newton += st["newton_iters"]
    threads = int(os.environ.get("ANDO_ORACLE_THREADS", "0")) or (os.cpu_count() or 1)
    value = round(frames / secs, 4)
    sample = (f"frames {args.warmup}-{args.warmup + frames - 1} of seed 0 of {WORKLOAD} ({frames} of the {args.steps} asked "
              f"for fit the {args.reference_budget:.0f} s budget), FP32 oracle, CORRECTED semantics, block-Jacobi PCG; "
              f"sparse products, PCG updates, queries and time-of-impact pairs on {threads} threads")
    base = {"value": value, "unit": "frames/s", "cores": threads, "kind": "port", "sample": sample}
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": frames, "warmup": args.warmup, "ms_per_step": round(secs * 1e3 / frames, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded curtains, scenes.c4)",
            "config": {"workload": WORKLOAD, "vertices": sc.num_vertices, "semantics": "CORRECTED", "preconditioner": "block_jacobi",
                       "frames": f"{args.warmup}-{args.warmup + frames - 1} of seed 0", "newton_iters_per_frame": round(newton / frames, 2)},
            "cpu_baseline": base, "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            out = run_reference(args, rank, world, pg)
        else:
            out, sc, weights = run_ours(args, rank, world, local, pg)
            if rank == 0 and world == 1 and not args.no_cpu_baseline:
                out["cpu_baseline"], out["fp64_step_error"] = cpu_baseline(args, sc, local, weights)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if pg:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
