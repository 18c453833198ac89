"""Kernel timeline of a few CORRECTED frames of the two-curtain workload.

    python -m andosim_b200.trace_frames [--n 256] [--warmup 4] [--frames 2]
        [--precond learned|block_jacobi] [--out trace.json]

Runs the frames under torch.profiler (CUPTI kernel and CUDA runtime activity,
warm caches, no serialisation), writes the Chrome trace and prints a summary:
the span of the traced frames, the time some kernel was running (kernels on
two streams overlap, so their summed durations can exceed it), the idle gaps
between kernels, the runtime calls and the per-kernel totals.
"""
from __future__ import annotations

import argparse
import collections
import json

from . import abi, learned, scenes


def summarise(trace: dict) -> dict:
    ev = trace["traceEvents"] if isinstance(trace, dict) else trace
    gpu = sorted((e for e in ev if e.get("cat") in ("kernel", "gpu_memcpy", "gpu_memset") and "dur" in e), key=lambda e: e["ts"])
    if not gpu:
        return {}
    t0, end, busy, idle = gpu[0]["ts"], gpu[0]["ts"], 0.0, 0.0
    for e in gpu:
        if e["ts"] > end:
            idle += e["ts"] - end
        busy += e["dur"]
        end = max(end, e["ts"] + e["dur"])
    per = collections.defaultdict(lambda: [0, 0.0])
    for e in gpu:
        name = e["name"].replace("ando::(anonymous namespace)::", "").replace("void ", "")
        name = name.split("<")[0] if name.startswith("cub::") else name.split("(")[0]
        per[name][0] += 1
        per[name][1] += e["dur"]
    api = collections.defaultdict(lambda: [0, 0.0])
    for e in ev:
        if e.get("cat") == "cuda_runtime" and "dur" in e:
            api[e["name"]][0] += 1
            api[e["name"]][1] += e["dur"]
    top = sorted(per.items(), key=lambda kv: -kv[1][1])
    return {"span_us": round(end - t0, 1), "gpu_busy_us": round(end - t0 - idle, 1), "kernel_sum_us": round(busy, 1),
            "idle_us": round(idle, 1),
            "kernels": [{"name": k, "launches": v[0], "total_us": round(v[1], 1), "avg_us": round(v[1] / v[0], 1)} for k, v in top],
            "runtime_calls": {k: {"calls": v[0], "total_us": round(v[1], 1)} for k, v in sorted(api.items(), key=lambda kv: -kv[1][1])}}


def main(argv=None):
    import torch
    from torch.profiler import ProfilerActivity, profile

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--frames", type=int, default=2)
    ap.add_argument("--precond", default="learned", choices=["learned", "block_jacobi"])
    ap.add_argument("--out", default="trace.json")
    a = ap.parse_args(argv)
    sc = scenes.c4(n=a.n)
    S = abi.Scene(sc.vertices, sc.triangles, sc.material)
    S.set_precond_weights(learned.load_weights())
    p = abi.make_params(sc.params, semantics="corrected", precond=a.precond)
    for f in range(a.warmup):
        S.apply_gravity(sc.gravity, p.dt)
        S.step(p, sc.pins_at(f), sc.walls)
    torch.cuda.synchronize()
    stats = []
    with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
        for f in range(a.warmup, a.warmup + a.frames):
            S.apply_gravity(sc.gravity, p.dt)
            stats.append(S.step(p, sc.pins_at(f), sc.walls))
        torch.cuda.synchronize()
    S.close()
    prof.export_chrome_trace(a.out)
    with open(a.out) as fh:
        summary = summarise(json.load(fh))
    summary["frames"] = [{k: st[k] for k in ("newton_iters", "pcg_iters", "contacts", "substeps", "device_ms")} for st in stats]
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main()
