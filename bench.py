"""Throughput benchmark of the B200 rigid-body step.

python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl b3|reference]

Prints one JSON line (rank 0). `value` is whole-job body-steps/s with the
scene resident in HBM, timed with CUDA events over K graph-replayed steps
(max over ranks). `e2e` is the same metric through the C ABI with the body
state uploaded from pinned host memory and positions/orientations read
back every step. The per-kernel roofline uses live CUDA-event stage times.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c1": "Plain step, 4,096 unit cubes over a 200x200x1 m ground box (configs[0])",
    "c2": "Plain step, 131,072 mixed hulls: 1/2 cubes, 1/4 12-point hulls, 1/4 42-vertex icospheres (configs[1])",
    "c3": "Batched step, 4,096 worlds of log-uniform[8,512] cubes/12-point hulls (configs[2])",
    "c5": "Plain step, 1,048,576 unit cubes (configs[4] forward)",
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def make_scene(name):
    from experiments_b200 import scenes
    return {"c1": scenes.c1, "c2": scenes.c2, "c3": scenes.c3, "c5": scenes.c5}[name]()


def stage_bytes(scene_n, counters, key_bits, body_bits, iters):
    """Algorithmic HBM bytes per launch of each stage (compulsory traffic,
    each intermediate written once and read once)."""
    N = scene_n
    P = counters["numPairs"]
    C = counters["numManifolds"]
    S = 8 * (2 * math.ceil(key_bits / 8) + 1)
    S2 = 8 * (2 * math.ceil(body_bits / 8) + 1)
    return {
        "aabb_hash": N * (64 + 8 + 32 + 8),            # pos+quat read, vel rw (dyn), aabb write, key/val write
        "sort_cells": N * (S + 12),
        "find_pairs": N * (8 + 32) + P * (8 + 32),      # sorted key/val + own AABB, pair write + other AABB
        "narrowphase": P * (8 + 64) + C * 96,           # pair + two poses, manifold write
        "manifolds": P * 8 + C * (96 + 16) + 2 * C * S2,
        "solve": C * (96 + 640) + iters * (C * 2 * 576 + N * 4 * 64),
        "integrate": N * (64 + 64 + 32),
    }


STAGES = ["aabb_hash", "sort_cells", "find_pairs", "narrowphase", "manifolds", "solve", "integrate"]


def run_b3(args, rank, world_size, local_rank):
    import torch
    from experiments_b200 import b3, scenes
    torch.cuda.set_device(local_rank)
    ctx = b3.Context(local_rank)
    sc = make_scene(args.workload)
    w = scenes.build_world(ctx, sc, useGraph=1)
    st = torch.cuda.current_stream()
    stream = st.cuda_stream
    for _ in range(args.warmup):
        w.stepSimulation(1, stream=stream)
    torch.cuda.synchronize()
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        e0.record(st)
        w.stepSimulation(args.steps, stream=stream)
        e1.record(st)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world_size > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    counters = w.counters()
    # stage breakdown: extra untimed steps with per-stage CUDA events
    w2 = scenes.build_world(ctx, sc, useGraph=0)
    for _ in range(args.warmup):
        w2.stepSimulation(1)
    w2.set_stage_timing(True)
    acc = np.zeros(len(STAGES))
    reps = 3
    for _ in range(reps):
        w2.stepSimulation(1)
        acc += np.array(w2.stage_times()[:len(STAGES)])
    stage_ms = acc / reps
    c2 = w2.counters()
    w2.close()
    # e2e: through the C ABI with host buffers every step
    n = sc.n
    pos, quat, lin, ang = w.read_state()
    hp = torch.from_numpy(pos).pin_memory().numpy()
    hq = torch.from_numpy(quat).pin_memory().numpy()
    hl = torch.from_numpy(lin).pin_memory().numpy()
    ha = torch.from_numpy(ang).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 20))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(st)
    for _ in range(e2e_steps):
        w.write_state(hp, hq, hl, ha, stream=stream)
        w.stepSimulation(1, stream=stream)
        p_, q_, l_, a_ = w.read_state(stream=stream)
        hp[:], hq[:], hl[:], ha[:] = p_, q_, l_, a_
    e3.record(st)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3) / e2e_steps
    wall_e2e = (time.perf_counter() - t0) / e2e_steps * 1e3
    e2e_ms = max(e2e_ms, wall_e2e)
    return dict(sc=sc, ms=ms, counters=counters, stage_ms=stage_ms, c2=c2, clocks=clk.summary(),
                e2e_ms=e2e_ms, w=w, n=n)


def cpu_baseline_port(sc_name, budget_s=15.0):
    """The oracle (single-threaded port) on a bounded sample of the workload."""
    import oracle
    from experiments_b200 import b3, scenes
    sc = make_scene(sc_name)
    hc = b3.Context(-1)
    w = b3.PhysicsWorld(hc, scenes.world_config(sc))
    scenes.register_scene(w, sc)
    o = oracle.oracle_from_world(w, sc)
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < budget_s and steps < 1000:
        o.step(1)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": sc.n * steps / dt, "unit": "body-steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} steps of the full {sc.n}-body scene in {dt:.1f} s, 1 thread"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b3", choices=["b3", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    args.warmup = max(3, args.warmup)

    if args.impl == "reference":
        if rank != 0:
            return
        r = cpu_baseline_port(args.workload, budget_s=max(10.0, min(60.0, args.steps * 2.0)))
        line = {"metric": "body-steps/s", "value": r["value"], "unit": "body-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "impl": "reference", "config": {"workload": WORKLOADS[args.workload]},
                "cpu_baseline": r, "e2e": {"value": r["value"], "unit": "body-steps/s",
                                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world_size > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = run_b3(args, rank, world_size, local_rank)
    sc = res["sc"]
    ms_per_step = res["ms"] / args.steps
    value = sc.n * args.steps * world_size / (res["ms"] / 1e3)
    peak, peak_kind = peaks()
    from experiments_b200 import b3 as _b3  # noqa: F401
    w = res["w"]
    key_bits = w.cfg.gridDims[0].bit_length() - 1 + w.cfg.gridDims[1].bit_length() - 1 + \
        w.cfg.gridDims[2].bit_length() - 1 + (max(1, sc.num_worlds - 1).bit_length() if sc.num_worlds > 1 else 0)
    body_bits = max(1, int(sc.n).bit_length())
    sb = stage_bytes(sc.n, res["c2"], key_bits, body_bits, 10)
    sm = dict(zip(STAGES, res["stage_ms"].tolist()))
    dom = max(sm, key=lambda k: sm[k])
    achieved = sb[dom] / (sm[dom] / 1e3) / 1e9
    passes = math.ceil(key_bits / 8)
    passes2 = math.ceil(body_bits / 8)
    launches = 1 + 1 + (1 + passes) + 1 + 1 + 1 + 2 + 1 + (1 + passes2) + 1 + 1 + 1 + 1
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload], "bodies": sc.n, "worlds": sc.num_worlds,
                   "pairs": res["counters"]["numPairs"], "manifolds": res["counters"]["numManifolds"],
                   "contact_points": res["counters"]["numContactPoints"], "iterations": 10,
                   "refined_axes": res["counters"].get("refinedAxes"),
                   "refined_clips": res["counters"].get("refinedClips"),
                   "parallelism": "replicas" if world_size > 1 else "single",
                   "l2": "working set exceeds L2" if sc.n > 100000 else "working set L2-resident; no flush"},
        "contacts_per_s": res["counters"]["numContactPoints"] * args.steps * world_size / (res["ms"] / 1e3),
        "stage_ms": sm,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind},
        "clocks": res["clocks"],
        "e2e": {"value": sc.n / (res["e2e_ms"] / 1e3) * world_size, "unit": "body-steps/s",
                "h2d_bytes_per_step": 64 * sc.n, "d2h_bytes_per_step": 64 * sc.n},
        "gpu_launches": launches * args.steps,
    }
    if rank == 0 and not args.no_cpu_baseline and world_size == 1:
        line["cpu_baseline"] = cpu_baseline_port(args.workload)
    if rank == 0:
        print(json.dumps(line))
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
