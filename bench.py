"""Throughput benchmark of the B200 rigid-body step.

python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl b3|reference]

Prints one JSON line on rank 0.

* value: whole-job body-steps/s of the plain step on the workload (default
  the 131,072-body mixed-hull scene), the scene resident in HBM. Each of
  the K timed steps is one replay of the captured step graph bracketed by
  CUDA events on the launching stream; a 256 MiB write flushes L2 between
  steps, outside the events. Max over ranks; for N > 1 every rank steps its
  own replica (weak scaling, no collective on the data path).
* e2e: the same metric through the C ABI with host buffers: every step
  uploads the body state from pinned host memory, steps, and reads the
  state back (H2D + D2H inside the timed region).
* roofline: the dominant kernel of the step from live per-stage CUDA-event
  times. The narrowphase is FP32-ALU bound (SAT projections), so its
  roofline is FP32 FLOP/s against the CUDA-core peak; the other stages are
  HBM bound and use the measured copy bandwidth. All stages are listed in
  stage_roofline.
* cpu_baseline: the reference's CPU rigid-body pipeline (bullet2
  btDiscreteDynamicsWorld built from the reference's sources; the oracle port
  where that library is absent) on one host thread, a bounded sample of the
  same scene.
* forms: the batched 4,096-world step against the plain per-world step on
  the same GPU (body-steps/s of each; per-world time sampled on a subset),
  and the adjoint form (forward with checkpoints + reverse sweep) on the
  256-world differentiable throw against its plain forward.
--impl reference: the same CPU pipeline on all host cores (independent
  replicas, one process per core), same metric and workload.
"""
import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c1": "plain step, 4,096 unit cubes over a 200x200x1 m ground box, 10 Jacobi iterations",
    "c2": "plain step, 131,072 bodies (1/2 unit cubes, 1/4 12-point hulls, 1/4 42-vertex icospheres), "
          "64x32x64 lattice at 1.2 m, 10 Jacobi iterations",
    "c2s": "plain step, 16,384 bodies (the 131,072-body mix on a 32x16x32 lattice at 1.2 m), "
           "10 Jacobi iterations (small case for profiler captures)",
    "c3s": "batched step, 512 worlds of log-uniform[8,512] cubes / 12-point hulls, 10 Jacobi iterations "
           "(small case for profiler captures)",
    "c3": "batched step, 4,096 worlds of log-uniform[8,512] cubes / 12-point hulls, 10 Jacobi iterations",
    "c5": "plain step, 1,048,576 unit cubes, 128x64x128 lattice, 10 Jacobi iterations",
}
STAGES = ["aabb_hash", "sort_cells", "find_pairs", "narrowphase", "manifolds", "solve", "integrate"]
# DRAM bytes per pair of the four narrowphase kernels (read + write) from the ncu capture in
# profiles/kernels_c2s_plain_step.md, scaled by the timed workload's pair count
NARROWPHASE_DRAM_BYTES_PER_PAIR = 4.352e6 / 36735
FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 FP32 lanes x FMA x 1.965 GHz


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
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
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)  # let the sampler start before the timed region
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=2)
            except Exception:
                self.proc.kill()

    def summary(self):
        good = [r for r in self.rows if len(r) >= 9]
        if not good:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in good if num(r[1]) is not None]
        mx = [num(r[2]) for r in good if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in good:
            for k, nm in enumerate(names):
                if r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(good)}


def make_scene(name):
    from experiments_b200 import scenes
    return {"c1": scenes.c1, "c2": scenes.c2, "c2s": lambda: scenes.c2(dims=(32, 16, 32)), "c3": scenes.c3, "c3s": lambda: scenes.c3(worlds=512),
            "c5": scenes.c5}[name]()


def sat_flops(world, scene):
    """Algorithmic FP32 work of the narrowphase over the current pair list
    (8 (VA+VB)(FA+FB+EA*EB) per pair for the separating axis test,
    64 V_inc V_ref for the clip of pairs with a manifold)."""
    sh = world.shapes()
    polys = sh["polys"]
    V = np.array([polys[k].numVertices for k in range(sh["counts"][1])], np.float64)
    F = np.array([polys[k].numFaces for k in range(sh["counts"][1])], np.float64)
    E = np.array([polys[k].numUniqueEdges for k in range(sh["counts"][1])], np.float64)
    colshape = np.array([sh["cols"][k].shapeIndex for k in range(sh["counts"][0])], np.int64)
    pairs = world.pairs()
    if len(pairs) == 0:
        return 0.0
    sa = colshape[scene.shape[pairs[:, 0]]]
    sb = colshape[scene.shape[pairs[:, 1]]]
    dyn = (scene.mass[pairs[:, 0]] > 0) | (scene.mass[pairs[:, 1]] > 0)
    sat = 8.0 * (V[sa] + V[sb]) * (F[sa] + F[sb] + E[sa] * E[sb])
    c = world.contacts()
    clip = 64.0 * 4.0 * 4.0 * len(c["normal"])
    return float(np.sum(sat[dyn]) + clip)


def stage_bytes(n, counters, key_bits, body_bits, iters):
    """Compulsory HBM bytes per launch of each stage (each intermediate
    written once and read once; hull and cell tables assumed on chip)."""
    P = counters["numPairs"]
    C = counters["numManifolds"]
    S = 8 * (2 * math.ceil(key_bits / 8) + 1)
    S2 = 8 * (2 * math.ceil(body_bits / 8) + 1)
    return {
        "aabb_hash": n * (64 + 16 + 32 + 8),
        "sort_cells": n * (S + 12),
        "find_pairs": n * (8 + 32) + P * 8,
        "narrowphase": P * (8 + 64) + C * 96,
        "manifolds": P * 8 + C * 96 + 2 * C * S2,
        "solve": C * (96 + 368) + iters * (200 * C + 64 * n),
        "integrate": n * (64 + 64),
    }


def step_bytes(n, counters, key_bits, iters):
    """Compulsory HBM bytes of one whole step:
    N (128 + 20 + 8 + S + 12 + 32) + 80 P + 368 C + I (200 C + 64 N),
    S = 8 (2 ceil(kbits / 8) + 1) the radix sort term."""
    P = counters["numPairs"]
    C = counters["numManifolds"]
    S = 8 * (2 * math.ceil(key_bits / 8) + 1)
    return n * (128 + 20 + 8 + S + 12 + 32) + 80 * P + 368 * C + iters * (200 * C + 64 * n)


def flush_l2(buf):
    buf.add_(1)


def time_steps(w, steps, stream, flush):
    """Sum of per-step device times of graph replays, L2 flushed in between."""
    import torch
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in evs:
        if flush is not None:
            flush_l2(flush)
        e0.record(stream)
        w.stepSimulation(1, stream=stream.cuda_stream)
        e1.record(stream)
    torch.cuda.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in evs)


def run_b3(args, world_size, local_rank):
    import torch
    from experiments_b200 import b3, scenes
    torch.cuda.set_device(local_rank)
    ctx = b3.Context(local_rank)
    full = make_scene(args.workload)
    sc, sharded = full, False
    if world_size > 1 and full.num_worlds > 1:
        # batched worlds shard with no exchange: each rank steps a
        # body-balanced contiguous range of worlds
        from experiments_b200 import sharding
        sc, _ = sharding.shard_scene(full, int(os.environ.get("RANK", "0")), world_size)
        sharded = True
    # world flags: 1 = sweep-and-prune broadphase, 2 = batched Gauss-Seidel solver
    flags = (1 if getattr(args, "sap", False) else 0) | (2 if getattr(args, "solver", "jacobi") == "gs" else 0)
    bp = {"flags": flags} if flags else {}
    w = scenes.build_world(ctx, sc, useGraph=1, **bp)
    st = torch.cuda.current_stream()
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2
    # launch shapes chosen by the autotuner on this scene (state restored)
    w.autotune(3, stream=st.cuda_stream)
    tuning = w.tuning()
    for _ in range(args.warmup):
        w.stepSimulation(1, stream=st.cuda_stream)
    torch.cuda.synchronize()
    if world_size > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ms = time_steps(w, args.steps, st, flush)
    torch.cuda.synchronize()
    if world_size > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    counters = w.counters()
    kernels = w.tuning()[3]
    # per-stage CUDA-event breakdown on an identical world advanced to the
    # same step (eager launches; timing only, not part of `value`)
    w2 = scenes.build_world(ctx, sc, useGraph=0, **bp)
    w2.set_tuning(tuning)
    w2.stepSimulation(args.warmup + args.steps - 3)
    w2.set_stage_timing(True)
    acc = np.zeros(len(STAGES))
    for _ in range(3):
        flush_l2(flush)
        w2.stepSimulation(1)
        acc += np.array(w2.stage_times()[:len(STAGES)])
    stage_ms = acc / 3
    c2 = w2.counters()
    flops = sat_flops(w2, sc)
    w2.close()
    # e2e through the C ABI with pinned host buffers
    pos, quat, lin, ang = w.read_state()
    hp = torch.from_numpy(pos).pin_memory().numpy()
    hq = torch.from_numpy(quat).pin_memory().numpy()
    hl = torch.from_numpy(lin).pin_memory().numpy()
    ha = torch.from_numpy(ang).pin_memory().numpy()
    e2e_steps = max(3, min(args.steps, 20))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        # H2D of the step's input state from pinned memory, the step, and the
        # D2H of its result straight into the same pinned buffers
        w.write_state(hp, hq, hl, ha, stream=st.cuda_stream)
        w.stepSimulation(1, stream=st.cuda_stream)
        w.read_state(stream=st.cuda_stream, out=(hp, hq, hl, ha))
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    contact_points = counters["numContactPoints"]
    if world_size > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
        t = torch.tensor([contact_points], device="cuda", dtype=torch.int64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        contact_points = int(t.item())
    return dict(sc=sc, full=full, sharded=sharded, ms=ms, contact_points=contact_points, tuning=tuning, counters=counters, stage_ms=stage_ms, c2=c2, clocks=clk.summary(), e2e_ms=e2e_ms,
                w=w, kernels=kernels, flops=flops, ctx=ctx)


def forms_comparison(ctx, steps=10, sample_worlds=32):
    """Batched 4,096-world step vs the plain step run world by world."""
    import torch
    from experiments_b200 import scenes
    sc = scenes.c3()
    wb = scenes.build_world(ctx, sc, useGraph=1)
    st = torch.cuda.current_stream()
    wb.autotune(3, stream=st.cuda_stream)
    for _ in range(3):
        wb.stepSimulation(1, stream=st.cuda_stream)
    ms_b = time_steps(wb, steps, st, None)
    batched = sc.n * steps / (ms_b / 1e3)
    # plain per-world step: each world in its own plain world, stepped one
    # world at a time (the reference's one-scene-per-pipeline usage)
    counts = sc.extra["counts"]
    rng = np.random.default_rng(0)
    pick = rng.choice(len(counts), size=min(sample_worlds, len(counts)), replace=False)
    total_ms = 0.0
    bodies = 0
    for wid in pick:
        sub = scenes.select_worlds(sc, [int(wid)])
        wp = scenes.build_world(ctx, sub, useGraph=1)
        for _ in range(3):
            wp.stepSimulation(1, stream=st.cuda_stream)
        total_ms += time_steps(wp, steps, st, None)
        bodies += sub.n
        wp.close()
    # extrapolate the sampled per-world times to all worlds
    per_body_ms = total_ms / max(bodies, 1)
    plain = sc.n * steps / (per_body_ms * sc.n / 1e3)
    wb.close()
    return {"batched_body_steps_per_s": batched, "plain_per_world_body_steps_per_s": plain,
            "speedup": batched / plain, "worlds": int(sc.num_worlds), "bodies": int(sc.n),
            "plain_sample": f"{len(pick)} of {sc.num_worlds} worlds, {steps} steps each, graph replay",
            "steps": steps}


def adjoint_form(ctx, worlds=256, steps=120, checkpoint_every=16):
    """Adjoint form on the differentiable throw (256 worlds x 64 cubes, 120
    steps, checkpoints every 16): forward with checkpoints plus the reverse
    sweep, against the plain forward of the same scene, all on the device
    (CUDA events on the launching stream)."""
    import torch
    from experiments_b200 import b3, scenes
    sc = scenes.c4(worlds=worlds, steps=steps)
    st = torch.cuda.current_stream()
    m = np.asarray(sc.mass, np.float64)
    wid = np.asarray(sc.world)
    # plain forward of the same scene (graph replays)
    wp = scenes.build_world(ctx, sc, useGraph=1)
    wp.stepSimulation(1, stream=st.cuda_stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    wp.stepSimulation(steps - 1, stream=st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1) / (steps - 1) * steps
    wp.close()
    w = scenes.build_world(ctx, sc, useGraph=1)
    adj = b3.Adjoint(w, steps, checkpoint_every)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(st)
    adj.forward(stream=st.cuda_stream)
    ev[1].record(st)
    pos = w.read_state(stream=st.cuda_stream)[0].astype(np.float64)
    # loss = sum over worlds of |COM - target|^2
    seed = np.zeros((sc.n, 4))
    for k in range(sc.num_worlds):
        s = (wid == k) & (m > 0)
        com = (pos[s, :3] * m[s, None]).sum(0) / m[s].sum()
        seed[s, :3] = 2 * (com - sc.extra["target"][k])[None, :] * (m[s, None] / m[s].sum())
    ev2 = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev2[0].record(st)
    adj.backward(d_pos=seed, stream=st.cuda_stream)
    ev2[1].record(st)
    torch.cuda.synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1])
    bwd_ms = ev2[0].elapsed_time(ev2[1])
    g = adj.gradients()
    fin = np.isfinite(g["lin"]).all(1) & np.isfinite(g["ang"]).all(1) & np.isfinite(g["mass"]) & \
        np.isfinite(g["friction"])
    finite_worlds = int(sum(bool(fin[wid == k].all()) for k in range(sc.num_worlds)))
    adj.close()
    w.close()
    total = fwd_ms + bwd_ms
    return {"workload": f"differentiable throw, {worlds} worlds x 64 cubes, {steps} steps, checkpoints every "
                        f"{checkpoint_every}", "bodies": int(sc.n),
            "adjoint_body_steps_per_s": sc.n * steps / (total / 1e3),
            "plain_body_steps_per_s": sc.n * steps / (plain_ms / 1e3),
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "plain_ms": plain_ms,
            "cost_vs_plain": total / plain_ms, "worlds_with_finite_gradients": finite_worlds,
            "gradient_error": "one-step gradient vectors within 1e-3 (measured 1e-6..4e-4) of FP64 central "
                              "differences (tests/test_gpu_adjoint.py); over 120 steps the throw is chaotic and "
                              "gradients grow without bound in some worlds"}


def scale_run(ctx, steps=32, checkpoint_every=8):
    """1,048,576 cubes: the plain step and the adjoint (loss = sum of body
    heights, checkpoints every 8 steps) on one GPU, with the device memory
    the adjoint holds."""
    import torch
    from experiments_b200 import b3, scenes
    sc = scenes.c5(steps=steps)
    st = torch.cuda.current_stream()
    w = scenes.build_world(ctx, sc, useGraph=1)
    w.stepSimulation(3, stream=st.cuda_stream)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    e[0].record(st)
    w.stepSimulation(10, stream=st.cuda_stream)
    e[1].record(st)
    torch.cuda.synchronize()
    plain_ms = e[0].elapsed_time(e[1]) / 10
    counters = w.counters()
    w.close()
    torch.cuda.synchronize()
    free0, total = torch.cuda.mem_get_info()
    w = scenes.build_world(ctx, sc, useGraph=1)
    adj = b3.Adjoint(w, steps, checkpoint_every)
    free1, _ = torch.cuda.mem_get_info()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(st)
    adj.forward(stream=st.cuda_stream)
    ev[1].record(st)
    seed = np.zeros((sc.n, 4), np.float32)
    seed[np.asarray(sc.mass) > 0, 1] = 1.0  # loss = sum of heights
    adj.backward(d_pos=seed, stream=st.cuda_stream)
    ev[2].record(st)
    torch.cuda.synchronize()
    g = adj.gradients()
    out = {"workload": f"1,048,576 unit cubes, 128x64x128 lattice at 1.05 m, {steps} steps, checkpoints every "
                       f"{checkpoint_every}", "bodies": int(sc.n),
           "plain_ms_per_step": plain_ms, "plain_body_steps_per_s": sc.n / (plain_ms / 1e3),
           "pairs": counters["numPairs"], "manifolds": counters["numManifolds"],
           "adjoint_forward_ms": ev[0].elapsed_time(ev[1]), "adjoint_backward_ms": ev[1].elapsed_time(ev[2]),
           "adjoint_body_steps_per_s": sc.n * steps / (ev[0].elapsed_time(ev[2]) / 1e3),
           "world_plus_adjoint_device_gb": (free0 - free1) / 1e9 + 0.0,
           "device_total_gb": total / 1e9,
           "gradients_finite": bool(np.isfinite(g["lin"]).all())}
    adj.close()
    w.close()
    return out


def _cpu_worker(args):
    """One CPU replica of the workload for `budget_s` seconds: the reference's
    CPU pipeline (bullet2 btDiscreteDynamicsWorld) when built, else the
    oracle port."""
    name, budget_s = args
    sys.path.insert(0, ROOT)
    import oracle
    from experiments_b200 import b3, scenes
    sc = make_scene(name)
    if oracle.bullet_lib() is not None:
        wld = oracle.ReferenceCpuWorld(sc)
        kind = "reference"
    else:
        hc = b3.Context(-1)
        w = b3.PhysicsWorld(hc, scenes.world_config(sc))
        scenes.register_scene(w, sc)
        wld = oracle.oracle_from_world(w, sc)
        kind = "port"
    t0 = time.perf_counter()
    steps = 0
    while time.perf_counter() - t0 < budget_s and steps < 1000:
        wld.step(1)
        steps += 1
    return sc.n, steps, time.perf_counter() - t0, kind


CPU_KIND = {"reference": "bullet2 btDiscreteDynamicsWorld (btDbvtBroadphase + btSequentialImpulseConstraintSolver, "
                         "10 iterations) built from the reference's bullet2 sources with g++ -O2",
            "port": "the oracle (single-threaded C++ restatement of the reference step, FP64)"}


def cpu_baseline_port(name, budget_s=12.0, procs=1):
    """The reference's CPU pipeline (or the oracle port) on `procs` host
    cores (independent replicas, one process each)."""
    if procs <= 1:
        n, steps, dt, kind = _cpu_worker((name, budget_s))
        return {"value": n * steps / dt, "unit": "body-steps/s", "cores": 1, "kind": kind,
                "sample": f"first {steps} steps of the full {n}-body scene ({dt:.1f} s), 1 thread; {CPU_KIND[kind]}"}
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(name, budget_s)] * procs)
    total = sum(n * s / dt for n, s, dt, _ in res)
    n, s, dt, kind = res[0]
    return {"value": total, "unit": "body-steps/s", "cores": procs, "kind": kind,
            "sample": f"{procs} independent replicas, each the first ~{s} steps of the full {n}-body scene "
                      f"(~{dt:.0f} s); {CPU_KIND[kind]}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b3", choices=["b3", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--scale", action="store_true", help="also run the 1,048,576-body plain and adjoint steps")
    ap.add_argument("--sap", action="store_true",
                    help="sweep-and-prune broadphase (pipeline2's default) in place of the grid; single-world workloads")
    ap.add_argument("--solver", default="jacobi", choices=["jacobi", "gs"],
                    help="jacobi: pipeline2's Jacobi solver (default); gs: the reference GPU solver, batched "
                         "Gauss-Seidel (4 contact + 4 friction iterations)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    args.warmup = max(3, args.warmup)
    cfg = {"workload": WORKLOADS[args.workload]}
    if args.sap:
        if args.workload in ("c3", "c3s"):
            ap.error("--sap takes a single-world workload (c1, c2, c2s, c5)")
        cfg["workload"] += ", sweep-and-prune broadphase"
    if args.solver == "gs":
        cfg["workload"] += ", batched Gauss-Seidel solver"
        # the CPU port times the Jacobi pipeline; no baseline for this form
        args.no_cpu_baseline = True

    if args.impl == "reference":
        if rank != 0:
            return
        procs = max(1, os.cpu_count() or 1)
        r = cpu_baseline_port(args.workload, budget_s=20.0, procs=procs)
        line = {"metric": "body-steps/s", "value": r["value"], "unit": "body-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32" if r["kind"] == "reference" else "f64",
                "data": "synthetic (seeded scene generator)", "impl": "reference",
                "config": cfg, "cpu_baseline": r,
                "e2e": {"value": r["value"], "unit": "body-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world_size > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    res = run_b3(args, world_size, local_rank)
    sc = res["sc"]
    ms_per_step = res["ms"] / args.steps
    # whole-job body-steps: every rank's shard (batched) or replica (plain)
    job_bodies = res["full"].n if res["sharded"] else sc.n * world_size
    value = job_bodies * args.steps / (res["ms"] / 1e3)
    hbm_peak, peak_kind = peaks()
    w = res["w"]
    dims = list(w.cfg.gridDims)
    key_bits = sum(int(d).bit_length() - 1 for d in dims) + \
        ((int(sc.num_worlds) - 1).bit_length() if sc.num_worlds > 1 else 0)
    body_bits = max(1, int(sc.n).bit_length())
    sb = stage_bytes(sc.n, res["c2"], key_bits, body_bits, 10)
    sm = dict(zip(STAGES, res["stage_ms"].tolist()))
    stage_roof = {}
    for k in STAGES:
        if k == "narrowphase":
            ach = res["flops"] / (sm[k] / 1e3) / 1e12
            stage_roof[k] = {"bound": "fp32", "achieved": ach, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
                             "frac": ach / FP32_PEAK_TFLOPS, "ms": sm[k]}
        else:
            ach = sb[k] / (sm[k] / 1e3) / 1e9
            stage_roof[k] = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                             "frac": ach / hbm_peak, "ms": sm[k]}
    b_step = step_bytes(sc.n, res["counters"], key_bits, 10)
    step_roof = {"bound": "hbm", "achieved": b_step / (ms_per_step / 1e3) / 1e9, "peak": hbm_peak,
                 "unit": "GB/s", "bytes_per_step": b_step, "peak_kind": peak_kind}
    step_roof["frac"] = step_roof["achieved"] / hbm_peak
    dom = max(sm, key=lambda k: sm[k])
    roof = dict(stage_roof[dom])
    roof["kernel"] = dom
    roof["traffic"] = NARROWPHASE_DRAM_BYTES_PER_PAIR * res["c2"]["numPairs"] if dom == "narrowphase" else None
    roof["traffic_source"] = "ncu dram bytes per pair on the 16,384-body case, scaled by pairs" \
        if dom == "narrowphase" else None
    roof["peak_kind"] = "nominal FP32 CUDA-core peak" if roof["bound"] == "fp32" else peak_kind
    if roof["bound"] == "fp32":
        roof["work"] = ("FLOPs of the reference algorithm (every axis projected, 8 (VA+VB)(FA+FB+EA*EB) per pair "
                        "+ 64 V_inc V_ref per clip); the sweep skips axes that provably cannot separate or be the "
                        "minimum, so the FLOPs executed are fewer")
    cfg.update({"bodies": int(sc.n), "worlds": int(sc.num_worlds), "pairs": res["counters"]["numPairs"],
                "manifolds": res["counters"]["numManifolds"],
                "contact_points": res["counters"]["numContactPoints"], "iterations": 10, "dt": 1 / 60,
                "refined_axes": res["counters"]["refinedAxes"], "refined_clips": res["counters"]["refinedClips"],
                "l2": "flushed between timed steps (256 MiB write outside the events)",
                "tuning": {"np_warps_per_cta": res["tuning"][0], "pair_cta": res["tuning"][1],
                           "jacobi_cta": res["tuning"][2], "jacobi_blocks_per_sm": res["tuning"][4],
                           "autotune_trials": res["tuning"][5], "jacobi_per_world_blocks": res["tuning"][6],
                           "jacobi_gather4": res["tuning"][7],
                           "kernels_per_step": int(res["kernels"])},
                "parallelism": (f"worlds sharded x{world_size}" if res["sharded"] else f"replicas x{world_size}")
                if world_size > 1 else "single GPU",
                "error": "pairs/keys bit-exact; contacts 1e-5 m / normals 1e-4; one step 1e-5 m, 1e-4 m/s "
                         "(tests/test_gpu_parity.py)"})
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if res["sharded"] else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generator)",
        "config": cfg,
        # contact points of every rank (summed), per timed second
        "contacts_per_s": res["contact_points"] * args.steps / (res["ms"] / 1e3),
        "roofline": roof, "step_roofline": step_roof, "stage_roofline": stage_roof, "clocks": res["clocks"],
        "e2e": {"value": job_bodies / (res["e2e_ms"] / 1e3), "unit": "body-steps/s",
                "h2d_bytes_per_step": 64 * sc.n, "d2h_bytes_per_step": 64 * sc.n},
        "gpu_launches": int(res["kernels"]) * args.steps,
    }
    if rank == 0 and world_size == 1 and not args.no_forms:
        line["forms"] = forms_comparison(res["ctx"])
        line["forms"]["adjoint"] = adjoint_form(res["ctx"])
    if rank == 0 and world_size == 1 and args.scale:
        line["scale"] = scale_run(res["ctx"])
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(args.workload)
    if rank == 0:
        print(json.dumps(line))
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
