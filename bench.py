"""Throughput benchmark of the B200 rigid-body step.

python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2] [--impl b3|reference]

Prints one JSON line on rank 0.

* value: whole-job body-steps/s of the plain step on the workload (default
  the 131,072-body mixed-hull scene), the scene resident in HBM, timed in
  the contact-rich part of the run: the scene is stepped to the settle step
  (300 of c2's 1,000: every layer has landed), then W warm-up steps, then K
  timed steps. Each timed step is one replay of the captured step graph
  bracketed by CUDA events on the launching stream; a 256 MiB write
  flushes L2 between steps, outside the events. `early` holds the same
  measurement over the free-fall start (steps W+1..W+K). Max over ranks;
  for N > 1 every rank steps its own replica (weak scaling, no collective
  on the data path).
* e2e: the same metric through the C ABI with host buffers, in the settled
  window: every step uploads the body state from pinned host memory,
  steps, and reads the state back (H2D + D2H inside the timed region).
* error: one step of the timed state checked against the oracle, stage by
  stage (oracle/parity.py), measured in this run.
* roofline: the kernel that takes the most time in the settled step, from
  live per-kernel CUDA-event times: the separating-axis sweep and the FP32
  clip against the FP32 CUDA-core peak at the sampled SM clock, with the
  FP32 work they execute (per pair, from the ncu capture summarised in
  profiles/); the other kernels against the measured HBM copy bandwidth
  with their compulsory bytes. step_roofline is the whole step's
  compulsory bytes against HBM; stage_roofline lists every stage.
* cpu_baseline: the reference's CPU rigid-body pipeline (bullet2
  btDiscreteDynamicsWorld built from the reference's sources; the oracle
  port where that library is absent) on one host thread, timed in the
  settled window of one column of the scene (a 1/16 block of the lattice
  footprint, all layers, with the ground), stepped alone to the same settle
  step.
* forms: the batched 4,096-world step against the plain step run world by
  world on the same GPU, both at the settle step (body-steps/s of each;
  per-world time sampled on a subset), with the batched step's one-step
  error against the oracle; and the adjoint form (forward with checkpoints
  + reverse sweep) on the 256-world differentiable throw against its plain
  forward.
* scale: the 1,048,576-cube plain step and adjoint.
--impl reference: the same CPU pipeline on all host cores: one replica per
  core, each one column block of the scene stepped to the settle step and
  then timed (the 16 blocks tile the whole scene), same metric.
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
# per-kernel CUDA-event times that b3_get_stage_times appends after the 7 stages
KERNELS = ["k_np_sweep", "k_np_refine", "k_np_clip", "k_np_exact", "k_setup_rows", "k_jacobi"]
# The settle step of each workload: the timed window starts there (the
# contact-rich part of the configuration's run); c5 runs 32 steps in all.
SETTLE = {"c1": 150, "c2": 300, "c2s": 300, "c3": 300, "c3s": 300, "c5": 24}
# Lattice dimensions of the single-world lattice workloads (CPU column blocks).
LATTICE = {"c1": (16, 16, 16), "c2": (64, 32, 64), "c2s": (32, 16, 32), "c5": (128, 64, 128)}


def fp32_peak_tflops(sm_mhz):
    """FP32 CUDA-core peak at an SM clock: 148 SMs x 128 FP32 lanes x 2
    (FMA) x clock. No FP32 peak is measured for this device, so this is the
    nominal peak at the clock sampled during the timed region."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


# Per-unit figures from the ncu capture of the settled 16,384-body case (the
# same kernels; summarised under profiles/): FP32 operations each kernel
# executes (2 per FFMA + FADD + FMUL, 4 per FFMA2, 2 per FMUL2, per thread)
# and DRAM bytes (read + write), per pair or per manifold.
NCU_SOURCE = "ncu capture of the settled 16,384-body mixed-hull step (profiles/)"
NCU_PER_UNIT = {
    "k_np_sweep": {"fp32_ops_per_pair": 26729.0, "dram_bytes_per_pair": 13.2, "source": NCU_SOURCE},
    "k_np_clip": {"fp32_ops_per_manifold": 4740.0, "dram_bytes_per_manifold": 106.8, "source": NCU_SOURCE},
    "k_setup_rows": {"dram_bytes_per_manifold": 301.3, "source": NCU_SOURCE},
    "k_jacobi": {"dram_bytes_per_manifold": 618.5, "source": NCU_SOURCE},
}


def profile_constants():
    return NCU_PER_UNIT


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


def window_counts(c, n, steps_done):
    """N, P, C and contact points of the last step, for the record."""
    return {"step": int(steps_done), "bodies": int(n), "pairs": int(c["numPairs"]),
            "manifolds": int(c["numManifolds"]), "contact_points": int(c["numContactPoints"]),
            "manifolds_per_body": c["numManifolds"] / max(n, 1), "iterations": 10,
            "refined_axes": int(c["refinedAxes"]), "refined_clips": int(c["refinedClips"])}


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
    settle = max(args.settle, args.warmup + args.steps)

    def barrier():
        torch.cuda.synchronize()
        if world_size > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world_size > 1:
            import torch.distributed as dist
            t = torch.tensor([x], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    # early window: the free-fall start of the run, launch shapes tuned there
    w.autotune(3, stream=st.cuda_stream)
    for _ in range(args.warmup):
        w.stepSimulation(1, stream=st.cuda_stream)
    barrier()
    early_ms = max_over_ranks(time_steps(w, args.steps, st, flush))
    early = window_counts(w.counters(), sc.n, args.warmup + args.steps)
    early["ms_per_step"] = early_ms / args.steps
    done = args.warmup + args.steps
    # settled window: step on to the settle step, retune there, warm up, time
    if settle - args.warmup > done:
        w.stepSimulation(settle - args.warmup - done, stream=st.cuda_stream)
        done = settle - args.warmup
    if args.tuning:
        # fixed launch shapes (b3_get_tuning order) instead of the autotuner:
        # a profiler run repeats the shapes the plain run chose
        w.set_tuning([int(x) for x in args.tuning.split(",")])
    else:
        w.autotune(3, stream=st.cuda_stream)
    tuning = w.tuning()
    for _ in range(args.warmup):
        w.stepSimulation(1, stream=st.cuda_stream)
    done += args.warmup
    barrier()
    if args.profile_window:
        torch.cuda.profiler.start()
    with ClockSampler(local_rank) as clk:
        ms = time_steps(w, args.steps, st, flush)
    if args.profile_window:
        torch.cuda.profiler.stop()
    barrier()
    ms = max_over_ranks(ms)
    done += args.steps
    counters = w.counters()
    kernels = w.tuning()[3]
    # per-stage and per-kernel CUDA events on three more eager steps of the
    # same world (timing only, not part of `value`)
    w.set_stage_timing(True)
    acc = None
    for _ in range(3):
        flush_l2(flush)
        w.stepSimulation(1, stream=st.cuda_stream)
        t = np.array(w.stage_times(), np.float64)
        acc = t if acc is None else acc + t
    w.set_stage_timing(False)
    done += 3
    stage_ms = acc / 3
    c2 = w.counters()
    flops = sat_flops(w, sc)
    # e2e through the C ABI with pinned host buffers
    pos, quat, lin, ang = w.read_state()
    hp = torch.from_numpy(pos).pin_memory().numpy()
    hq = torch.from_numpy(quat).pin_memory().numpy()
    hl = torch.from_numpy(lin).pin_memory().numpy()
    ha = torch.from_numpy(ang).pin_memory().numpy()
    e2e_steps = max(3, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        # H2D of the step's input state from pinned memory, the step, and the
        # D2H of its result straight into the same pinned buffers
        w.write_state(hp, hq, hl, ha, stream=st.cuda_stream)
        w.stepSimulation(1, stream=st.cuda_stream)
        w.read_state(stream=st.cuda_stream, out=(hp, hq, hl, ha))
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps)
    done += e2e_steps
    contact_points = counters["numContactPoints"]
    if world_size > 1:
        import torch.distributed as dist
        t = torch.tensor([contact_points], device="cuda", dtype=torch.int64)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        contact_points = int(t.item())
    settled = window_counts(counters, sc.n, settle + args.steps)
    settled["ms_per_step"] = ms / args.steps
    return dict(sc=sc, full=full, sharded=sharded, ms=ms, contact_points=contact_points, tuning=tuning,
                counters=counters, stage_ms=stage_ms, c2=c2, clocks=clk.summary(), e2e_ms=e2e_ms, w=w,
                kernels=kernels, flops=flops, ctx=ctx, early=early, settled=settled, early_ms=early_ms,
                steps_done=done)


def oracle_check(w, sc):
    """One step of the device world's current state against the oracle
    (the checker: oracle/parity.py), reported next to the throughput."""
    import oracle
    from oracle import parity
    o = oracle.oracle_from_world(w, sc)
    rep = parity.one_step_report(w, o, dynamic=np.asarray(sc.mass) > 0,
                                 make_oracle=lambda f32: oracle.oracle_from_world(w, sc, f32=f32))
    o.close()
    keep = ["pos_err_m", "lin_vel_err_mps", "ang_vel_err_radps", "quat_err", "contact_point_err_m", "normal_err",
            "aabbs_bit_exact", "keys_bit_exact", "permutation_bit_exact", "pairs_bit_exact", "manifold_set_equal",
            "pairs", "manifolds", "pair_overflow", "narrowphase_within_bars", "solver_err", "fp32_envelope",
            "contact_sensitivity", "bars_used", "step_bars_used", "within_bars", "check_s"]
    out = {k: rep[k] for k in keep}
    out["manifolds_differing"] = len(rep["manifold_differences"])
    out["bars"] = ("pairs/keys/permutation bit-exact; contacts 1e-5 m, normals 1e-4; one step 1e-5 m, 1e-4 m/s, or "
                   "twice the FP32 envelope (the oracle's FP32 build against its FP64 build from the same contacts) "
                   "where that is larger; solver_err: the device's solve against the FP64 oracle's from the "
                   "device's contacts")
    return out


def forms_comparison(ctx, steps=10, sample_worlds=32, settle=SETTLE["c3"], check=True):
    """Batched 4,096-world step vs the plain step run world by world, both
    from the batched scene's state at the settle step (piles in contact)."""
    import torch
    from experiments_b200 import scenes
    sc = scenes.c3()
    wb = scenes.build_world(ctx, sc, useGraph=1)
    st = torch.cuda.current_stream()
    wb.stepSimulation(settle, stream=st.cuda_stream)
    wb.autotune(3, stream=st.cuda_stream)
    for _ in range(3):
        wb.stepSimulation(1, stream=st.cuda_stream)
    ms_b = time_steps(wb, steps, st, None)
    batched = sc.n * steps / (ms_b / 1e3)
    cb = wb.counters()
    # the state the batched timing started from is gone; take the current
    # one for the per-world worlds and time them over the same count of steps
    pos, quat, lin, ang = wb.read_state()
    # plain per-world step: each world in its own plain world, stepped one
    # world at a time (the reference's one-scene-per-pipeline usage)
    counts = sc.extra["counts"]
    rng = np.random.default_rng(0)
    pick = rng.choice(len(counts), size=min(sample_worlds, len(counts)), replace=False)
    total_ms = 0.0
    bodies = 0
    for wid in pick:
        sub = scenes.select_worlds(sc, [int(wid)])
        idx = np.nonzero(np.asarray(sc.world) == int(wid))[0]
        wp = scenes.build_world(ctx, sub, useGraph=1)
        wp.write_state(pos[idx], quat[idx], lin[idx], ang[idx])
        for _ in range(3):
            wp.stepSimulation(1, stream=st.cuda_stream)
        total_ms += time_steps(wp, steps, st, None)
        bodies += sub.n
        wp.close()
    # extrapolate the sampled per-world times to all worlds
    per_body_ms = total_ms / max(bodies, 1)
    plain = sc.n * steps / (per_body_ms * sc.n / 1e3)
    out = {"batched_body_steps_per_s": batched, "plain_per_world_body_steps_per_s": plain,
           "speedup": batched / plain, "worlds": int(sc.num_worlds), "bodies": int(sc.n),
           "plain_sample": f"{len(pick)} of {sc.num_worlds} worlds, {steps} steps each, graph replay, "
                           f"from the batched scene's state at step {settle + 3 + steps}",
           "steps": steps, "window": window_counts(cb, sc.n, settle + 3 + steps)}
    if check:
        out["error"] = oracle_check(wb, sc)
    wb.close()
    return out


def adjoint_form(ctx, worlds=256, steps=120, checkpoint_every=16, check_worlds=8):
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
    err = adjoint_gradient_error(ctx, sc, g, pos, check_worlds) if check_worlds else None
    total = fwd_ms + bwd_ms
    return {"workload": f"differentiable throw, {worlds} worlds x 64 cubes, {steps} steps, checkpoints every "
                        f"{checkpoint_every}", "bodies": int(sc.n),
            "adjoint_body_steps_per_s": sc.n * steps / (total / 1e3),
            "plain_body_steps_per_s": sc.n * steps / (plain_ms / 1e3),
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "plain_ms": plain_ms,
            "cost_vs_plain": total / plain_ms, "worlds_with_finite_gradients": finite_worlds,
            "gradient_error": err}


def adjoint_gradient_error(ctx, sc, g, final_pos, check_worlds):
    """The adjoint run's gradients on its first `check_worlds` worlds
    against the FP64 tangent-linear oracle chained along the device's own
    trajectory (the checker: oracle/tangent_chain.py): the trajectory is
    recorded step by step on a plain world of the same scene, checked to be
    the checkpointed forward's bit for bit, and the FP64 one-step Jacobians
    at its states are chained along random directions of each parameter
    set. Worlds are independent, so the first worlds of the throw are the
    throw of that many worlds."""
    import time as _time
    import torch
    import oracle
    from oracle import tangent_chain
    from experiments_b200 import scenes
    t0 = _time.perf_counter()
    st = torch.cuda.current_stream()
    wt = scenes.build_world(ctx, sc, useGraph=1)
    traj = [[a.astype(np.float64) for a in wt.read_state(stream=st.cuda_stream)]]
    for _ in range(sc.steps):
        wt.stepSimulation(1, stream=st.cuda_stream)
        traj.append([a.astype(np.float64) for a in wt.read_state(stream=st.cuda_stream)])
    wt.close()
    same_forward = bool(np.array_equal(traj[-1][0], final_pos))
    sub = scenes.c4(worlds=check_worlds, steps=sc.steps)
    per = 64
    idx = np.concatenate([np.arange(check_worlds), sc.num_worlds + np.arange(check_worlds * per)])
    assert np.array_equal(np.asarray(sub.mass), np.asarray(sc.mass)[idx])
    straj = [[a[idx] for a in s] for s in traj]
    sg = {k: np.asarray(g[k])[idx] for k in ("lin", "ang", "mass", "friction")}
    seeds = tangent_chain.com_seeds(sub, straj[-1][0])
    wr = scenes.build_world(ctx, sub, useGraph=1)
    o = oracle.oracle_from_world(wr, sub, dual=True)
    ov = oracle.oracle_from_world(wr, sub)
    ii = wr.inertias()[:, :3].astype(np.float64)
    wr.close()
    rel, stable = tangent_chain.gradient_errors(o, ii, sub, straj, sg, seeds, o_value=ov)
    o.close()
    ov.close()
    allrel = np.concatenate(list(rel.values()))
    return {"worlds_checked": int(check_worlds), "robust_worlds": int(stable.sum()),
            "trajectory_is_checkpointed_forward": same_forward,
            "median_rel": float(np.median(allrel)),
            "quartiles_rel": [float(np.percentile(allrel, q)) for q in (25, 75)],
            "max_rel": float(allrel.max()),
            "fraction_within_1e-3": float(np.mean(allrel < 1e-3)),
            "max_rel_by_parameter": {k: float(r.max()) for k, r in rel.items()},
            "reference": "FP64 tangent-linear oracle chained along the device's own trajectory, 2 random "
                         "directions per parameter set (velocities, masses, friction), per world and parameter set; "
                         "robust worlds: the FP64 discrete choices along the trajectory do not flip under "
                         "perturbations of the recorded states at the device's one-step deviation",
            "check_s": _time.perf_counter() - t0}


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
    """One CPU replica: the reference's CPU pipeline (bullet2
    btDiscreteDynamicsWorld) when built, else the oracle port, on one column
    block of a lattice workload (or the whole scene of a batched one). It is
    stepped untimed to the settle step, then timed for up to `budget_s`
    seconds (at least one step)."""
    name, block, settle, budget_s = args
    sys.path.insert(0, ROOT)
    import oracle
    from experiments_b200 import b3, scenes
    sc = make_scene(name)
    if block is not None and name in LATTICE:
        sc = scenes.lattice_block(sc, LATTICE[name], block)
    if oracle.bullet_lib() is not None:
        wld = oracle.ReferenceCpuWorld(sc)
        kind = "reference"
    else:
        hc = b3.Context(-1)
        w = b3.PhysicsWorld(hc, scenes.world_config(sc))
        scenes.register_scene(w, sc)
        wld = oracle.oracle_from_world(w, sc)
        kind = "port"
    ts = time.perf_counter()
    wld.step(settle)
    settle_s = time.perf_counter() - ts
    t0 = time.perf_counter()
    steps = 0
    while steps < 1 or (time.perf_counter() - t0 < budget_s and steps < 1000):
        wld.step(1)
        steps += 1
    return sc.n, steps, time.perf_counter() - t0, kind, settle_s


CPU_KIND = {"reference": "bullet2 btDiscreteDynamicsWorld (btDbvtBroadphase + btSequentialImpulseConstraintSolver, "
                         "10 iterations) built from the reference's bullet2 sources with g++ -O2",
            "port": "the oracle (single-threaded C++ restatement of the reference step, FP64)"}


def cpu_baseline_port(name, budget_s=10.0, procs=1, settle=None):
    """The reference's CPU pipeline (or the oracle port) on `procs` host
    cores, one replica per core. For a lattice workload replica r runs
    column block r mod 16 of the scene (the 16 blocks tile the footprint),
    stepped alone to the settle step and then timed; a batched workload runs
    whole, timed from the start."""
    settle = SETTLE.get(name, 0) if settle is None else settle
    lattice = name in LATTICE
    blocks = [k % 16 if lattice else None for k in range(max(1, procs))]
    st = settle if lattice else 0
    if procs <= 1:
        res = [_cpu_worker((name, blocks[0], st, budget_s))]
    else:
        ctx = mp.get_context("spawn")
        with ctx.Pool(procs) as pool:
            res = pool.map(_cpu_worker, [(name, b, st, budget_s) for b in blocks])
    total = sum(n * s / dt for n, s, dt, _, _ in res)
    n, s, dt, kind, settle_s = res[0]
    if lattice:
        what = (f"{len(res)} replica(s), each one 1/16 column block of the scene ({n} bodies with the ground; the "
                f"16 blocks tile the footprint) stepped alone to step {st} ({settle_s:.0f} s untimed), then ~{s} "
                f"steps timed (~{dt:.0f} s)")
    else:
        what = f"{len(res)} replica(s), each the first ~{s} steps of the full {n}-body scene (~{dt:.0f} s)"
    return {"value": total, "unit": "body-steps/s", "cores": len(res), "kind": kind,
            "sample": f"{what}; {CPU_KIND[kind]}"}


def kernel_roofline(name, ms, sc, counters, key_bits, body_bits, hbm_peak, peak_kind, sm_mhz, consts):
    """Roofline of one kernel or stage from its CUDA-event time. The sweep
    and the FP32 clip are FP32-issue bound: achieved = the FP32 operations
    they execute (per unit, from the ncu capture) / time, against the FP32
    CUDA-core peak at the sampled clock. Everything else is HBM bound:
    compulsory bytes / time against the measured copy bandwidth."""
    n = sc.n
    P = counters["numPairs"]
    C = counters["numManifolds"]
    iters = 10
    sb = stage_bytes(n, counters, key_bits, body_bits, iters)
    hbm_bytes = dict(sb)
    hbm_bytes["k_setup_rows"] = C * (96 + 368)
    hbm_bytes["k_jacobi"] = iters * (200 * C + 64 * n)
    hbm_bytes["k_np_refine"] = None
    hbm_bytes["k_np_exact"] = None
    units = {"k_np_sweep": ("pair", P), "k_np_clip": ("manifold", C)}
    if name in units:
        unit, count = units[name]
        c = consts.get(name, {})
        ops = c.get("fp32_ops_per_" + unit)
        peak = fp32_peak_tflops(sm_mhz or 1965.0)
        r = {"kernel": name, "bound": "fp32", "unit": "TFLOP/s", "peak": peak, "ms": ms,
             "peak_kind": f"nominal FP32 CUDA-core peak at the sampled SM clock ({sm_mhz} MHz); no measured FP32 peak"}
        if ops is not None:
            r["achieved"] = ops * count / (ms / 1e3) / 1e12
            r["frac"] = r["achieved"] / peak
            r["work"] = (f"executed FP32 operations: {ops:.0f} per {unit} (2 per FFMA + FADD + FMUL, 4 per FFMA2, "
                         f"2 per FMUL2, per thread) "
                         f"from {c.get('source')}, times {count} {unit}s")
        else:
            r["achieved"] = None
            r["frac"] = None
            r["work"] = "no ncu capture of this kernel's executed FP32 operations"
        dram = c.get("dram_bytes_per_" + unit)
        r["traffic"] = dram * count if dram is not None else None
        r["traffic_source"] = c.get("source") if dram is not None else None
        if name == "k_np_clip":
            r["launches"] = ("the FP32 clip stage: k_np_clip_groups (eight-lane groups) when the tuning selects it, "
                             "then k_np_clip on the pairs it passes on")
        return r
    b = hbm_bytes.get(name)
    r = {"kernel": name, "bound": "hbm", "unit": "GB/s", "peak": hbm_peak, "ms": ms, "peak_kind": peak_kind}
    if b is None:
        r.update(achieved=None, frac=None, traffic=None, work="latency-bound minority path; no byte model")
        return r
    r["achieved"] = b / (ms / 1e3) / 1e9
    r["frac"] = r["achieved"] / hbm_peak
    r["bytes"] = b
    c = consts.get(name, {})
    unit = "manifold" if name in ("k_setup_rows", "k_jacobi") else "body"
    dram = c.get("dram_bytes_per_" + unit)
    r["traffic"] = dram * (C if unit == "manifold" else n) if dram is not None else None
    r["traffic_source"] = c.get("source") if dram is not None else None
    return r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="b3", choices=["b3", "reference"])
    ap.add_argument("--settle", type=int, default=None,
                    help="step at which the timed window starts (default: per workload, c2 300)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-scale", action="store_true", help="skip the 1,048,576-body plain and adjoint steps")
    ap.add_argument("--no-check", action="store_true", help="skip the one-step oracle checks")
    ap.add_argument("--tuning", default=None,
                    help="settled-window launch shapes as b3_get_tuning's comma-separated values (np warps per CTA, "
                         "pair CTA, Jacobi CTA, -, Jacobi blocks per SM, -, Jacobi mode, Jacobi gather[, pair search "
                         "form[, clip form]]) instead of "
                         "autotuning, e.g. to repeat a plain run's shapes under a profiler")
    ap.add_argument("--profile-window", action="store_true",
                    help="bracket the settled window's timed steps with cudaProfilerStart / cudaProfilerStop, so that "
                         "a profiler started with --profile-from-start off sees those launches only")
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
    if args.settle is None:
        args.settle = SETTLE[args.workload]
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
        r = cpu_baseline_port(args.workload, budget_s=15.0, procs=procs, settle=args.settle)
        cfg["window"] = f"settled: timed from step {args.settle}" if args.workload in LATTICE else "from the start"
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
    sm_mhz = res["clocks"].get("sm_mhz")
    consts = profile_constants()
    sb = stage_bytes(sc.n, res["c2"], key_bits, body_bits, 10)
    stage_ms = res["stage_ms"].tolist()
    sm = dict(zip(STAGES, stage_ms[:len(STAGES)]))
    km = dict(zip(KERNELS, stage_ms[len(STAGES):len(STAGES) + len(KERNELS)]))
    stage_roof = {}
    for k in STAGES:
        if k == "narrowphase":
            ach = res["flops"] / (sm[k] / 1e3) / 1e12
            pk = fp32_peak_tflops(sm_mhz or 1965.0)
            stage_roof[k] = {"bound": "fp32", "algorithmic_tflops": ach, "peak": pk, "unit": "TFLOP/s",
                             "ms": sm[k],
                             "work": "FLOPs of the reference algorithm (every axis projected: 8 (VA+VB)(FA+FB+EA*EB) "
                                     "per pair + 64 V_inc V_ref per clip); the kernels skip axes that provably cannot "
                                     "separate or be the minimum, so they execute fewer (see roofline)"}
        else:
            ach = sb[k] / (sm[k] / 1e3) / 1e9
            stage_roof[k] = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                             "frac": ach / hbm_peak, "ms": sm[k]}
    kernel_roof = {}
    for k, t in list(km.items()) + [(s_, sm[s_]) for s_ in ("aabb_hash", "sort_cells", "find_pairs", "manifolds",
                                                            "integrate")]:
        if t > 0:
            kernel_roof[k] = kernel_roofline(k, t, sc, res["c2"], key_bits, body_bits, hbm_peak, peak_kind, sm_mhz,
                                             consts)
    b_step = step_bytes(sc.n, res["counters"], key_bits, 10)
    step_roof = {"bound": "hbm", "achieved": b_step / (ms_per_step / 1e3) / 1e9, "peak": hbm_peak,
                 "unit": "GB/s", "bytes_per_step": b_step, "peak_kind": peak_kind,
                 "model": "N (128 + 20 + 8 + S + 12 + 32) + 80 P + 368 C + I (200 C + 64 N)"}
    step_roof["frac"] = step_roof["achieved"] / hbm_peak
    # the dominant kernel of the settled step
    dom = max(kernel_roof, key=lambda k: kernel_roof[k]["ms"])
    roof = dict(kernel_roof[dom])
    roof["share_of_step"] = roof["ms"] / max(sum(sm.values()), 1e-9)
    early_bytes = step_bytes(sc.n, {"numPairs": res["early"]["pairs"], "numManifolds": res["early"]["manifolds"]},
                             key_bits, 10)
    early = dict(res["early"])
    early["body_steps_per_s"] = job_bodies / (early["ms_per_step"] / 1e3)
    early["step_roofline_frac"] = early_bytes / (early["ms_per_step"] / 1e3) / 1e9 / hbm_peak
    settled = dict(res["settled"])
    settled["step_roofline_frac"] = step_roof["frac"]
    cfg.update({"bodies": int(sc.n), "worlds": int(sc.num_worlds), "iterations": 10, "dt": 1 / 60,
                "window": f"steps {args.settle + 1}..{args.settle + args.steps} of the run (settle step "
                          f"{args.settle}, {args.warmup} warm-up steps before it)",
                "pairs": res["counters"]["numPairs"], "manifolds": res["counters"]["numManifolds"],
                "contact_points": res["counters"]["numContactPoints"],
                "l2": "flushed between timed steps (256 MiB write outside the events)",
                "tuning": {"np_warps_per_cta": res["tuning"][0], "pair_cta": res["tuning"][1],
                           "jacobi_cta": res["tuning"][2], "jacobi_blocks_per_sm": res["tuning"][4],
                           "autotune_trials": res["tuning"][5], "jacobi_per_world_blocks": res["tuning"][6],
                           "jacobi_gather4": res["tuning"][7], "pair_search_warp_per_body": res["tuning"][8],
                           "clip_lane_groups": res["tuning"][9],
                           "kernels_per_step": int(res["kernels"])},
                "parallelism": (f"worlds sharded x{world_size}" if res["sharded"] else f"replicas x{world_size}")
                if world_size > 1 else "single GPU"})
    line = {
        "metric": "body-steps/s", "value": value, "unit": "body-steps/s", "n_gpus": world_size,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong" if res["sharded"] else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene generator)",
        "config": cfg,
        # contact points of every rank (summed), per timed second
        "contacts_per_s": res["contact_points"] * args.steps / (res["ms"] / 1e3),
        "settled": settled, "early": early,
        "roofline": roof, "step_roofline": step_roof, "kernel_roofline": kernel_roof,
        "stage_roofline": stage_roof, "clocks": res["clocks"],
        "e2e": {"value": job_bodies / (res["e2e_ms"] / 1e3), "unit": "body-steps/s",
                "h2d_bytes_per_step": 64 * sc.n, "d2h_bytes_per_step": 64 * sc.n},
        "gpu_launches": int(res["kernels"]) * args.steps,
    }
    if rank == 0 and world_size == 1 and not args.no_check:
        line["error"] = oracle_check(w, sc)
    if rank == 0 and world_size == 1 and not args.no_forms:
        line["forms"] = forms_comparison(res["ctx"], check=not args.no_check)
        line["forms"]["adjoint"] = adjoint_form(res["ctx"], check_worlds=0 if args.no_check else 8)
    if rank == 0 and world_size == 1 and not args.no_scale:
        line["scale"] = scale_run(res["ctx"])
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_port(args.workload, settle=args.settle)
    if rank == 0:
        print(json.dumps(line))
    if world_size > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
