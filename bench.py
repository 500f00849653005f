#!/usr/bin/env python
"""Throughput of the XPBD cloth substep on B200: cloth-steps/s (one cloth advanced one 1/60 s frame of 10 substeps x
10 iterations).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c1|c3|c0|c2] [--impl ours|reference]

Default workload (the headline): c1 — one 256x256 sheet (65,536 particles, 390,658 constraints), colored
Gauss–Seidel, damping 0.01. The same JSON line also carries the batched workload c3 (256 seeded cloths of 16..192
vertices a side, plain Jacobi with degree-averaged corrections) under "batched", measured the same way.

Timing: W untimed warm-up steps, then exactly K steps bracketed by a barrier + device synchronize; each step is timed
with CUDA events on the stream the library launches on, max over ranks. Working sets below the 126 MB L2 are
flushed (256 MiB write) between timed steps outside the events; larger ones are not. `e2e` is the same metric through
the public API with host buffers: per step the parameter block goes host->device, one frame is stepped and the
positions come back device->host, timed on the host clock. Multi-GPU: one process per GPU (torchrun); c1 runs one
independent replica per rank, c3 shards the cloths across ranks — no collective in the step (weak scaling).

The same line also carries `warm_start`: the convergence solve (Jacobi to a 1e-4 residual, capped) with a plain,
previous-λ and learned (on-GPU trained MLP) start — passes per cloth-substep and cloth-steps/s for each.

--impl reference times the CPU restatement of the reference solver (src/xpbd_cpu.rs, OpenMP over the independent
loops) on the same workload and prints the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "cloth-steps/s at 256² & batched; iters to 1e-4 strain residual, learned vs plain"
UNIT = "cloth-steps/s"
L2_BYTES = 126 * 1024 * 1024
DEV_PARAMS_BYTES = 128  # sizeof(XpbdDevParams): the per-call parameter block uploaded by xpbd_set_params


# ------------------------------------------------------------------------------------------------ workloads
def make_workload(name: str, rank: int = 0, world: int = 1, c3_cloths: int = 0) -> dict:
    from bevy_xpbd_b200 import plugin as P
    from bevy_xpbd_b200 import workloads as wl
    dt, inv_dt = wl.substep_dt(10)
    if name == "c1":
        specs = [wl.config1_sheet()]
        prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 10, linear_drag_per_sec=0.01)
        cfg = P.ClothSimConfig(solver=P.SOLVER_GAUSS_SEIDEL, solve_substeps=10)
        desc = "c1: 256x256 sheet, 2 m, top edge pinned, colored Gauss-Seidel, 10 substeps x 10 iterations, damping 0.01"
        total_cloths = world  # one replica per rank
    elif name == "c0":
        specs = [wl.config0_sheet()]
        prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 10)
        cfg = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
        desc = "c0: 32x32 sheet, 1 m, two corners pinned, plain Jacobi (degree-averaged), 10 substeps x 10 iterations"
        total_cloths = world
    elif name == "c2":
        specs = [wl.config2_sheet()]
        prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 10)
        cfg = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
                               collision=P.COLLISION_RING_FILTER, thickness=0.002, hash_cell=0.004,
                               hash_table_bits=20, ring_depth=2, ground_enabled=True, ground_y=0.0)
        desc = ("c2: 512x512 sheet, 2 m, unpinned, falling and folding; self collision every substep (hash cell 4 mm, "
                "2^20 table, stable 3x8-bit radix sort, 27-cell query, 2-ring filter, thickness 2 mm); Jacobi 10x10")
        total_cloths = world
    elif name == "c3":
        allspecs = wl.config3_batch()
        if c3_cloths:
            allspecs = allspecs[:c3_cloths]
        from bevy_xpbd_b200.sharding import shard_by_constraints
        mine = shard_by_constraints([s.num_constraints for s in allspecs], world)[rank]
        specs = [allspecs[k] for k in mine]
        prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 10)
        cfg = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
        desc = (f"c3: {len(allspecs)} cloths, sides seeded uniform 16..192 vertices, random pins and stretch compliance, "
                "packed into one persistent launch per frame, plain Jacobi (degree-averaged), 10 substeps x 10 "
                "iterations")
        total_cloths = len(allspecs)
    else:
        raise ValueError(name)
    n = sum(s.num_particles for s in specs)
    e = sum(s.num_constraints for s in specs)
    S, I = cfg.solve_substeps, prm.inner_iterations
    # algorithmic bytes per frame (fp32): S*(100N + I*(28N + 16E)) — per pass x read+write and inverse mass (28 B per
    # particle) plus i, j, rest, compliance (16 B per constraint); per substep 100 B per particle for predict + velocity
    bytes_alg = S * (100 * n + I * (28 * n + 16 * e))
    if cfg.collision:
        # self collision every substep, 124 B per particle: hash keys (read x 16, write key + value 8), three 8-bit
        # radix passes (histogram reads keys 4, scatter reads and writes key + value 16 -> 60), bucket starts (read
        # sorted keys 4, write 4), resolve (read and write the position once each, 32)
        bytes_alg += S * 124 * n
    full_launch = name != "c3" or (not c3_cloths and world == 1)
    # c2 is timed after the sheet has folded onto the ground (60 untimed frames of the 240), not during the free fall
    pre_frames = 60 if name == "c2" else 0
    return dict(name=name, specs=specs, params=prm, cfg=cfg, desc=desc, n=n, e=e, cloths=len(specs),
                total_cloths=total_cloths, bytes_per_frame=bytes_alg, full_launch=full_launch, pre_frames=pre_frames)


_CONFIGS: dict = {}


def workload_config(name: str, world: int) -> dict:
    """The `config` object of both arms' JSON lines: the whole job's workload (every rank's cloths), how it is split
    over ranks, and the L2 policy of the timed region; identical for the GPU arm and the reference arm."""
    if (name, world) in _CONFIGS:
        return dict(_CONFIGS[(name, world)])
    w = make_workload(name, 0, 1)
    reps = world if name != "c3" else 1
    flush = working_set_bytes(w) < L2_BYTES
    _CONFIGS[(name, world)] = {"workload": w["desc"], "cloths": w["total_cloths"] * reps, "particles": w["n"] * reps,
            "constraints": w["e"] * reps, "substeps": w["cfg"].solve_substeps,
            "iterations": w["params"].inner_iterations,
            "parallelism": ("replicas" if name != "c3" else "cloth shards balanced by constraints") + f" x{world}",
            "l2": ("GPU arm: L2 flushed between timed steps (256 MiB write outside the events); CPU arm: n/a" if flush
                   else f"GPU arm: inputs larger than L2 (working set {working_set_bytes(w) / 1e6:.0f} MB); "
                        "CPU arm: n/a")}
    return dict(_CONFIGS[(name, world)])


def working_set_bytes(w: dict) -> int:
    # x, v, two Jacobi buffers, rest (16 B each per particle); 8 B per incidence + 16 B per constraint (two tables)
    return 80 * w["n"] + 16 * w["e"] + 32 * w["e"]


# ------------------------------------------------------------------------------------------------ helpers
def load_peaks() -> dict:
    for p in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        if os.path.exists(p):
            with open(p) as f:
                d = json.load(f)
            return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=6650.0, source="fallback")


def load_traffic(kernel: str, workload: str):
    """DRAM bytes per launch of `kernel` on `workload` from the committed ncu summary (profiles/traffic.txt lines
    'workload kernel bytes_per_launch'), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 3 and not line.startswith("#") and parts[0] == workload and parts[1] == kernel:
            return float(parts[2])
    return None


class ClockSampler:
    """nvidia-smi samples (every 200 ms) while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        import tempfile
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if self.proc is None or not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ------------------------------------------------------------------------------------------------ GPU arm
def build_plugin(w: dict, device: int):
    from bevy_xpbd_b200 import plugin as P
    plug = P.ClothComputePlugin(device)
    for s in w["specs"]:
        plug.add_spec(s)
    plug.commit()
    plug.set_params(w["params"], w["cfg"])
    return plug


def time_device(w: dict, plug, steps: int, warmup: int, world: int, device: int, flush: bool):
    """K frames, each bracketed by CUDA events on the library's stream (torch's current stream)."""
    import torch
    stream = torch.cuda.Stream()  # a real stream handle: the library launches on it, the events are recorded on it
    plug.set_stream(stream.cuda_stream)
    flush_buf = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda") if flush else None
    if w.get("pre_frames"):
        plug.step(frames=w["pre_frames"])
    for _ in range(warmup):
        plug.step(frames=1)
    plug.sync()
    torch.cuda.synchronize()
    st0 = plug.stats()
    if flush_buf is not None:
        flush_buf.record_stream(stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        for a, b in evs:
            if flush_buf is not None:
                with torch.cuda.stream(stream):
                    flush_buf.zero_()
            a.record(stream)
            plug.step(frames=1)
            b.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    plug.sync()
    st1 = plug.stats()
    per = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(per), world)
    launches = int(st1["kernel_launches"] - st0["kernel_launches"])
    plug.set_stream(None)
    return total_ms, per, launches, clk.summary(), st1


def time_e2e(w: dict, plug, steps: int, warmup: int, world: int):
    """Through the public API with host buffers: params H2D, one frame, positions D2H, per step (host clock)."""
    import torch
    host = np.empty((plug.num_particles, 3), np.float32)
    for _ in range(warmup):
        plug.set_params(w["params"])
        plug.step(frames=1)
        plug.positions_into(host)
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(steps):
        plug.set_params(w["params"])
        plug.step(frames=1)
        plug.positions_into(host)
    t1 = time.perf_counter()
    barrier(world)
    ms = max_over_ranks((t1 - t0) * 1e3, world)
    return ms, host


def roofline(w: dict, mean_ms: float, kernel: str, peaks: dict) -> dict:
    achieved = w["bytes_per_frame"] / (mean_ms * 1e-3) / 1e9
    # the committed per-launch traffic is of the full single-GPU workload: a sample of c3's cloths (--c3-cloths) or a
    # rank's shard of them launches less, and gets none
    traffic = load_traffic(kernel, w["name"]) if w["full_launch"] else None
    return {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
            "alg_bytes_per_launch": int(w["bytes_per_frame"]), "traffic": traffic}


def fixed_schedule(args) -> bool:
    return (args.no_autotune or args.jacobi_kernel is not None or args.block is not None or args.bps is not None
            or args.cluster is not None or args.gs_strips is not None)


def apply_schedule(w: dict, plug, args):
    """Autotuned schedule, or the one given on the command line (profiling runs pin it)."""
    if not fixed_schedule(args):
        return plug.autotune(frames=2)
    cfg = w["cfg"]
    if args.jacobi_kernel is not None:
        cfg.jacobi_kernel = args.jacobi_kernel
    if args.block is not None:
        cfg.block_threads = args.block
    if args.bps is not None:
        cfg.blocks_per_sm = args.bps
    if args.cluster is not None:
        cfg.cluster_ctas = args.cluster
    if args.gs_strips is not None:
        cfg.gs_strips = args.gs_strips
    plug.set_params(w["params"], cfg)
    return cfg


def run_gpu_workload(name: str, args, rank: int, world: int, device: int, peaks: dict, with_e2e: bool) -> dict:
    w = make_workload(name, rank, world, args.c3_cloths if name == "c3" else 0)
    t0 = time.time()
    plug = build_plugin(w, device)
    setup_s = time.time() - t0
    tuned = apply_schedule(w, plug, args)
    flush = working_set_bytes(w) < L2_BYTES
    steps = args.steps if name == args.workload else args.batched_steps
    total_ms, per, launches, clocks, st = time_device(w, plug, steps, args.warmup, world, device, flush)
    mean_ms = total_ms / steps
    cloth_steps = w["total_cloths"] * steps
    kernel = {0: "jacobi_persistent_kernel", 1: "gs_persistent_kernel", 2: "jacobi_patch_kernel",
              3: "gs_cluster_kernel", 5: "jacobi_row_kernel", 6: "jacobi_converge_kernel",
              7: "jacobi_cloth_kernel", 8: "jacobi_small_batch_kernel", 9: "gs_strip_kernel"}[st["solver_kernel"]]
    res = {
        "value": round(cloth_steps / (total_ms * 1e-3), 2),
        "ms_per_step": round(mean_ms, 4),
        "steps": steps,
        "gpu_launches": launches,
        "config": workload_config(name, world),
        "schedule": {"rank0_cloths": w["cloths"], "rank0_particles": w["n"], "rank0_constraints": w["e"],
                     "colors": st["num_colors"], "block_threads": st["block_threads"],
                     "grid_blocks": st["grid_blocks"], "blocks_per_sm_tuned": tuned.blocks_per_sm,
                     "solver_kernel": kernel, "cluster_ctas": st["cluster_ctas"],
                     "cuda_graph": bool(st["graph_captured"]), "cooperative_launch": bool(st["cooperative_launch"]),
                     "setup_s": round(setup_s, 2)},
        "roofline": roofline(w, mean_ms, kernel, peaks),
        "clocks": clocks,
        "step_ms_min_max": [round(min(per), 4), round(max(per), 4)],
    }
    if with_e2e:
        e2e_ms, _ = time_e2e(w, plug, steps, args.warmup, world)
        res["e2e"] = {"value": round(cloth_steps / (e2e_ms * 1e-3), 2), "unit": UNIT,
                      "h2d_bytes_per_step": DEV_PARAMS_BYTES, "d2h_bytes_per_step": 12 * w["n"],
                      "ms_per_step": round(e2e_ms / steps, 4)}
    if w["cloths"] == 1:
        res["_state"] = (plug.positions(), plug.velocities())
    plug.close()
    res["_w"] = w
    return res


# ------------------------------------------------------------------------------------------------ warm-start leg
def run_warm_leg(args, device: int) -> dict:
    """Config 4: convergence solve, learned vs plain (and previous-substep λ) warm start.

    Per substep, Jacobi (degree-averaged) iterates each cloth until its max residual |C + α̃λ|/rest — the strain
    |‖xi−xj‖−rest|/rest for the rigid (α = 0) constraints — is at or below 1e-4, capped at 4096 passes (the library's
    maximum). Training data: 16 cloths of side 64..256 (config-3 generator, seed 41) simulated for 2,000 frames under
    seeded random wind (0..5 m/s, horizontal, drag 1/s) and random grab displacements (a random vertex pulled up to
    0.3 m from where it is, re-drawn every 100 frames, held for 50); every 20 frames two convergence-solve substeps
    run at 100 iterations (tolerance 0: the 100-iteration λ is the target), the second one's constraints are sampled.
    The MLP (BF16 tensor-core kernels) is fitted with 4000 Adam steps of 4096 samples; the factor that shrinks its
    predicted change toward the previous multiplier (plugin.mlp_scale_change) is chosen on 4 training cloths.
    Measurement: the config-3 batch (256 cloths) plus one 256x256 sheet, `warm_frames` frames per mode after one
    untimed frame from the same initial state: mean passes per cloth-substep, fraction of capped cloth-substeps,
    fallbacks to the plain start, cloth-steps/s timed with CUDA events."""
    import torch

    from bevy_xpbd_b200 import plugin as P
    from bevy_xpbd_b200 import workloads as wl
    cap, tol = 4096, 1e-4
    dt, inv_dt = wl.substep_dt(10)
    prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, cap, linear_drag_per_sec=0.01)
    plain_prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 10, linear_drag_per_sec=0.01)
    collect_prm = P.XpbdCpuTimeStepParams(float(dt), float(inv_dt), 1.0, 100, linear_drag_per_sec=0.01)

    def cfg(warm, t=tol):
        return P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10,
                                tolerance=t, warm_start=warm)

    plain_cfg = P.ClothSimConfig(solver=P.SOLVER_JACOBI, relaxation=P.RELAX_AVERAGE, solve_substeps=10)
    train = wl.config3_batch(seed=41, count=16, side_lo=64, side_hi=256)
    rng = np.random.default_rng(41)
    t0 = time.time()
    tr = P.ClothComputePlugin(device)
    for sp in train:
        tr.add_spec(sp)
    tr.commit()
    tr.mlp_init(seed=1, capacity=1 << 21)
    for k in range(len(train)):
        ang = rng.uniform(0, 2 * np.pi)
        speed = rng.uniform(0.0, 5.0)
        tr.set_cloth_wind(k, (speed * np.cos(ang), 0.0, speed * np.sin(ang)), 1.0)
    frames, every = 2000, 20
    e_total = sum(sp.num_constraints for sp in train)
    # every stride-th constraint of each collected substep, so that the 100 collections fill the 2^21-sample store
    stride = max(1, int(np.ceil(e_total * (frames // every) / (1 << 21))))
    tr.set_params(plain_prm, plain_cfg)
    samples = 0
    for f in range(frames):
        if f % 100 == 0:  # grab a random free vertex of each cloth toward a random displacement
            x = tr.positions()
            for k, sp in enumerate(train):
                free = np.flatnonzero(sp.inv_mass > 0)
                v = int(rng.choice(free))
                g = x[sum(s.num_particles for s in train[:k]) + v] + rng.uniform(-0.3, 0.3, 3)
                tr.set_cloth_grab(k, v, g, 0.28)
        elif f % 100 == 50:
            for k in range(len(train)):
                tr.set_cloth_grab(k, None)
        if f % every == every - 1:
            tr.set_params(collect_prm, cfg(P.WARM_NONE, 1e-30))
            tr.substep(1)                            # establishes the previous substep's λ (a feature)
            samples = tr.mlp_collect(1, stride=stride)
            tr.set_params(plain_prm, plain_cfg)
        else:
            tr.step(frames=1)
    tr.sync()
    tr.mlp_fit_normalization()
    t1 = time.time()
    l1 = tr.mlp_train(3000, batch=4096, lr=2e-3, seed=3)
    l2 = tr.mlp_train(1000, batch=4096, lr=3e-4, seed=4)
    torch.cuda.synchronize()
    t2 = time.time()
    params, norm = tr.mlp_params()
    tr.close()

    def passes_on(specs, p_, n_):  # passes per cloth-substep of the learned start over one frame after one frame
        c = P.ClothComputePlugin(device)
        for sp in specs:
            c.add_spec(sp)
        c.commit()
        c.mlp_init(seed=0, capacity=16)
        c.mlp_set_params(p_, n_)
        c.set_params(prm, cfg(P.WARM_LEARNED))
        c.step(frames=1)
        c.sync()
        a0 = c.stats()
        c.step(frames=1)
        c.sync()
        a1 = c.stats()
        c.close()
        return (a1["converge_iterations"] - a0["converge_iterations"]) / max(
            a1["converge_substeps"] - a0["converge_substeps"], 1)

    # shrink of the predicted change toward the previous multiplier, chosen on 4 of the training cloths
    calib_specs = train[:4]
    calib = {f: round(passes_on(calib_specs, *P.mlp_scale_change(params, norm, f)), 1) for f in (1.0, 0.5, 0.15)}
    factor = min(calib, key=calib.get)
    params, norm = P.mlp_scale_change(params, norm, factor)
    t3 = time.time()
    test = wl.config3_batch() + [wl.config1_sheet()]
    out = {"workload": "config 4: the config-3 batch (256 cloths) plus one 256x256 sheet; trained on 16 cloths of "
                       "side 64..256 under random wind and grabs; tolerance "
                       f"{tol:g} on max |C + a~lambda|/rest, cap {cap} passes per substep, 10 substeps",
           "train": {"frames": frames, "collected_substeps": frames // every, "samples": samples, "stride": stride,
                     "collect_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2), "adam_steps": 4000,
                     "batch": 4096, "loss_first10": round(float(l1[:10].mean()), 4),
                     "loss_last50": round(float(l2[-50:].mean()), 4), "change_scale": factor,
                     "change_scale_passes_on_4_training_cloths": calib, "calibration_s": round(t3 - t2, 2)}}
    n = sum(sp.num_particles for sp in test)
    for name, warm in (("plain", P.WARM_NONE), ("previous", P.WARM_PREVIOUS), ("learned", P.WARM_LEARNED)):
        q = P.ClothComputePlugin(device)
        for sp in test:
            q.add_spec(sp)
        q.commit()
        q.mlp_init(seed=0, capacity=16)
        q.mlp_set_params(params, norm)
        q.set_params(prm, cfg(warm))
        stream = torch.cuda.Stream()
        q.set_stream(stream.cuda_stream)
        q.step(frames=1)
        q.sync()
        s0 = q.stats()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.warm_frames)]
        per = []
        for a, b in evs:
            a.record(stream)
            q.step(frames=1)
            b.record(stream)
            per.append(q.converge_cloth_iterations().astype(np.int64))  # last substep of the frame
        torch.cuda.synchronize()
        s1 = q.stats()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        its = s1["converge_iterations"] - s0["converge_iterations"]
        cs = s1["converge_substeps"] - s0["converge_substeps"]
        last = np.array(per)
        out[name] = {"passes_per_cloth_substep": round(its / max(cs, 1), 2),
                     "capped_frac_last_substeps": round(float((last >= cap).mean()), 4),
                     "fallbacks": int(s1["warm_start_fallbacks"] - s0["warm_start_fallbacks"]),
                     "cloth_steps_per_s": round(len(test) * args.warm_frames / (ms * 1e-3), 2),
                     "ms_per_frame": round(ms / args.warm_frames, 3), "gpu_launches":
                         int(s1["kernel_launches"] - s0["kernel_launches"]), "particles": n, "cloths": len(test)}
        q.set_stream(None)
        q.close()
    p, l_, v_ = out["plain"], out["learned"], out["previous"]
    out["iteration_ratio_plain_over_learned"] = round(p["passes_per_cloth_substep"] /
                                                      max(l_["passes_per_cloth_substep"], 1e-9), 3)
    out["iteration_ratio_previous_over_learned"] = round(v_["passes_per_cloth_substep"] /
                                                         max(l_["passes_per_cloth_substep"], 1e-9), 3)
    out["speed_ratio_learned_over_plain"] = round(l_["cloth_steps_per_s"] / max(p["cloth_steps_per_s"], 1e-9), 3)
    out["targets"] = {"iterations_2x_fewer": out["iteration_ratio_plain_over_learned"] >= 2.0,
                      "cloth_steps_1p5x": out["speed_ratio_learned_over_plain"] >= 1.5}
    return out


# ------------------------------------------------------------------------------------------------ CPU arm
def run_prep_leg(device: int, reps: int = 5) -> dict:
    """Mesh preparation of the c3 batch (256 cloths in one call): greedy coloring and neighbour table on the GPU
    (inputs resident, CUDA events on the stream) against the host coloring on all host threads (one cloth per task,
    as xpbd_commit runs it). The coloring is timed with the cloth ranges given (one CTA per cloth) and without them
    (schedule over the whole grid); the former's colors are checked against the host's."""
    import ctypes as C
    from concurrent.futures import ThreadPoolExecutor

    import torch

    from bevy_xpbd_b200 import _native as N
    from bevy_xpbd_b200 import workloads as wl
    L = N.load()
    specs = wl.config3_batch()
    voff = np.cumsum([0] + [s.num_particles for s in specs])
    n, e = int(voff[-1]), sum(s.num_constraints for s in specs)
    ci = np.concatenate([s.constraint_i + o for s, o in zip(specs, voff)]).astype(np.uint32)
    cj = np.concatenate([s.constraint_j + o for s, o in zip(specs, voff)]).astype(np.uint32)
    dev = f"cuda:{device}"
    st = torch.cuda.current_stream(device)
    sp = C.c_void_p(st.cuda_stream)
    h2d0, h2d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hci = torch.from_numpy(ci.view(np.int32)).pin_memory()
    hcj = torch.from_numpy(cj.view(np.int32)).pin_memory()
    h2d0.record(st)
    dci, dcj = hci.to(dev, non_blocking=True), hcj.to(dev, non_blocking=True)
    h2d1.record(st)
    perm = torch.empty(e, dtype=torch.int32, device=dev)
    colors = torch.empty(e, dtype=torch.int32, device=dev)
    offs = torch.empty(e + 2, dtype=torch.int32, device=dev)
    eoff = np.cumsum([0] + [s.num_constraints for s in specs]).astype(np.uint32)
    cbytes = L.xpbd_color_constraints_device_scratch_bytes(n, e, len(specs))
    tbytes = L.xpbd_neighbor_table_device_scratch_bytes(n, e)
    scratch = torch.empty(max(cbytes, tbytes), dtype=torch.uint8, device=dev)
    row = torch.empty(n + 1, dtype=torch.int32, device=dev)
    other = torch.empty(2 * e, dtype=torch.int32, device=dev)
    eid = torch.empty(2 * e, dtype=torch.int32, device=dev)
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    bc = C.c_uint32()

    def color(per_cloth=True):
        nc = len(specs) if per_cloth else 0
        r = L.xpbd_color_constraints_device(n, e, vp(dci), vp(dcj), 0, nc, eoff.ctypes.data if nc else None,
                                            vp(perm), vp(colors), vp(offs), C.byref(bc), vp(scratch), cbytes, sp)
        if r != 0:
            raise RuntimeError(f"xpbd_color_constraints_device: {r}")

    def table():
        r = L.xpbd_neighbor_table_device(n, e, vp(dci), vp(dcj), vp(row), vp(other), vp(eid), vp(scratch), tbytes, sp)
        if r != 0:
            raise RuntimeError(f"xpbd_neighbor_table_device: {r}")

    def timed(fn):
        ts = []
        for k in range(reps + 2):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize(device)
            a.record(st)
            fn()
            b.record(st)
            torch.cuda.synchronize(device)
            if k >= 2:
                ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    grid_ms = timed(lambda: color(False))
    color_ms = timed(color)  # the per-cloth schedule (cloth ranges given): its colors are checked below
    table_ms = timed(table)
    # host coloring, one cloth per task on every host thread

    def host_one(k):
        s = specs[k]
        a = np.ascontiguousarray(s.constraint_i, np.uint32)
        b = np.ascontiguousarray(s.constraint_j, np.uint32)
        pm = np.zeros(s.num_constraints, np.uint32)
        of = np.zeros(s.num_constraints + 2, np.uint32)
        nb = C.c_uint32()
        L.xpbd_color_constraints(s.num_particles, s.num_constraints, a.ctypes.data, b.ctypes.data, 0, pm.ctypes.data,
                                 of.ctypes.data, C.byref(nb))
        return pm, of[: nb.value + 1]

    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        host = list(ex.map(host_one, range(len(specs))))
    host_ms = (time.perf_counter() - t0) * 1e3
    gcol = colors.cpu().numpy().view(np.uint32)
    for k, (pm, of) in enumerate(host):
        mine = gcol[eoff[k]:eoff[k + 1]][pm]
        if np.any(np.diff(mine.astype(np.int64)) < 0) or not np.array_equal(np.searchsorted(mine, np.arange(len(of)), side="left"), of):
            raise RuntimeError(f"device coloring differs from the host coloring on cloth {k}")
    return {"workload": f"c3: {len(specs)} cloths in one call, {n} particles, {e} constraints",
            "device_color_ms": round(color_ms, 2), "device_color_ms_whole_grid_schedule": round(grid_ms, 2),
            "device_neighbor_table_ms": round(table_ms, 2),
            "h2d_ms": round(h2d0.elapsed_time(h2d1), 2), "host_color_ms": round(host_ms, 1),
            "host_threads": threads, "batches": bc.value, "identical_to_host": True}


def cpu_oracle_run(w: dict, budget_s: float, max_cloths: int | None = None, min_frames: int = 1,
                   variant: str = "omp", warmup_frames: int = 1, state=None):
    """Times the CPU restatement of xpbd_cpu.rs (OpenMP build, or the serial build with the reference's loop order)
    on a bounded sample of workload `w`: every `len/max_cloths`-th cloth, as many whole frames as fit in `budget_s`
    (at least `min_frames`), after `warmup_frames` untimed frames. `state` = (positions, velocities) of a one-cloth
    workload to start from (the GPU arm's state after its untimed frames)."""
    from oracle import oracle as orc
    from tests.helpers import oracle_params
    orc.select(variant)
    specs = w["specs"]
    if max_cloths is not None and len(specs) > max_cloths:
        specs = specs[:: len(specs) // max_cloths][:max_cloths]
    sims = []
    for sp in specs:
        perm, _, offs = orc.partition(sp.num_particles, sp.constraint_i, sp.constraint_j)
        s = orc.OracleSim(sp.positions, sp.inv_mass, sp.constraint_i[perm], sp.constraint_j[perm],
                          sp.rest_len[perm], sp.compliance[perm], v=sp.velocities, rest_pos=sp.rest_positions,
                          ctype=sp.constraint_type[perm])
        s.set_params(oracle_params(w["params"], w["cfg"]))
        s.set_batches(offs)
        if state is not None and len(specs) == 1:
            s.set_state(state[0], state[1])
        sims.append(s)
    S = w["cfg"].solve_substeps
    for _ in range(max(warmup_frames, 1) - 1):  # untimed warm-up frames
        for s in sims:
            s.substeps(S)
    t0 = time.perf_counter()
    for s in sims:  # the last untimed frame also gives the per-frame estimate
        s.substeps(S)
    per_frame = time.perf_counter() - t0
    frames = max(min_frames, int(budget_s / max(per_frame, 1e-6)))
    t0 = time.perf_counter()
    for _ in range(frames):
        for s in sims:
            s.substeps(S)
    t1 = time.perf_counter()
    return dict(value=len(sims) * frames / (t1 - t0), frames=frames, cloths=len(sims), seconds=t1 - t0,
                cores=orc.threads() if variant == "omp" else 1, per_frame_s=(t1 - t0) / frames)


def run_reference(args, rank: int, world: int):
    """CPU restatement of the reference solver on all host cores; rank 0 only (other ranks exit without work)."""
    if rank != 0:
        return
    w = make_workload(args.workload, 0, 1)
    max_cloths = 16 if args.workload == "c3" else None
    res = cpu_oracle_run(w, budget_s=0.0, max_cloths=max_cloths, min_frames=args.steps, warmup_frames=args.warmup)
    sample = (f"{res['frames']} frames of {res['cloths']} of the workload's {len(w['specs'])} cloths"
              if max_cloths else f"{res['frames']} frames of the workload")
    line = {"metric": METRIC, "value": round(res["value"], 4), "unit": UNIT, "n_gpus": world,
            "steps": res["frames"], "warmup": max(args.warmup, 1), "ms_per_step": round(res["per_frame_s"] * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "impl": "reference",
            "data": "synthetic: seeded procedural sheets (no dataset)",
            "config": workload_config(args.workload, world),
            "cpu_baseline": {"value": round(res["value"], 4), "unit": UNIT, "cores": res["cores"], "kind": "port",
                             "sample": sample + ", OpenMP build of the oracle"},
            "e2e": {"value": round(res["value"], 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c0", "c1", "c2", "c3"])
    ap.add_argument("--batched-steps", type=int, default=30)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-warm", action="store_true", help="skip the learned-vs-plain convergence leg")
    ap.add_argument("--warm-frames", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="skip the c0 and c2 legs")
    ap.add_argument("--no-prep", action="store_true", help="skip the mesh-preparation leg (GPU vs host coloring)")
    ap.add_argument("--c3-cloths", type=int, default=0, help="first K cloths of c3 only (profiling cases)")
    ap.add_argument("--no-autotune", action="store_true", help="library default schedule")
    ap.add_argument("--jacobi-kernel", type=int, default=None, help="1 warp tiles, 2 spatial patches, 3 rows")
    ap.add_argument("--block", type=int, default=None)
    ap.add_argument("--bps", type=int, default=None)
    ap.add_argument("--cluster", type=int, default=None, help="Gauss-Seidel cluster size (0 = grid kernel)")
    ap.add_argument("--gs-strips", type=int, default=None, help="Gauss-Seidel over this many clusters (strips)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":  # CPU only, rank 0 alone: no process group needed
        run_reference(args, int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, world, local = dist_setup()
    import torch
    torch.cuda.set_device(local)
    peaks = load_peaks()
    main_res = run_gpu_workload(args.workload, args, rank, world, local, peaks, with_e2e=not args.no_e2e)
    w = main_res.pop("_w")
    main_state = main_res.pop("_state", None)
    line = {"metric": METRIC, "value": main_res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": main_res["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded procedural sheets (no dataset)", "config": main_res["config"],
            "schedule": main_res["schedule"],
            "roofline": main_res["roofline"], "e2e": main_res.get("e2e"), "gpu_launches": main_res["gpu_launches"],
            "clocks": main_res["clocks"], "step_ms_min_max": main_res["step_ms_min_max"],
            "substeps_per_s": round(main_res["value"] * w["cfg"].solve_substeps, 1)}
    if not args.no_batched and args.workload != "c3":
        b = run_gpu_workload("c3", args, rank, world, local, peaks, with_e2e=False)
        b.pop("_w")
        line["batched"] = {"value": b["value"], "unit": UNIT, "ms_per_step": b["ms_per_step"], "steps": b["steps"],
                           "substeps_per_s": round(b["value"] * 10, 1),
                           "config": b["config"], "schedule": b["schedule"], "roofline": b["roofline"],
                           "gpu_launches": b["gpu_launches"],
                           "clocks": b["clocks"]}
    if world == 1 and not args.no_legs:
        # the other single-sheet configurations: 32x32 Jacobi (c0) and the 512x512 self-collision sheet (c2)
        for name in ("c0", "c2"):
            if name == args.workload:
                continue
            r = run_gpu_workload(name, args, rank, world, local, peaks, with_e2e=True)
            wx = r.pop("_w")
            stx = r.pop("_state", None)
            leg = {k: r[k] for k in ("value", "ms_per_step", "steps", "config", "schedule", "roofline", "e2e",
                                     "gpu_launches", "clocks")}
            leg["unit"] = UNIT
            if not args.no_cpu_baseline:
                c = cpu_oracle_run(wx, args.cpu_seconds / 2, state=stx)
                leg["cpu_baseline"] = {"value": round(c["value"], 4), "unit": UNIT, "cores": c["cores"],
                                       "kind": "port",
                                       "sample": f"{c['frames']} frames, {c['seconds']:.1f} s, OpenMP build of the "
                                                 "oracle" + (", from the GPU arm's final state" if stx else "")}
            line[name] = leg
    if rank == 0 and world == 1 and not args.no_warm:
        line["warm_start"] = run_warm_leg(args, local)
    if rank == 0 and world == 1 and not args.no_prep:
        line["mesh_prep"] = run_prep_leg(local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_oracle_run(w, args.cpu_seconds, max_cloths=16 if args.workload == "c3" else None,
                           state=main_state if args.workload == "c2" else None)
        line["cpu_baseline"] = {"value": round(r["value"], 4), "unit": UNIT, "cores": r["cores"], "kind": "port",
                                "sample": f"{r['frames']} frames of {r['cloths']} cloth(s) of the workload, "
                                          f"{r['seconds']:.1f} s, OpenMP build of the oracle"}
        r1 = cpu_oracle_run(w, args.cpu_seconds / 3, max_cloths=16 if args.workload == "c3" else None,
                            variant="serial")
        line["cpu_baseline_serial"] = {"value": round(r1["value"], 4), "unit": UNIT, "cores": 1, "kind": "port",
                                       "sample": f"{r1['frames']} frames of {r1['cloths']} cloth(s), "
                                                 f"{r1['seconds']:.1f} s, serial build (the reference's loop order)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
