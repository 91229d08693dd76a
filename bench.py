"""Benchmark: body-steps/s of the AVBD step on the 65,536-box stack grid, with the batched
(4,096 uneven worlds) and differentiable (1,000-box tower, bwd/fwd) forms in the same line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl cuda|reference]

A step is one Solver::step of the whole scene (broadphase, narrowphase, warm start,
10 coloured primal/dual iterations, velocities), device-resident. Each rank runs an
independent replica of the scene (the single-world step does not shard: "replicas
only"); value = bodies x steps summed over ranks / slowest rank's time.

--impl reference times the reference's own CPU solver (built from its sources into
oracle/_ref; the C oracle port stands in if that library is absent) on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from avbd_demo3d_b200.sharding import max_over_ranks  # noqa: E402

METRIC = "body-steps/s at 65k boxes"
UNIT = "body-steps/s"
GRID = (64, 64, 16)
SEED = 1
WORKLOAD = "stack grid 64x64x16 = 65,536 boxes + ground (seed 1); dt 1/60, 10 iterations, alpha 0.99, " \
           "gamma 0.99, betaLin 1e5, g -9.81"
L2_FLUSH_BYTES = 256 << 20


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from one ncu capture
# of the kernel on this workload, with the capture's summary file and date, the commit the
# capture ran on and a digest of the kernel sources' code at capture time
# (kernel_sources_sha, comments left out): when the code has changed since, the figure no
# longer describes the kernel and the line reports no traffic.
NCU_TRAFFIC = {
    "k_iterations": {"bytes_per_launch": 30868224, "summary": "profiles/iterations_stacks65k_ncu.txt",
                     "captured": "2026-12-04", "commit": "9466f58", "sources_sha": "6b8145f7b8c71b4a"},
    "k_iterations_batched": {"bytes_per_launch": 9873686000, "summary": "profiles/iterations_batched4096_ncu.txt",
                             "captured": "2026-12-04", "commit": "64ded38", "sources_sha": "6b8145f7b8c71b4a"},
    "k_primal": {"bytes_per_launch": None, "summary": "profiles/primal_stacks65k_ncu.txt",
                 "captured": "2026-12-04", "sources_sha": ""},
}
KERNEL_SOURCES = ("avbd_demo3d_b200/csrc/avbd_kernels.cuh", "avbd_demo3d_b200/csrc/avbd_math.cuh",
                  "avbd_demo3d_b200/csrc/avbd_round.cuh", "avbd_demo3d_b200/csrc/avbd_colour.cuh")


def code_only(text: str) -> str:
    """C/C++/CUDA source with its comments removed (string and character literals kept) and
    trailing whitespace and blank lines dropped: what the compiler sees, so that a capture
    stays matched across comment edits."""
    out, i, n = [], 0, len(text)
    while i < n:
        c = text[i]
        if c in "\"'":
            j = i + 1
            while j < n and text[j] != c:
                j += 2 if text[j] == "\\" else 1
            out.append(text[i:j + 1])
            i = j + 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    lines = (line.rstrip() for line in "".join(out).split("\n"))
    return "\n".join(line for line in lines if line)


def kernel_sources_sha(read=None) -> str:
    """Hash of the kernel sources' code (comments and blank lines left out); `read(path)`
    gives a file's text (default: the working tree)."""
    import hashlib

    read = read or (lambda f: open(os.path.join(ROOT, f), encoding="utf-8").read())
    h = hashlib.sha256()
    for f in KERNEL_SOURCES:
        h.update(code_only(read(f)).encode())
    return h.hexdigest()[:16]


def ncu_traffic(kernel: str):
    """(bytes per launch or None, provenance) of the kernel's recorded ncu capture."""
    rec = NCU_TRAFFIC.get(kernel)
    if not rec:
        return None, None
    current = rec["sources_sha"] == kernel_sources_sha()
    prov = {"summary": rec["summary"], "captured": rec["captured"], "commit": rec.get("commit"),
            "matches_current_source": current}
    return (rec["bytes_per_launch"] if current else None), prov


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 8:
                self.rows.append(parts)

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def algorithmic_primal_bytes(world) -> tuple[int, dict]:
    """Bytes one primal iteration must move (per-colour launches summed): 128 per solved body
    (100 B state read + 28 B pose write), 164 per contact row incidence on a dynamic body
    (108 B row + 56 B partner pose/initial), 176 per joint and 96 per spring incidence."""
    m = world.manifolds()
    mass = world.props["mass"]
    dyn = mass > 0
    ab = m["ab"]
    n_rows = m["n"].astype(np.int64)
    ic = int((n_rows * dyn[ab[:, 0]]).sum() + (n_rows * dyn[ab[:, 1]]).sum())
    j = world.joints()
    ij = int(sum(dyn[a] for a in j["ab"][:, 0] if a >= 0) + dyn[j["ab"][:, 1]].sum()) if len(j["ab"]) else 0
    sab = world._force_arrays["s_ab"]
    isp = int(dyn[sab[:, 0]].sum() + dyn[sab[:, 1]].sum()) if len(sab) else 0
    solved = int(world.stats()["solved_bodies"])
    per_iter = 128 * solved + 164 * ic + 176 * ij + 96 * isp
    return per_iter, {"solved_bodies": solved, "contact_incidences": ic, "joint_incidences": ij,
                      "spring_incidences": isp, "contacts": int(n_rows.sum()), "manifolds": int(len(n_rows))}


def run_cuda(args):
    import torch
    import torch.distributed as dist

    from avbd_demo3d_b200 import World, scenes

    rank, world_size, local = dist_env()
    torch.cuda.set_device(local)
    if world_size > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    scene = scenes.stack_grid(*GRID, seed=SEED)
    stream = torch.cuda.Stream(device=local)
    w = World(scene, device=local, stream=stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    w.step(args.warmup)
    w.set_iteration_mode(args.iteration_mode)
    if args.primal_variant >= 0:  # fixed variant (profiling captures), no sweep
        tuned, variant_us = args.primal_variant, []
        w.set_primal_variant(tuned)
    else:
        tuned, variant_us = w.autotune(3)  # pick the primal variant on this scene's colouring

    # ---- timed region: device-resident step, L2 flushed before every step
    w.set_profiling(True)
    w.reset_profile()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world_size > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                starts[k].record(stream)
            w.step(1, sync=False)
            with torch.cuda.stream(stream):
                ends[k].record(stream)
        torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    prof = w.profile()
    w.set_profiling(False)
    max_ms = max_over_ranks(total_ms, device=f"cuda:{local}")
    bodies = scene.n_bodies - 1  # the static ground is not counted
    value = world_size * bodies * args.steps / (max_ms / 1e3)

    # ---- roofline of the dominant kernel: the iteration kernel (one launch per step) or, in
    # the per-colour form, the coloured primal sweep
    per_iter, counts = algorithmic_primal_bytes(w)
    iters = scene.params.iterations
    persistent = w.iteration_mode() == 1
    if persistent:  # each contact's dual update also writes its multiplier and penalties (32 B)
        per_iter += 32 * counts["contacts"]
    primal_ms = prof["primal_ms"]
    primal_launches = max(1, prof["primal_spans"])
    achieved = per_iter * iters * prof["steps"] / (primal_ms / 1e3) / 1e9 if primal_ms > 0 else None
    peak, peak_kind = measured_peak()
    traffic, traffic_source = ncu_traffic("k_iterations" if persistent else "k_primal")
    kernel = ("k_iterations (every iteration of a step: coloured primal sweeps, contact dual updates fused into "
              "the rows, joint dual updates)" if persistent else "k_primal (coloured primal sweep, one launch per "
              "colour)")
    roofline = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "traffic_source": traffic_source,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "algorithmic_bytes_per_launch": per_iter * iters * prof["steps"] / primal_launches,
                "avg_launch_us": primal_ms * 1e3 / primal_launches, "launches": primal_launches,
                "iteration_mode": "one launch per step" if persistent else "one launch per colour", **counts}
    phases = {k[:-3]: round(v / max(1, prof["steps"]), 4) for k, v in prof.items() if k.endswith("_ms")}
    # the whole step against the same peak: the iterations' bytes plus the setup phases'
    # (broadphase N (40 + 16 x 3 sort passes), narrowphase and force warm start 120 per
    # manifold + 216 per contact, body warm start and velocities 176 per body)
    setup_bytes = bodies * (40 + 16 * 3) + 120 * counts["manifolds"] + 216 * counts["contacts"] + 176 * bodies
    step_bytes = per_iter * iters + setup_bytes
    step_gbs = step_bytes / (max_ms / args.steps / 1e3) / 1e9
    roofline["whole_step"] = {"algorithmic_bytes": step_bytes, "setup_bytes": setup_bytes,
                              "ms": max_ms / args.steps, "achieved": step_gbs, "frac": step_gbs / peak}
    st_now = w.stats()

    # ---- end to end through the C ABI with host buffers (H2D state, step, D2H state)
    st = w.bodies()
    # the caller's arrays in page-locked memory (allocated once, reused every step): the
    # library copies them to and from the device directly
    pinned = {k: torch.empty(v.shape, dtype=torch.float32, pin_memory=True) for k, v in st.items()}
    host = {k: t.numpy() for k, t in pinned.items()}
    for k in host:
        host[k][...] = st[k]
    h2d = sum(host[k].nbytes for k in ("pos", "quat", "vel", "angvel", "prevvel"))
    e2e_steps = max(3, args.steps)
    torch.cuda.synchronize()
    if world_size > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        w.write_bodies(pos=host["pos"], quat=host["quat"], vel=host["vel"], angvel=host["angvel"],
                       prevvel=host["prevvel"])
        w.step(1, sync=False)
        w.bodies(out=host)  # the caller's arrays, reused from step to step
    e2e_s = time.perf_counter() - t0
    d2h = sum(host[k].nbytes for k in ("pos", "quat", "vel", "angvel", "prevvel"))
    e2e_max = max_over_ranks(e2e_s, device=f"cuda:{local}")
    e2e = {"value": world_size * bodies * e2e_steps / e2e_max, "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": e2e_steps,
           "path": "avbd_write_bodies (a kernel reads the caller's page-locked arrays in place over the bus) + "
                   "avbd_step + avbd_read_bodies (a kernel writes them in place); arrays allocated once, reused "
                   "every step; host timer"}

    # the end of the configuration's 300 steps, timed the same way (the stacks have settled)
    late = None
    if not args.no_late:
        done_steps = args.warmup + args.steps + e2e_steps
        w.step(max(0, 280 - done_steps))
        late_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        torch.cuda.synchronize()
        for a_ev, b_ev in late_ev:
            with torch.cuda.stream(stream):
                flush.fill_(2.0)
                a_ev.record(stream)
            w.step(1, sync=False)
            with torch.cuda.stream(stream):
                b_ev.record(stream)
        torch.cuda.synchronize()
        late_ms = max_over_ranks(sum(a_ev.elapsed_time(b_ev) for a_ev, b_ev in late_ev),
                                 device=f"cuda:{local}") / 20
        late = {"steps": f"{max(done_steps, 280) + 1}-{max(done_steps, 280) + 20}", "ms_per_step": late_ms,
                "value": world_size * bodies * 1e3 / late_ms, "manifolds": int(w.stats()["manifold_count"])}
    collision = collision_only(w, scene, rank, world_size, local, reference=not args.no_cpu_baseline)
    w.close()
    lbvh = lbvh_line(args, local, stream) if (rank == 0 and not args.no_lbvh) else None

    cpu, fp64 = None, None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scene)
        if not args.no_fp64:  # after the timed CPU baseline, so as not to share its cores
            fp64 = CpuFp64Reference()
    batched = batched_line(args, rank, world_size, local, stream) if not args.no_batched else None
    adjoint = adjoint_line(args, local, stream) if (rank == 0 and not args.no_adjoint) else None
    mixed = mixed_line(args, local, stream, reference=cpu is not None) \
        if (rank == 0 and not args.no_mixed) else None
    if fp64 is not None:
        cpu["err_vs_fp64"] = fp64.result(local, stream)
    if world_size > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "bodies_per_gpu": bodies, "parallelism": f"replicas x{world_size}",
                           "l2": "flushed before every timed step (256 MiB device write)",
                           "timing": "CUDA events on the solver stream, summed per step, max over ranks"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks.summary(),
                "gpu_launches": prof["launches"], "phases_ms_per_step": phases, "batched": batched,
                "adjoint": adjoint, "collision_only": collision, "mixed200k": mixed, "lbvh_mode": lbvh,
                "late_window": late,
                "autotune": {"primal_variant": World.primal_variants()[tuned],
                             "sweep_us": [round(float(x), 1) for x in variant_us]},
                "step_ms_min_max": [min(step_ms), max(step_ms)],
                "device_steps": {"issued": int(st_now["device_steps"]), "redone_on_host": int(st_now["redone_steps"]),
                                 "note": "steps run with every count on the device; a step that stops on the "
                                         "device is redone synchronously and counted here"}}
        print(json.dumps(line), flush=True)


def lbvh_line(args, local, stream, steps: int = 10):
    """The same 65,536-box scene with the sorted-Morton LBVH broadphase mode (the grid's pair
    set and creation order, binned candidates from the tree): ms per step and per phase
    (CUDA events on the solver stream, L2 flushed before each step), and whether the state
    after the steps equals the grid mode's bit for bit."""
    import copy

    import torch

    from avbd_demo3d_b200 import World, scenes

    scene = scenes.stack_grid(*GRID, seed=SEED)
    out = {}
    states = {}
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    for mode, name in ((scenes.BROADPHASE_LBVH, "lbvh"), (scenes.BROADPHASE_GRID, "grid")):
        w = World(scene, device=local, stream=stream.cuda_stream)
        p = copy.copy(scene.params)
        p.broadphase = mode
        w.set_params(p)
        w.step(max(3, args.warmup))
        w.set_profiling(True)
        w.reset_profile()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        for a, b in ev:
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
                a.record(stream)
            w.step(1, sync=False)
            with torch.cuda.stream(stream):
                b.record(stream)
        torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        prof = w.profile()
        w.set_profiling(False)
        states[name] = w.bodies()
        out[name] = {"ms_per_step": ms, "broadphase_ms": prof["broadphase_ms"] / max(1, prof["steps"])}
        w.close()
    out["same_bits_as_grid"] = all(np.array_equal(states["lbvh"][k].view(np.uint32), states["grid"][k].view(np.uint32))
                                   for k in states["grid"])
    out["steps"] = steps
    return out


def collision_only(w, scene, rank, world_size, local, reference: bool, frames: int = 10):
    """The reference's collision-only benchmark frame (Solver::benchmarkBroadphaseOnly: drop
    every manifold, run the grid broadphase alone) on the same scene, after the timed steps;
    host timer around the C-ABI call, which waits for its result. The reference's own CPU
    frame is timed beside it on the same state (rank 0, one process, 2 frames)."""
    import torch

    w.broadphase_only()  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(frames):
        w.broadphase_only()
    dt = max_over_ranks((time.perf_counter() - t0) / frames, device=f"cuda:{local}")
    st = w.stats()
    out = {"ms_per_frame": dt * 1e3, "bodies_per_s": world_size * (scene.n_bodies - 1) / dt,
           "new_pairs": int(st["manifold_count"]), "pair_checks": int(st["pair_checks"]), "frames": frames}
    if reference and rank == 0:
        with REFERENCE_LOCK:
            ref, kind = reference_world(scene)
            ref.step(1)
            t0 = time.perf_counter()
            for _ in range(2):
                ref.broadphase_only()
            ref_ms = (time.perf_counter() - t0) / 2 * 1e3
        out["cpu_reference"] = {"ms_per_frame": ref_ms, "kind": kind,
                                "cores": cpu_cores(kind),
                                "state": "the scene after one step (the GPU frames ran on the state after the "
                                         "timed steps; the pair count is of the same order)"}
    return out


def batched_line(args, rank, world_size, local, stream):
    """World-steps/s of the 4,096-world uneven batch against looping the plain single-world
    step over a sample of the same worlds (one resident context per world). With N ranks the
    worlds are sharded (size-balanced) and each rank steps its shard in one context; the
    time is the slowest rank's."""
    import torch
    import torch.distributed as dist

    from avbd_demo3d_b200 import World, scenes
    from avbd_demo3d_b200.sharding import shard_worlds

    all_worlds = scenes.batched_worlds(4096, seed=3)
    shard = shard_worlds([sc.n_bodies for sc in all_worlds], world_size)[rank]
    worlds = [all_worlds[i] for i in shard]
    w = World(worlds, device=local, stream=stream.cuda_stream)
    w.step(max(3, args.warmup))
    steps = max(3, min(args.steps, 10))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world_size > 1:
        dist.barrier()
    w.set_profiling(True)
    w.reset_profile()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    w.step(steps, sync=False)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    batched_s = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, device=f"cuda:{local}")
    n_bodies = int(sum(sc.n_bodies - 1 for sc in all_worlds))
    # the iteration kernel of the whole batch, against the same peak (counts at the end)
    prof = w.profile()
    w.set_profiling(False)
    per_iter, counts = algorithmic_primal_bytes(w)
    per_iter += 32 * counts["contacts"]
    iters = worlds[0].params.iterations
    it_s = prof["primal_ms"] / max(1, prof["steps"]) / 1e3
    peak, _ = measured_peak()
    achieved = per_iter * iters / it_s / 1e9 if it_s > 0 else None
    traffic, traffic_source = ncu_traffic("k_iterations_batched")
    batched_roofline = {"kernel": "k_iterations (all worlds in one launch)", "bound": "hbm", "achieved": achieved,
                        "peak": peak, "unit": "GB/s", "frac": achieved / peak if achieved else None,
                        "traffic": traffic, "traffic_source": traffic_source,
                        "algorithmic_bytes_per_launch": per_iter * iters, "avg_launch_us": it_s * 1e6, **counts,
                        "phases_ms_per_step": {k[:-3]: round(v / max(1, prof["steps"]), 4) for k, v in prof.items()
                                               if k.endswith("_ms")}}
    w.close()
    # loop baseline: the plain step looped over a sample of this rank's worlds, each resident
    sample = worlds[:: max(1, len(worlds) // 128)][:128]
    ctxs = [World(sc, device=local, stream=stream.cuda_stream) for sc in sample]
    for c in ctxs:
        c.step(3)
    loop_steps = 3
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    for _ in range(loop_steps):
        for c in ctxs:
            c.step(1, sync=False)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    loop_s = ev0.elapsed_time(ev1) / 1e3
    for c in ctxs:
        c.close()
    batched_rate = len(all_worlds) * steps / batched_s
    # the looped plain step would run on every rank too
    loop_rate = world_size * len(sample) * loop_steps / max_over_ranks(loop_s, device=f"cuda:{local}")
    return {"metric": "world-steps/s", "worlds": len(all_worlds), "bodies": n_bodies, "steps": steps,
            "value": batched_rate, "ms_per_step": batched_s * 1e3 / steps,
            "body_steps_per_s": n_bodies * steps / batched_s,
            "sharding": f"{world_size} rank(s), size-balanced; {len(worlds)} worlds on rank {rank}",
            "loop_plain_step": {"value": loop_rate, "sample_worlds": len(sample), "steps": loop_steps},
            "speedup_vs_loop": batched_rate / loop_rate, "roofline": batched_roofline,
            "workload": "4,096 worlds, box counts log-uniform in [8, 2048] (seed 3): stack fields, jointed "
                        "chains and drop piles, one ground each; same solver parameters"}


def adjoint_line(args, local, stream):
    """Differentiable step on the 1,000-box tower (10 x 10 stacks x 10 high, seed 4): 120 steps
    at 10 iterations, a checkpoint every 10 steps, loss |COM(x_120) - target|^2. Times the
    plain forward (avbd_step), the taping forward (avbd_adjoint_forward) and the backward
    (avbd_adjoint_backward) with a host timer around the C-ABI calls, and checks the gradient
    against FP64 central differences (h = 1e-4, 32 seeded unit directions over initial
    velocities, angular velocities, masses and per-pair friction) of the frozen-branch
    replay recorded by the oracle's bit-identical FP32 run."""
    import torch

    from avbd_demo3d_b200 import World, scenes
    from avbd_demo3d_b200.solver import box_properties

    scene = scenes.tower(10, 10, 10, seed=4)
    T, every = 120, 10
    mass = np.ascontiguousarray(box_properties(scene.size, scene.density)[0][::-1]).astype(np.float64)
    dyn = mass > 0
    M = float(mass[dyn].sum())
    pos0 = np.ascontiguousarray(scene.pos[::-1]).astype(np.float64)
    com0 = (mass[dyn, None] * pos0[dyn]).sum(0) / M
    target = com0 + np.random.default_rng(7).uniform(-1, 1, 3)

    def clock(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    fwd, afwd, bwd = [], [], []
    grad = None
    for rep in range(4):  # the first repetition warms up and is not counted
        w = World(scene, device=local, stream=stream.cuda_stream)
        f_s, _ = clock(lambda: w.step(T))
        w.close()
        w = World(scene, device=local, stream=stream.cuda_stream)
        a_s, _ = clock(lambda: w.adjoint_forward(T, every))
        final = w.adjoint_replay_state()["pos"]
        com = (mass[dyn, None] * final[dyn]).sum(0) / M
        r = com - target
        dpos = np.zeros_like(final)
        dpos[dyn] = 2.0 * r[None, :] * (mass[dyn, None] / M)
        b_s, g = clock(lambda: w.adjoint_backward(d_pos=dpos))
        w.close()
        if rep:
            fwd.append(f_s)
            afwd.append(a_s)
            bwd.append(b_s)
        dmass = np.zeros(len(mass))
        dmass[dyn] = 2.0 * ((final[dyn] - com) @ r) / M
        grad = np.concatenate([(g["vel"] + g["prevvel"]).ravel(), g["angvel"].ravel(), g["mass"] + dmass,
                               g["pair_friction"]])
    f_s, a_s, b_s = (statistics.median(x) for x in (fwd, afwd, bwd))
    # roofline of the forward + backward pair against the same peak. Bytes per step: the
    # FP32 forward's iteration bytes; the backward replays each iteration in FP64 (twice the
    # FP32 bytes), reads the stored per-iteration snapshots and factors (64 B per solved
    # body and per contact slot, 224 B of factors per solved body) and reads and writes the
    # FP64 adjoints of the same rows (twice the FP32 bytes again).
    wr = World(scene, device=local, stream=stream.cuda_stream)
    wr.step(T // 2)
    per_iter, counts = algorithmic_primal_bytes(wr)
    wr.close()
    per_iter += 32 * counts["contacts"]
    iters = scene.params.iterations
    fwd_bytes = per_iter * iters * T
    bwd_bytes = iters * T * (4 * per_iter + (64 + 224) * counts["solved_bodies"] + 64 * 8 * counts["manifolds"])
    peak, _ = measured_peak()
    ach = (fwd_bytes + bwd_bytes) / (a_s + b_s) / 1e9
    adjoint_roofline = {"form": "taping forward + backward", "bound": "hbm", "achieved": ach, "peak": peak,
                        "unit": "GB/s", "frac": ach / peak, "algorithmic_bytes": fwd_bytes + bwd_bytes,
                        "counts_at_step": T // 2, **counts}
    out = {"workload": "tower 10x10x10 = 1,000 boxes + ground (seed 4), 120 steps, 10 iterations, checkpoint "
                       "every 10 steps; loss |COM(x_120) - target|^2, target = COM_0 + U[-1,1]^3 (seed 7)",
           "forward_ms": f_s * 1e3, "adjoint_forward_ms": a_s * 1e3, "backward_ms": b_s * 1e3,
           "bwd_over_fwd": b_s / f_s, "fwd_plus_bwd_over_fwd": (a_s + b_s) / f_s,
           "timing": "host timer around the C-ABI calls (the step itself reads a few counts per step), "
                     "median of 3 after one warm-up", "params": int(grad.size), "roofline": adjoint_roofline}
    if not args.no_adjoint_check:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import checkers

        ref = checkers.World(scene, "oracle", order_mode=1)
        ref.tape_begin()
        ref.step(T)
        th = ref.adj_theta0()
        n = ref.n
        mask = np.zeros(th.size, bool)
        mask[:3 * n] = np.repeat(dyn, 3)
        mask[3 * n:6 * n] = np.repeat(dyn, 3)
        mask[6 * n:7 * n] = dyn
        mask[7 * n:] = True
        dirs = np.random.default_rng(1).standard_normal((32, th.size)) * mask
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        fd = ref.adj_fd(th, target, dirs, h=1e-4)
        t0 = time.perf_counter()
        _, rg = ref.adj_gradient(th, target)
        ref_s = time.perf_counter() - t0
        ad = dirs @ grad
        out["check"] = {"fd_directions": 32, "fd_h": 1e-4,
                        "max_rel_err_vs_fd": float((np.abs(ad - fd) / np.abs(fd)).max()),
                        "rel_err_vs_reference_adjoint": float(np.linalg.norm(grad - rg) / np.linalg.norm(rg)),
                        "cpu_reference_adjoint_s": ref_s, "cpu_reference_cores": 1}
    return out


def _rot_apply(q, v):
    """Rotate vectors v by unit quaternions q = (x, y, z, w), in double precision."""
    q = np.asarray(q, np.float64)
    v = np.asarray(v, np.float64)
    u, w = q[:, :3], q[:, 3:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def scene_checks(scene, bodies) -> dict:
    """The reference's long-run checks on one state (bodies in list order), in double
    precision: the largest ground penetration of a dynamic box (the ground top is the
    highest static box top, clearance = z - the box's vertical extent - ground top, values
    within 1e-5 count as 0; headless_server.cpp:395-490) and the largest ball-joint
    position error |x_A + R_A r_A - (x_B + R_B r_B)| (the linear constraint C of
    Joint::updatePrimal, joint.cpp:61-64)."""
    from avbd_demo3d_b200.solver import box_properties

    n = scene.n_bodies
    mass = box_properties(scene.size, scene.density)[0][::-1]
    size = np.asarray(scene.size, np.float64)[::-1]
    pos = np.asarray(bodies["pos"], np.float64)
    q = np.asarray(bodies["quat"], np.float64)
    static = mass <= 0
    ground_top = float((pos[static, 2] + 0.5 * size[static, 2]).max()) if static.any() else 0.0
    dyn = ~static
    ez = (np.abs(2 * (q[:, 0] * q[:, 2] - q[:, 3] * q[:, 1])) * 0.5 * size[:, 0] +
          np.abs(2 * (q[:, 1] * q[:, 2] + q[:, 3] * q[:, 0])) * 0.5 * size[:, 1] +
          np.abs(1 - 2 * (q[:, 0] ** 2 + q[:, 1] ** 2)) * 0.5 * size[:, 2])
    clear = pos[:, 2] - ez - ground_top
    clear[np.abs(clear) < 1e-5] = 0.0
    pen = np.where(dyn & (clear < -1e-5), -clear, 0.0)
    jm = scene.ftype == 1
    jerr = 0.0
    if jm.any():
        fa, fb = scene.fa[jm], scene.fb[jm]
        a = np.where(fa >= 0, n - 1 - fa, 0)
        b = n - 1 - fb
        xa = np.where((fa >= 0)[:, None], pos[a] + _rot_apply(q[a], scene.frA[jm]), scene.frA[jm])
        xb = pos[b] + _rot_apply(q[b], scene.frB[jm])
        jerr = float(np.linalg.norm(xa - xb, axis=1).max())
    return {"max_penetration_m": float(pen.max()) if n else 0.0, "below_ground": int((pen > 0).sum()),
            "max_joint_error_m": jerr}


def mixed_line(args, local, stream, reference: bool, steps: int = 600, chunk: int = 10, ref_steps: int = 5,
               diverged_speed: float = 100.0):
    """The mixed-constraint scene: 200,000 boxes (2,048 jointed chains of 48 boxes, springs
    between 5% of the rest) dropped from a 200 x 200 x 100 m volume onto the ground, up to
    600 steps at 10 iterations. The drop diverges in the reference's own CPU solver as in the
    GPU's colour order: boxes of log-uniform sizes and random orientations landing at up to
    44 m/s (free fall from the volume's top) are thrown off at hundreds of m/s and more, with
    or without the joints and springs. So the run stops at the first chunk whose fastest box
    exceeds diverged_speed, and the line gives that step and the fastest box's speed every
    chunk. Body-steps/s from CUDA events around chunks of 10 device-resident steps (state
    read back between chunks, outside the events) over the steps run, the iteration kernel's
    roofline, and the reference's long-run checks over the same steps: the largest ground
    penetration and joint error (sampled every chunk, every step for the first ref_steps),
    and, when the run reaches step 600, the resting drift (the largest displacement between
    steps 500 and 600 of the boxes slower than 0.05 m/s at step 500). The reference's CPU
    solver (its own list order) gives the same checks for its first ref_steps steps, beside
    the GPU's over the same steps."""
    import torch

    from avbd_demo3d_b200 import World, scenes

    scene = scenes.mixed_drop()
    w = World(scene, device=local, stream=stream.cuda_stream)
    bodies = scene.n_bodies - 1
    w.set_profiling(True)
    w.reset_profile()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * (steps // chunk + ref_steps))]
    spans, k, done = [], 0, 0
    worst = {"max_penetration_m": 0.0, "below_ground": 0, "max_joint_error_m": 0.0}
    early, settled, x500, speeds, diverged, redone_in_run = [], None, None, [], None, 0
    torch.cuda.synchronize()
    while done < steps:
        m = 1 if done < ref_steps else min(chunk, steps - done)
        with torch.cuda.stream(stream):
            ev[k].record(stream)
        w.step(m, sync=False)
        with torch.cuda.stream(stream):
            ev[k + 1].record(stream)
        spans.append((ev[k], ev[k + 1], m))
        k += 2
        done += m
        b = w.bodies()
        c = scene_checks(scene, b)
        for key in worst:
            worst[key] = max(worst[key], c[key])
        if done <= ref_steps:
            early.append(c)
        fastest = float(np.linalg.norm(b["vel"].astype(np.float64), axis=1).max())
        speeds.append([done, round(fastest, 3)])
        redone_in_run = int(w.stats()["redone_steps"])
        if done == 500:
            speed = np.linalg.norm(b["vel"], axis=1)
            settled = speed < 0.05
            x500 = b["pos"].astype(np.float64)
        if fastest > diverged_speed:
            diverged = done
            break
    torch.cuda.synchronize()
    total_s = sum(a.elapsed_time(e) for a, e, _ in spans) / 1e3
    b_end = w.bodies()
    drift = float(np.linalg.norm(b_end["pos"].astype(np.float64)[settled] - x500[settled], axis=1).max()) \
        if (done == 600 and settled is not None and settled.any()) else None
    prof = w.profile()
    w.set_profiling(False)
    st = w.stats()
    per_iter, counts = algorithmic_primal_bytes(w)
    per_iter += 32 * counts["contacts"]
    peak, _ = measured_peak()
    it_ms = prof["primal_ms"]
    achieved = per_iter * scene.params.iterations / (it_ms / max(1, prof["steps"]) / 1e3) / 1e9 if it_ms else None
    out = {"workload": "200,000 boxes + ground (mixed_drop, seed 2): 2,048 chains of 48 boxes on ball joints "
                       "(96,256 joints), springs between 5% of the other boxes; up to 600 steps, dt 1/60, "
                       "10 iterations",
           "value": bodies * done / total_s, "unit": UNIT, "ms_per_step": total_s * 1e3 / done, "steps": done,
           "diverged_at_step": diverged,
           "divergence": f"the run stops after the first chunk whose fastest box exceeds {diverged_speed} m/s "
                         "(free fall from the top of the volume reaches 44.5 m/s)",
           "fastest_box_m_per_s": speeds,
           "final": {"manifolds": int(st["manifold_count"]), "colours": int(st["colours"]),
                     "joints": int(st["joint_count"]), "springs": int(st["spring_count"])},
           "checks_over_run": {**worst, "resting_drift_m": drift,
                               "resting_bodies": int(settled.sum()) if settled is not None else None,
                               "sampling": f"every step for the first {ref_steps}, then every {chunk}"},
           "roofline": {"kernel": "k_iterations", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak if achieved else None,
                        "algorithmic_bytes_per_launch": per_iter * scene.params.iterations,
                        "avg_launch_us": it_ms * 1e3 / max(1, prof["primal_spans"]), **counts,
                        "note": f"counts at step {done}"},
           "phases_ms_per_step": {kk[:-3]: round(v / max(1, prof["steps"]), 4) for kk, v in prof.items()
                                  if kk.endswith("_ms")},
           "device_steps": int(st["device_steps"]), "redone_steps": redone_in_run}
    w.close()
    gpu_early = {key: max(c[key] for c in early) for key in ("max_penetration_m", "max_joint_error_m")}
    out["checks_first_steps"] = {"steps": ref_steps, "gpu": gpu_early}
    if reference:
        with REFERENCE_LOCK:  # waits for the FP64 checker's thread if it still runs
            ref, kind = reference_world(scene)
            ref_checks = []
            t0 = time.perf_counter()
            for _ in range(ref_steps):
                ref.step(1)
                ref_checks.append(scene_checks(scene, ref.bodies()))
            ref_s = time.perf_counter() - t0
            ref.close()
        out["checks_first_steps"]["reference"] = {key: max(c[key] for c in ref_checks)
                                                  for key in ("max_penetration_m", "max_joint_error_m")}
        out["checks_first_steps"]["reference_kind"] = kind
        out["cpu_reference"] = {"value": bodies * ref_steps / ref_s, "unit": UNIT, "kind": kind,
                                "cores": cpu_cores(kind), "sample": f"the first {ref_steps} steps of the same scene"}
    return out


class CpuFp64Reference:
    """CPU checker leg: the reference's double-precision build (oracle/_ref/libavbd_ref64.so,
    made by oracle/make_fp64.py from the reference's own sources) stepped in its own list
    order on a background thread (the stepping call releases the GIL), for the 65,536-box
    stack field to steps 10 and 60 and the 210-box pyramid to steps 10, 60 and 600. The GPU's
    state at the same steps comes from fresh GPU runs (the step is deterministic), and the
    line states the largest position and rotation differences from FP64."""

    MARKS = {"stacks65k": (10, 60), "pyramid20": (10, 60, 600)}

    def __init__(self):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import checkers

        self.checkers = checkers
        self.available = checkers.ref64_available()
        self.states, self.error = {}, None
        self.thread = threading.Thread(target=self._run, daemon=True) if self.available else None
        if self.thread:
            self.thread.start()

    @staticmethod
    def scenes():
        from avbd_demo3d_b200 import scenes

        return {"stacks65k": scenes.stack_grid(*GRID, seed=SEED), "pyramid20": scenes.pyramid(20)}

    def _run(self):
        try:
            with REFERENCE_LOCK:
                for name, sc in self.scenes().items():
                    r = self.checkers.Fp64Reference(sc)
                    done, got = 0, {}
                    for m in self.MARKS[name]:
                        r.step(m - done)
                        done = m
                        got[m] = r.bodies()
                    r.close()
                    self.states[name] = got
        except Exception as e:  # reported in the line
            self.error = repr(e)

    def result(self, local, stream):
        from avbd_demo3d_b200 import World

        if not self.available:
            return {"unavailable": "oracle/_ref/libavbd_ref64.so not built"}
        gpu = {}
        for name, sc in self.scenes().items():
            w = World(sc, device=local, stream=stream.cuda_stream)
            done, got = 0, {}
            for m in self.MARKS[name]:
                w.step(m - done)
                done = m
                got[m] = w.bodies()
            w.close()
            gpu[name] = got
        self.thread.join()
        if self.error:
            return {"unavailable": self.error}
        out = {"reference": "the reference's double-precision build, its own list order (same inputs)"}
        for name, marks in self.MARKS.items():
            out[name] = {}
            for m in marks:
                dp, dq = self.checkers.pose_error(gpu[name][m], self.states[name][m])
                out[name][str(m)] = {"max_pos_m": dp, "max_rot_rad": dq}
        return out


# The reference's CPU solvers (its own build and its double-precision build) share one
# process-wide worker pool, which serves one caller at a time: every use of them in this
# process, the FP64 checker's background thread included, holds this lock.
REFERENCE_LOCK = threading.Lock()


def reference_world(scene):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import checkers

    kind = "ref" if checkers.ref_available() else "oracle"
    return checkers.World(scene, kind), ("reference" if kind == "ref" else "port")


def cpu_cores(kind: str) -> int:
    n = os.cpu_count() or 1
    # the reference's WorkerPool runs min(hw - 1, 7) workers plus the calling thread
    return min(n, 8) if kind == "reference" else 1


def cpu_baseline(scene, warm: int = 1, timed: int = 5):
    with REFERENCE_LOCK:
        w, kind = reference_world(scene)
        w.step(warm)
        t0 = time.perf_counter()
        w.step(timed)
        dt = time.perf_counter() - t0
    bodies = scene.n_bodies - 1
    return {"value": bodies * timed / dt, "unit": UNIT, "cores": cpu_cores(kind), "kind": kind,
            "sample": f"the same 65,536-box scene, steps {warm + 1}-{warm + timed} after {warm} untimed step(s), "
                      f"Solver::step with the CPU reference backend; {dt / timed * 1e3:.0f} ms/step"}


def run_reference(args):
    rank, world_size, _ = dist_env()
    if rank != 0:
        return
    from avbd_demo3d_b200 import scenes

    scene = scenes.stack_grid(*GRID, seed=SEED)
    w, kind = reference_world(scene)
    warm = min(args.warmup, 2)
    timed = max(1, min(args.steps, 8))
    w.step(warm)
    t0 = time.perf_counter()
    w.step(timed)
    dt = time.perf_counter() - t0
    bodies = scene.n_bodies - 1
    value = bodies * timed / dt
    cores = cpu_cores(kind)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size,
            "steps": timed, "warmup": warm, "ms_per_step": dt / timed * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "bodies_per_gpu": bodies, "parallelism": "cpu"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": f"{timed} steps of the 65,536-box scene after {warm} untimed "
                                       f"(bounded sample of --steps {args.steps})"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("cuda", "reference"), default="cuda")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-adjoint-check", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the 200,000-box mixed-constraint section")
    ap.add_argument("--no-fp64", action="store_true", help="skip the error against the FP64 reference build")
    ap.add_argument("--no-lbvh", action="store_true", help="skip the LBVH broadphase mode section")
    ap.add_argument("--no-late", action="store_true", help="skip the late window (steps 281-300)")
    ap.add_argument("--iteration-mode", type=int, default=1, choices=(0, 1),
                    help="0 = one launch per colour and iteration plus the dual sweep, 1 = one launch per step")
    ap.add_argument("--primal-variant", type=int, default=-1,
                    help="use this primal variant (index into World.primal_variants()) instead of autotuning")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_cuda(args)


if __name__ == "__main__":
    main()
