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


def ncu_traffic_per_launch(kernel: str = "k_primal"):
    """dram bytes per launch of `kernel` from its committed ncu summary, if present."""
    name = {"k_primal": "primal_stacks65k_ncu.md", "k_iterations": "iterations_stacks65k_ncu.md"}[kernel]
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


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
    traffic = ncu_traffic_per_launch("k_iterations" if persistent else "k_primal")
    kernel = ("k_iterations (every iteration of a step: coloured primal sweeps, contact dual updates fused into "
              "the rows, joint dual updates)" if persistent else "k_primal (coloured primal sweep, one launch per "
              "colour)")
    roofline = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "algorithmic_bytes_per_launch": per_iter * iters * prof["steps"] / primal_launches,
                "avg_launch_us": primal_ms * 1e3 / primal_launches, "launches": primal_launches,
                "iteration_mode": "one launch per step" if persistent else "one launch per colour", **counts}
    phases = {k[:-3]: round(v / max(1, prof["steps"]), 4) for k, v in prof.items() if k.endswith("_ms")}

    # ---- end to end through the C ABI with host buffers (H2D state, step, D2H state)
    st = w.bodies()
    host = {k: np.ascontiguousarray(v) for k, v in st.items()}
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
           "path": "avbd_write_bodies (pinned staging H2D) + avbd_step + avbd_read_bodies (D2H) into the "
                   "caller's arrays (allocated once, reused every step), host timer"}

    collision = collision_only(w, scene, rank, world_size, local, reference=not args.no_cpu_baseline)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(scene)
    batched = batched_line(args, rank, world_size, local, stream) if not args.no_batched else None
    adjoint = adjoint_line(args, local, stream) if (rank == 0 and not args.no_adjoint) else None
    w.close()
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
                "adjoint": adjoint, "collision_only": collision,
                "autotune": {"primal_variant": World.primal_variants()[tuned],
                             "sweep_us": [round(float(x), 1) for x in variant_us]},
                "step_ms_min_max": [min(step_ms), max(step_ms)]}
        print(json.dumps(line), flush=True)


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
        ref, kind = reference_world(scene)
        ref.step(1)
        t0 = time.perf_counter()
        for _ in range(2):
            ref.broadphase_only()
        out["cpu_reference"] = {"ms_per_frame": (time.perf_counter() - t0) / 2 * 1e3, "kind": kind,
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
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        ev0.record(stream)
    w.step(steps, sync=False)
    with torch.cuda.stream(stream):
        ev1.record(stream)
    torch.cuda.synchronize()
    batched_s = max_over_ranks(ev0.elapsed_time(ev1) / 1e3, device=f"cuda:{local}")
    n_bodies = int(sum(sc.n_bodies - 1 for sc in all_worlds))
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
            "speedup_vs_loop": batched_rate / loop_rate,
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
    out = {"workload": "tower 10x10x10 = 1,000 boxes + ground (seed 4), 120 steps, 10 iterations, checkpoint "
                       "every 10 steps; loss |COM(x_120) - target|^2, target = COM_0 + U[-1,1]^3 (seed 7)",
           "forward_ms": f_s * 1e3, "adjoint_forward_ms": a_s * 1e3, "backward_ms": b_s * 1e3,
           "bwd_over_fwd": b_s / f_s, "fwd_plus_bwd_over_fwd": (a_s + b_s) / f_s,
           "timing": "host timer around the C-ABI calls (the step itself reads a few counts per step), "
                     "median of 3 after one warm-up", "params": int(grad.size)}
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
