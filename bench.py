"""Benchmark of the explicit MPM step (ExplicitUSL) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Prints one JSON line. A "step" is one ExplicitUSL time step over the whole
workload (map build, P2G, contact, boundary, grid update, G2P, stress) with
the point and grid state resident in HBM; ``value`` is whole-job
particle-steps per second from CUDA events on the solver's stream, ``e2e``
is the same metric through the C ABI from host buffers (upload, K steps,
download of the final point state, all inside the timed region).

Workloads (seeded synthetic inputs, mpm_3d_b200.inputs):
  collision  two 0.25 m cubes colliding, 128^3 grid, 524,288 points, ContactHuang
  column     column collapse, 256x256x128 grid, 3,145,728 points

With N > 1 (torchrun) every rank runs an independent replica of the
workload (the single-instance step does not shard); ``value`` sums the
points of all ranks over the slowest rank's time.

``--impl reference`` times the reference solver's own CPU code
(ThreadPoolExplicitUSL + ThreadPoolPoints, compiled from its sources into
oracle/_ref/libmpmref_timing.so) on all host threads, on a bounded sample of
steps of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from mpm_3d_b200 import inputs  # noqa: E402

METRIC = "batched particle-steps/s vs plain FP64 GPU at ≤1e-4 rel err; p50/p99 latency"
UNIT = "particle-steps/s"
L2_BYTES = 126 * 1024 * 1024


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def make_workload(name: str):
    if name == "collision":
        return inputs.two_body_collision_3d(128)
    if name == "column":
        return inputs.column_collapse_3d(1)
    raise SystemExit(f"unknown workload {name}")


def bytes_per_point_step(active_nodes_per_point: float) -> float:
    """Algorithmic bytes per particle-step of the FP64 form: point state read
    (x, v, m, V, sigma(6), u, extent, active = 148 B) and written (x, v, V,
    sigma, u = 128 B), plus the grid term 112 B per active node per body
    (m, momentum, force accumulated and read once)."""
    return 276.0 + 112.0 * active_nodes_per_point


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_reference_run(case, steps: int, warmup: int, threads: int):
    """Times the reference's ThreadPoolExplicitUSL (own sources, timing
    build) on `threads` host threads: returns seconds per step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bridge

    d = tempfile.mkdtemp()
    cfg = inputs.write_case(case, d, solver_class="ThreadPoolExplicitUSL", points_class="ThreadPoolPoints",
                            threads=threads)
    with quiet_stdout():  # the reference reports its set-up on stdout
        job = bridge.ReferenceJob(cfg, build="timing")
        job.step(warmup)
        t0 = time.perf_counter()
        job.step(steps)
        dt = (time.perf_counter() - t0) / steps
        job.close()
    return dt


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null (C and C++ output included), so
    the benchmark's JSON line stays the only line on stdout."""

    def __enter__(self):
        import ctypes

        self.libc = ctypes.CDLL(None)
        sys.stdout.flush()
        self.libc.fflush(None)
        self.saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    case = make_workload(args.workload)
    threads = os.cpu_count() or 1
    steps = max(1, min(args.steps, args.ref_steps))
    warm = 1
    sec = cpu_reference_run(case, steps, warm, threads)
    value = case.n_points / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": warm, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mpm_3d_b200.inputs)",
        "config": {"workload": args.workload, "points": case.n_points, "grid": list(case.N), "dt": case.dt},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{steps} steps after {warm} warm-up of the full {args.workload} workload, "
                                   f"ThreadPoolExplicitUSL+ThreadPoolPoints, threads={threads}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import torch

    from mpm_3d_b200.native import GPUExplicitUSL

    torch.cuda.set_device(local)
    case = make_workload(args.workload)
    n = case.n_points
    state_bytes = 148 * n
    flush_l2 = state_bytes < 2 * L2_BYTES
    flush_buf = torch.empty(4 * L2_BYTES // 4, dtype=torch.float32, device="cuda") if flush_l2 else None

    sim = GPUExplicitUSL(case, device=local)
    stream = torch.cuda.ExternalStream(sim.stream())
    sim.step(args.warmup)
    sim.synchronize()
    sim.profile(True)
    launches0 = sim.launches()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    barrier(world)
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            if flush_l2:
                with torch.cuda.stream(stream):
                    flush_buf.fill_(float(k))
            starts[k].record(stream)
            sim.step(1)
            stops[k].record(stream)
        sim.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    step_ms = [starts[k].elapsed_time(stops[k]) for k in range(args.steps)]
    prof = sim.profile_read()
    launches = sim.launches() - launches0
    sim.profile(False)
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, world)
    points_all = sum_over_ranks(float(n), world)
    value = points_all * args.steps / (total_ms_max * 1e-3)

    # active nodes per point (grid term of the algorithmic bytes)
    active_ratio = active_nodes_ratio(sim, case)
    bpp = bytes_per_point_step(active_ratio)
    g_launches, g_ms = prof["g2p2g"]
    per_launch_ms = g_ms / max(1, g_launches)
    # the fused launches of a step together process every point once; the
    # algorithmic bytes of a launch are its points times bytes per point-step
    points_per_launch = n * args.steps / max(1, g_launches)
    achieved_gbs = points_per_launch * bpp / (per_launch_ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    sim.close()

    e2e = run_e2e(case, args.steps, local) if rank == 0 and not args.no_e2e else None
    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            threads = os.cpu_count() or 1
            csteps = max(1, min(args.steps, args.ref_steps))
            sec = cpu_reference_run(case, csteps, 1, threads)
            cpu = {"value": n / sec, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{csteps} steps after 1 warm-up of the full {args.workload} workload, "
                             f"ThreadPoolExplicitUSL+ThreadPoolPoints, threads={threads}"}
        except Exception as exc:  # the oracle build may be absent
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank != 0:
        return
    clk = clocks.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded mpm_3d_b200.inputs)",
        "config": {"workload": args.workload, "points": n, "bodies": len(case.bodies), "grid": list(case.N),
                   "dt": case.dt, "form": "fp64", "parallelism": f"replicas{world}",
                   "l2": "flushed between steps" if flush_l2 else "inputs larger than L2",
                   "active_nodes_per_point": round(active_ratio, 4)},
        "roofline": {"bound": "hbm", "kernel": "k_g2p2g", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                     "frac": achieved_gbs / peak, "peak_kind": peak_kind, "traffic": None,
                     "bytes_per_point_step": bpp, "launch_ms": per_launch_ms},
        "stage_ms_per_step": {k: v[1] / args.steps for k, v in prof.items()},
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def active_nodes_ratio(sim, case) -> float:
    """Active nodes (m > 0) per point, counted per body after the last step."""
    from mpm_3d_b200.native import GPUExplicitUSL  # noqa: F401

    tot = 0
    for b in range(len(case.bodies)):
        xt = sim.nodes(b, "x_t")
        tot += int(np.count_nonzero(np.any(xt != 0.0, axis=1)))
    return tot / max(1, case.n_points)


def run_e2e(case, steps: int, device: int):
    """Same metric through the C ABI from host buffers: create + upload,
    `steps` steps, download of every point's x, x_t and stress, destroy."""
    import torch

    from mpm_3d_b200.native import GPUExplicitUSL

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = GPUExplicitUSL(case, device=device)
    sim.step(steps)
    outs = []
    for b in range(len(case.bodies)):
        outs.append(sim.points(b, "x"))
        outs.append(sim.points(b, "x_t"))
        outs.append(sim.points(b, "T"))
    sim.close()
    dt = time.perf_counter() - t0
    n = case.n_points
    h2d = sum(b.n * (8 + 8 + 24 + 24 + 4) for b in case.bodies)
    d2h = sum(o.nbytes for o in outs)
    return {"value": n * steps / dt, "unit": UNIT, "h2d_bytes_per_step": h2d // steps,
            "d2h_bytes_per_step": d2h // steps, "steps": steps, "seconds": dt}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="timed steps (default: the workload's own step count)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--workload", default="collision", choices=["collision", "column"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-steps", type=int, default=4, help="steps of the CPU reference sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.steps <= 0:
        args.steps = make_workload(args.workload).steps
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
