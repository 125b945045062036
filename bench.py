"""Benchmark of the explicit MPM step (ExplicitUSL) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Prints one JSON line. A "step" is one ExplicitUSL time step of every job of
the workload (map build, P2G, contact, boundary, grid update, G2P, stress)
with the point and grid state resident in HBM; ``value`` is whole-job
particle-steps per second from CUDA events on the solver's stream, ``e2e``
is the same metric through the C ABI from host buffers (upload, K steps,
download of the final point state, all inside the timed region).

Workloads (seeded synthetic inputs, mpm_3d_b200.inputs):
  ensemble   (default) 512 independent 3D block drops (grids 16^3..96^3,
             16.75 M points, seed 1003) in one batch per form (FP64; mixed:
             FP32 point state with two-word x, x_t and m, FP64 nodal sums),
             one launch per stage replayed from a CUDA graph, kernel form
             and points per CTA chosen by the autotuner. ``value`` is the
             fastest batched form within 1e-4 of FP64 on every compared job
             (every 8th) after its full 500 steps; both forms are reported
             with their errors, beside the plain FP64 path (one handle per
             job, jobs one after another), the column collapse in plain
             FP64 (``column_fp64``, with its own roofline) and the full
             serving stream (``serving_full``, 60 s of arrivals).
  blockdrop2d  the 2D block drop, 20x20 grid, 144 points, 2000 steps (CPU-sized)
  collision  two 0.25 m cubes colliding, 128^3 grid, 524,288 points, ContactHuang (FP64)
  column     column collapse, 256x256x128 grid, 3,145,728 points (FP64)
  serving    Poisson request stream at 100/s (block drops with N in [16,128],
             200..5000 steps, 10 % two-body ContactHuang), admitted under a
             150 GB budget into one continuously batched mixed-form server;
             ``value`` is the particle-steps/s of the completed requests over
             the makespan, with p50/p99 time to completion. The ensemble
             line carries the same figures for --serve-seconds of arrivals
             (60 by default, the whole stream).

With N > 1 (torchrun) every rank runs its own copy of the workload (the
ensemble with seed 1003 + rank; the single jobs as replicas): no data
crosses ranks; ``value`` sums the points of all ranks over the slowest
rank's time.

``--impl reference`` times the reference solver's own CPU code
(ThreadPoolExplicitUSL + ThreadPoolPoints, compiled from its sources into
oracle/_ref/libmpmref_timing.so) on all host threads, on a bounded sample of
the same workload (for the ensemble: 16 of its jobs, every 32nd, a few steps
each, one after another).
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


ENSEMBLE_JOBS = 512
ENSEMBLE_SEED = 1003

# DRAM bytes (read + write) per point of one k_g2p2g launch, from ncu
# captures of the kernel (the ensemble's from a capture of its first 96 jobs,
# scaled to a launch by its points; the column's at full size). None where no
# capture exists.
TRAFFIC_BYTES_PER_POINT = {("ensemble", "mixed"): 289.2, ("ensemble", "fp64"): 341.2, ("column", "fp64"): 349.5,
                           ("column", "mixed"): 271.7}


def make_workload(name: str, rank: int = 0):
    if name == "collision":
        return inputs.two_body_collision_3d(128)
    if name == "column":
        return inputs.column_collapse_3d(1)
    if name == "ensemble":
        return inputs.block_drop_ensemble(ENSEMBLE_JOBS, seed=ENSEMBLE_SEED + rank)
    if name == "blockdrop2d":
        return inputs.block_drop_2d()
    raise SystemExit(f"unknown workload {name}")


def bytes_per_point_step(active_nodes_per_point: float, mixed: bool = False) -> float:
    """Algorithmic bytes per particle-step. FP64 form: point state read
    (x, v, m, V, sigma(6), u, extent, active = 148 B) and written (x, v, V,
    sigma, u = 128 B). Mixed form: x, x_t and m as two FP32 words (8 B per
    value), the other fields in FP32: read x 24, x_t 24, m 8, V 4, sigma 24,
    u 12, extent 4, active 4 = 104 B; written x, x_t, V, sigma, u = 88 B.
    Plus the grid term 112 B per active node per body (m, momentum, force
    accumulated and read once, FP64 in both forms)."""
    return (192.0 if mixed else 276.0) + 112.0 * active_nodes_per_point


def field_floor(case, field: str) -> float:
    """Physical scale of a field for relative errors (velocity: largest
    initial speed, at least 1 m/s; stress: one step of elastic stress at
    that speed over a cell; position: the domain)."""
    v0 = max(1.0, max(float(np.abs(b.x_t).max()) for b in case.bodies))
    h = min(case.h)
    E = max(b.E for b in case.bodies)
    return {"T": E * case.dt * v0 / h, "x_t": v0, "x": min(case.L)}.get(field, 0.0)


def rel_err(got, ref, floor: float) -> float:
    scale = max(float(np.max(np.abs(ref))) if ref.size else 0.0, floor)
    diff = float(np.max(np.abs(got - ref))) if ref.size else 0.0
    return diff / scale if scale > 0 else diff


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


def dist_setup(n_gpus: int, backend: str = "nccl"):
    """Rank, world size and local rank from the torchrun environment; joins
    the process group (NCCL between GPUs; gloo for the host-side tests)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return rank, world, local


def _reduce_device():
    import torch.distributed as dist

    return "cpu" if dist.get_backend() == "gloo" else "cuda"


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def cpu_reference_run(case, steps: int, warmup: int, threads: int):
    """Times the reference's solver (own sources, timing build) on `threads`
    host threads: ThreadPoolExplicitUSL with ThreadPoolPoints, or the serial
    ExplicitUSL for threads == 1. Returns seconds per step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import bridge

    d = tempfile.mkdtemp()
    if threads == 1:
        cfg = inputs.write_case(case, d)
    else:
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
    if args.workload in ("ensemble", "serving"):
        if args.workload == "serving":
            specs = inputs.serving_stream(rate=100.0, duration=args.serve_seconds, seed=1004)
            cases = [inputs.serving_case(sp) for sp in specs[::max(1, len(specs) // 16)][:16]]
        else:
            cases = make_workload("ensemble")
        steps = max(1, min(args.steps, args.ref_steps))
        cpu = cpu_ensemble_sample(cases, steps, args.warmup)
        value = cpu["value"]
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": f"synthetic (block_drop_ensemble seed {ENSEMBLE_SEED})",
            "config": {"workload": args.workload if args.workload == "serving" else f"ensemble{ENSEMBLE_JOBS}",
                       "jobs": len(cases), "points": sum(c.n_points for c in cases)},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
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


def timed_steps(sim, steps: int, flush_buf=None):
    """Times `steps` single steps with CUDA events on the solver's stream
    (L2 flushed before each when `flush_buf` is given); returns per-step ms,
    kernel launches in the timed region and the clock record."""
    import torch

    stream = torch.cuda.ExternalStream(sim.stream())
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    stops = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    sim.synchronize()
    torch.cuda.synchronize()
    launches0 = sim.launches()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for k in range(steps):
            if flush_buf is not None:
                with torch.cuda.stream(stream):
                    flush_buf.fill_(float(k))
            starts[k].record(stream)
            sim.step(1)
            stops[k].record(stream)
        sim.synchronize()
        torch.cuda.synchronize()
    launches = sim.launches() - launches0
    return [starts[k].elapsed_time(stops[k]) for k in range(steps)], launches, clocks.summary()


def profile_pass(sim, steps: int):
    """Per-stage device time over `steps` steps (stage by stage launches)."""
    sim.profile(True)
    sim.step(steps)
    prof = sim.profile_read()
    sim.profile(False)
    return prof


def roofline(points: int, steps: int, prof, active_ratio: float, mixed: bool, traffic_key=None):
    peak, peak_kind = peaks()
    bpp = bytes_per_point_step(active_ratio, mixed)
    g_launches, g_ms = prof["g2p2g"]
    per_launch_ms = g_ms / max(1, g_launches)
    # the fused launches of a step together process every point once; the
    # algorithmic bytes of a launch are its points times bytes per point-step
    points_per_launch = points * steps / max(1, g_launches)
    achieved_gbs = points_per_launch * bpp / (per_launch_ms * 1e-3) / 1e9
    tb = TRAFFIC_BYTES_PER_POINT.get(traffic_key)
    return {"bound": "hbm", "kernel": "k_g2p2g", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
            "frac": achieved_gbs / peak, "peak_kind": peak_kind,
            "traffic": tb * points_per_launch if tb else None,
            "traffic_source": "ncu dram__bytes per point x points per launch" if tb else None,
            "bytes_per_point_step": bpp, "launch_ms": per_launch_ms, "points_per_launch": points_per_launch}


def single_timed(case, form: str, steps: int, warmup: int, device: int, world: int = 1, traffic_key=None,
                 kernel=None):
    """One single-job handle: `warmup` steps, then `steps` steps timed with
    CUDA events (L2 flushed between steps when the point state would fit
    in it), a profiled pass for the fused kernel's launch time, and the
    roofline of that kernel."""
    import torch

    from mpm_3d_b200.native import GPUExplicitUSL

    n = case.n_points
    flush_l2 = 148 * n < 2 * L2_BYTES
    flush_buf = torch.empty(4 * L2_BYTES // 4, dtype=torch.float32, device="cuda") if flush_l2 else None
    sim = GPUExplicitUSL(case, device=device, mode=form, kernel=kernel)
    sim.step(warmup)
    barrier(world)
    step_ms, launches, clk = timed_steps(sim, steps, flush_buf)
    barrier(world)
    prof_steps = min(10, steps)
    prof = profile_pass(sim, prof_steps)
    active, _drift = sim.active_nodes()
    active_ratio = active / max(1, n)
    roof = roofline(n, prof_steps, prof, active_ratio, form == "mixed", traffic_key)
    used = sim.kernel()
    sim.close()
    del flush_buf
    return {"step_ms": step_ms, "launches": launches, "clocks": clk, "prof": prof, "prof_steps": prof_steps,
            "active_ratio": active_ratio, "roofline": roof, "l2_flushed": flush_l2, "kernel": used}


def run_single(args, rank, world, local):
    import torch

    torch.cuda.set_device(local)
    case = make_workload(args.workload)
    n = case.n_points
    r = single_timed(case, args.form, args.steps, args.warmup, local, world, (args.workload, args.form), args.kernel)
    step_ms, launches, clk, prof, prof_steps = r["step_ms"], r["launches"], r["clocks"], r["prof"], r["prof_steps"]
    flush_l2, active_ratio, roof = r["l2_flushed"], r["active_ratio"], r["roofline"]
    total_ms = sum(step_ms)
    total_ms_max = max_over_ranks(total_ms, world)
    points_all = sum_over_ranks(float(n), world)
    value = points_all * args.steps / (total_ms_max * 1e-3)

    e2e = run_e2e(case, args.steps, local, args.form) if rank == 0 and not args.no_e2e else None
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
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.form == "mixed" else "f64", "data": "synthetic (seeded mpm_3d_b200.inputs)",
        "config": {"workload": args.workload, "points": n, "bodies": len(case.bodies), "grid": list(case.N),
                   "dt": case.dt, "form": args.form, "kernel": r["kernel"][0], "points_per_item": r["kernel"][1],
                   "parallelism": f"replicas{world}",
                   "l2": "flushed between steps" if flush_l2 else "inputs larger than L2",
                   "active_nodes_per_point": round(active_ratio, 4)},
        "roofline": roof,
        "stage_ms_per_step": {k: v[1] / prof_steps for k, v in prof.items()},
        "gpu_launches": launches,
        "clocks": clk,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def ensemble_sample(cases, every: int = 8):
    return list(range(0, len(cases), every))


def run_batch(cases, mode: str, args, device: int, sample_ids):
    """One batch of every job: autotune, warm-up, K timed steps (graph
    replay), a profiled pass; returns figures and the final x, x_t, T of the
    sampled jobs."""
    from mpm_3d_b200.native import GPUBatch

    if args.kernel is None:
        b = GPUBatch(dim=3, mode=mode, device=device)
        jobs = [b.add(c) for c in cases]
        cap = b.autotune(steps=8)
    else:
        b = GPUBatch(dim=3, mode=mode, device=device, sort_interval=args.sort_interval, kernel=args.kernel)
        jobs = [b.add(c) for c in cases]
        cap = b.points_per_item()
    kernel = b.kernel_form()
    si = b.sort_interval()
    b.step(args.warmup)
    step_ms, launches, clk = timed_steps(b, args.steps)
    # one whole re-binning interval, so that the per-stage times carry one
    # re-binning per sort_interval steps, as the timed steps do
    prof_steps = max(3, si)
    prof = profile_pass(b, prof_steps)
    active, drift = b.active_nodes()
    steps_done = b.state(jobs[0])[0]
    b.close()
    return {"step_ms": step_ms, "launches": launches, "clocks": clk, "prof": prof, "prof_steps": prof_steps,
            "active": active, "drift": drift, "cap": cap, "kernel": kernel, "sort_interval": si,
            "steps_done": steps_done}


REL_ERR_BOUND = 1e-4


def form_errors_full(cases, sample_ids, device: int):
    """Errors of the batched forms after every sampled job's full step count
    (outside any timed region): the sampled jobs run as one FP64 batch and
    one mixed batch, and each as a single deterministic-FP64 handle, to
    their ends; x, x_t and the stress are compared per job. `mixed` is the
    mixed form against the FP64 batch; `fp64` is the FP64 batch against the
    deterministic form, i.e. how far two FP64 summation orders drift apart
    on these dynamics (the amplification of round-off)."""
    from mpm_3d_b200.native import GPUBatch, GPUExplicitUSL

    sub = [cases[i] for i in sample_ids]
    steps = max(c.steps for c in sub)
    keys = ("x", "x_t", "T")
    fields = {}
    for mode in ("fp64", "mixed"):
        b = GPUBatch(dim=3, mode=mode, device=device)
        jobs = [b.add(c) for c in sub]
        b.step(steps)
        fields[mode] = [{f: b.points(j, 0, f) for f in keys} for j in jobs]
        done = min(b.state(j)[0] for j in jobs)
        b.close()
    fields["det"] = []
    for c in sub:
        sim = GPUExplicitUSL(c, device=device, mode="fp64_deterministic")
        sim.step(c.steps)
        fields["det"].append({f: sim.points(0, f) for f in keys})
        sim.close()

    def summary(got, ref):
        worst = {f: 0.0 for f in keys}
        failing = []
        for k, c in enumerate(sub):
            e = {f: rel_err(fields[got][k][f], fields[ref][k][f], field_floor(c, f)) for f in keys}
            for f in keys:
                worst[f] = max(worst[f], e[f])
            if max(e.values()) > REL_ERR_BOUND:
                failing.append(sample_ids[k])
        return {**worst, "jobs_compared": len(sub), "jobs_within_bound": len(sub) - len(failing),
                "jobs_over_bound": failing, "bound": REL_ERR_BOUND, "after_steps": done,
                "norm": "max|a - b| / max(max|b|, field scale) per job and field; worst job"}

    return {"mixed": summary("mixed", "fp64"), "fp64": summary("fp64", "det")}


def column_fp64_record(device: int, steps: int = 400, warmup: int = 5):
    """The column collapse (3,145,728 points, 256x256x128 grid) in the plain
    FP64 form on one handle: the configuration the FP64 roofline target is
    stated on."""
    case = make_workload("column")
    r = single_timed(case, "fp64", steps, warmup, device, 1, ("column", "fp64"))
    total_ms = sum(r["step_ms"])
    return {"value": case.n_points * steps / (total_ms * 1e-3), "unit": UNIT, "ms_per_step": total_ms / steps,
            "steps": steps, "warmup": warmup, "points": case.n_points, "grid": list(case.N), "form": "fp64",
            "roofline": r["roofline"], "stage_ms_per_step": {k: v[1] / r["prof_steps"] for k, v in r["prof"].items()},
            "gpu_launches": r["launches"], "clocks": r["clocks"],
            "l2": "flushed between steps" if r["l2_flushed"] else "inputs larger than L2",
            "active_nodes_per_point": round(r["active_ratio"], 4)}


def plain_fp64(cases, steps: int, device: int):
    """The plain FP64 path: one single-job handle per job, the jobs one
    after another; per job 3 warm-up steps, then `steps` steps timed with
    CUDA events (set-up and teardown outside the timed regions)."""
    import torch

    from mpm_3d_b200.native import GPUExplicitUSL

    total_ms = 0.0
    points = 0
    for c in cases:
        sim = GPUExplicitUSL(c, device=device)
        sim.step(3)
        stream = torch.cuda.ExternalStream(sim.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sim.synchronize()
        e0.record(stream)
        sim.step(steps)
        e1.record(stream)
        sim.synchronize()
        total_ms += e0.elapsed_time(e1)
        points += c.n_points
        sim.close()
    return points * steps / (total_ms * 1e-3), total_ms


def run_ensemble(args, rank, world, local):
    """The ensemble in both batched forms. The line's `value` is the fastest
    batched form whose results stay within REL_ERR_BOUND of FP64 on every
    compared job after its full step count (the metric's condition): the
    mixed form when it holds, else the FP64 batch; the other form is
    reported beside it with its errors."""
    import torch

    torch.cuda.set_device(local)
    cases = make_workload("ensemble", rank)
    if args.jobs > 0:
        cases = cases[:args.jobs]
    n = sum(c.n_points for c in cases)
    sample_ids = ensemble_sample(cases)
    barrier(world)
    fp64 = run_batch(cases, "fp64", args, local, sample_ids) if not args.only_mixed else None
    mixed = run_batch(cases, "mixed", args, local, sample_ids) if not args.only_fp64 else None
    barrier(world)
    # the forms' errors after every sampled job's 500 steps
    errs = form_errors_full(cases, sample_ids, local) if fp64 and mixed and not args.no_errors else None
    if mixed is None:
        mixed_ok = False
    elif fp64 is None:
        mixed_ok = True
    else:
        mixed_ok = errs is not None and errs["mixed"]["jobs_within_bound"] == errs["mixed"]["jobs_compared"]
    head_mode = "mixed" if mixed_ok else "fp64"
    head = mixed if mixed_ok else fp64
    total_ms = sum(head["step_ms"])
    total_ms_max = max_over_ranks(total_ms, world)
    points_all = sum_over_ranks(float(n), world)
    value = points_all * args.steps / (total_ms_max * 1e-3)

    def form_value(r):
        return n * args.steps / (sum(r["step_ms"]) * 1e-3)

    def form_roof(r, mode):
        return roofline(n, r["prof_steps"], r["prof"], r["active"] / max(1, n), mode == "mixed", ("ensemble", mode))

    active_ratio = head["active"] / max(1, n)
    roof = form_roof(head, head_mode)
    plain_value, plain_ms = plain_fp64(cases, args.plain_steps, local) if not args.no_plain else (None, None)
    column = column_fp64_record(local) if not args.no_column else None
    serving = (run_serving(args.serve_seconds, local, head["sort_interval"], policy=args.policy)
               if args.serve_seconds > 0 else None)
    # end to end: every job runs its own step count (the workload's 500
    # steps), as a user runs the ensemble, in the headline's form
    e2e = (run_e2e_batch(cases, max(c.steps for c in cases), local, (head["kernel"], head["cap"]),
                         head["sort_interval"], head_mode)
           if rank == 0 and not args.no_e2e else None)
    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            cpu = cpu_ensemble_sample(cases, args.ref_steps)
            cpu["thread_variants"] = cpu_thread_variants(cases)
        except Exception as exc:  # the oracle build may be absent
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {exc}"}
    if rank != 0:
        return

    def form_record(r, mode):
        if r is None:
            return None
        return {"value": form_value(r), "unit": UNIT, "ms_per_step": sum(r["step_ms"]) / args.steps,
                "kernel": r["kernel"], "points_per_item": r["cap"], "sort_interval": r["sort_interval"],
                "roofline": form_roof(r, mode),
                "rel_err": errs[mode] if errs else None,
                "rel_err_against": "the FP64 batch" if mode == "mixed" else "deterministic FP64 (single handles)"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if head_mode == "mixed" else "f64",
        "data": f"synthetic (mpm_3d_b200.inputs.block_drop_ensemble, seed {ENSEMBLE_SEED}+rank)",
        "config": {"workload": f"ensemble{ENSEMBLE_JOBS}" + (f"[:{args.jobs}]" if args.jobs > 0 else ""),
                   "jobs": len(cases), "points": n,
                   "grids": "N^3, N log-uniform in [16,96]",
                   "form": ("mixed (FP32 point state with two-word x, x_t and m; FP64 nodal sums)"
                            if head_mode == "mixed" else "FP64"),
                   "form_rule": f"fastest batched form within {REL_ERR_BOUND:g} of FP64 on every compared job "
                                "after 500 steps",
                   "kernel": head["kernel"], "points_per_item": head["cap"],
                   "sort_interval": head["sort_interval"], "graph": True,
                   "parallelism": f"independent{world}",
                   "l2": "inputs larger than L2", "active_nodes_per_point": round(active_ratio, 4)},
        "batched_fp64": form_record(fp64, "fp64"),
        "batched_mixed": form_record(mixed, "mixed"),
        "plain_fp64": {"value": plain_value, "unit": UNIT, "steps_per_job": args.plain_steps,
                       "how": "one mpmgpu_handle per job, jobs in sequence, CUDA events around each job's steps"},
        "vs_plain_fp64": (value / plain_value) if plain_value else None,
        "mixed_rel_err_vs_fp64": errs["mixed"] if errs else None,
        "column_fp64": column,
        "serving_full": serving,
        "roofline": roof,
        "stage_ms_per_step": {k: v[1] / head["prof_steps"] for k, v in head["prof"].items()},
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def run_serving(seconds: float, device: int, sort_interval: int = 8, round_steps: int = 20, policy: str = "fifo"):
    """The serving stream for `seconds` of arrivals (seed 1004) until every
    request has completed, admitted by `policy`; p50/p99 time to completion
    and throughput."""
    from mpm_3d_b200.native import GPUServer
    from mpm_3d_b200.serving import run_stream

    specs = inputs.serving_stream(rate=100.0, duration=seconds, seed=1004)
    srv = GPUServer(budget_bytes=150 * 10**9, mode="mixed", device=device, sort_interval=sort_interval)
    rep = run_stream(srv, specs, round_steps=round_steps, policy=policy)
    srv.close()
    out = rep.summary()
    out.update({"arrivals_s": seconds, "rate_per_s": 100.0, "budget_bytes": 150 * 10**9, "round_steps": round_steps,
                "form": "mixed"})
    return out


def run_serving_workload(args, rank, world, local):
    import torch

    torch.cuda.set_device(local)
    rep = run_serving(args.serve_seconds, local, policy=args.policy)
    rep_max = max_over_ranks(rep["makespan_s"], world)
    steps_all = sum_over_ranks(float(rep["particle_steps"]), world)
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": steps_all / rep_max, "unit": UNIT, "n_gpus": world, "steps": None,
        "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (mpm_3d_b200.inputs.serving_stream, seed 1004)",
        "config": {"workload": "serving", "arrivals_s": args.serve_seconds, "rate_per_s": 100.0,
                   "budget_bytes": 150 * 10**9, "form": "mixed", "policy": args.policy,
                   "parallelism": f"independent{world}"},
        "serving": rep,
        "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)


def run_e2e_batch(cases, steps: int, device: int, kernel, sort_interval: int, mode: str = "mixed"):
    """The ensemble through the C ABI from host buffers: batch creation and
    upload of every job, `steps` steps (each job stops at its own count),
    download of every point's x, x_t and stress, teardown, all on the wall
    clock."""
    import torch

    from mpm_3d_b200.native import GPUBatch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    phases = {}
    b = GPUBatch(dim=3, mode=mode, device=device, sort_interval=sort_interval, kernel=kernel)
    jobs = [b.add(c) for c in cases]
    t1 = time.perf_counter()
    phases["create_upload_s"] = t1 - t0
    b.step(steps)
    b.synchronize()
    t2 = time.perf_counter()
    phases["steps_s"] = t2 - t1
    d2h = 0
    for f in ("x", "x_t", "T"):
        d2h += sum(o.nbytes for o in b.points_many(jobs, 0, f))
    t3 = time.perf_counter()
    phases["download_s"] = t3 - t2
    b.close()
    dt = time.perf_counter() - t0
    phases["teardown_s"] = dt - (t3 - t0)
    psteps = sum(c.n_points * min(c.steps, steps) for c in cases)
    h2d = sum(b_.n * (8 + 8 + 24 + 24 + 4) for c in cases for b_ in c.bodies)
    return {"value": psteps / dt, "unit": UNIT, "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps,
            "steps": steps, "seconds": dt, "phases": {k: round(v, 3) for k, v in phases.items()}}


def cpu_thread_variants(cases, steps: int = 2):
    """The reference's solver on 4 of the ensemble's jobs (every 128th) with
    one thread (the serial ExplicitUSL) and with all host threads but one
    (ThreadPoolExplicitUSL's main thread busy-waits on its workers,
    threadpool_explicit_usl.cpp:327-343)."""
    cores = os.cpu_count() or 1
    ids = list(range(0, len(cases), max(1, len(cases) // 4)))[:4]
    out = {}
    for t in sorted({1, max(1, cores - 1)}):
        sec = sum(cpu_reference_run(cases[i], steps, 1, t) * steps for i in ids)
        pts = sum(cases[i].n_points * steps for i in ids)
        out[f"threads_{t}"] = pts / sec
    out.update({"unit": UNIT, "jobs": ids, "steps": steps,
                "solver": "ExplicitUSL (1 thread), ThreadPoolExplicitUSL+ThreadPoolPoints (more)"})
    return out


def cpu_ensemble_sample(cases, steps: int, warmup: int = 1):
    """The reference's ThreadPoolExplicitUSL on 16 of the jobs (every 32nd),
    one after another, `steps` steps each after `warmup` warm-up steps."""
    threads = os.cpu_count() or 1
    ids = list(range(0, len(cases), max(1, len(cases) // 16)))[:16]
    pts = 0
    sec = 0.0
    for i in ids:
        dt = cpu_reference_run(cases[i], steps, warmup, threads)
        sec += dt * steps
        pts += cases[i].n_points * steps
    return {"value": pts / sec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"jobs {ids[0]}..{ids[-1]} step {ids[1] - ids[0] if len(ids) > 1 else 1} "
                      f"({len(ids)} jobs, {sum(cases[i].n_points for i in ids)} points), {steps} steps each after {warmup} "
                      f"warm-up, in sequence, ThreadPoolExplicitUSL+ThreadPoolPoints, threads={threads}"}


def run_e2e(case, steps: int, device: int, form: str = "fp64"):
    """Same metric through the C ABI from host buffers: create + upload,
    `steps` steps, download of every point's x, x_t and stress, destroy."""
    import torch

    from mpm_3d_b200.native import GPUExplicitUSL

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim = GPUExplicitUSL(case, device=device, mode=form)
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


def parse_kernel(spec: str):
    """'FORM/POINTS' -> (form, points per work item); '' -> None."""
    if not spec:
        return None
    form, _, cap = spec.partition("/")
    from mpm_3d_b200.native import KERNELS

    if form not in KERNELS or not cap.isdigit():
        raise SystemExit(f"--kernel wants FORM/POINTS with FORM one of {sorted(KERNELS)}")
    return form, int(cap)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=0, help="timed steps (default: the workload's own step count)")
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--workload", default="ensemble",
                    choices=["ensemble", "collision", "column", "serving", "blockdrop2d"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed", "fp64_deterministic"], help="form of the single-job workloads")
    ap.add_argument("--plain-steps", type=int, default=10, help="timed steps per job of the plain FP64 path")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--jobs", type=int, default=0, help="ensemble: only the first JOBS jobs (profiling cases)")
    ap.add_argument("--only-mixed", action="store_true", help="ensemble: skip the FP64 batch")
    ap.add_argument("--only-fp64", action="store_true", help="ensemble: skip the mixed batch")
    ap.add_argument("--no-errors", action="store_true",
                    help="ensemble: skip the 500-step error comparison of the forms (profiling runs)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="seconds of request arrivals of the serving stream (0: none)")
    ap.add_argument("--no-column", action="store_true", help="ensemble: skip the column FP64 record")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-steps", type=int, default=4, help="steps of the CPU reference sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--kernel", default="", metavar="FORM/POINTS",
                    help="fix the fused kernel's form and points per work item (e.g. point_per_thread/256) "
                         "instead of the default (single jobs) or the autotuner's choice (batches)")
    ap.add_argument("--sort-interval", type=int, default=8, help="re-binning interval of a batch with --kernel")
    ap.add_argument("--policy", default="fifo", choices=["fifo", "fit"], help="admission policy of the serving stream")
    args = ap.parse_args()
    args.kernel = parse_kernel(args.kernel)
    if args.warmup < 3:
        args.warmup = 3
    if args.steps <= 0:
        args.steps = 100 if args.workload in ("ensemble", "serving") else make_workload(args.workload).steps
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world)
        elif args.workload == "ensemble":
            run_ensemble(args, rank, world, local)
        elif args.workload == "serving":
            run_serving_workload(args, rank, world, local)
        else:
            run_single(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
