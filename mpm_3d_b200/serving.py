"""Serving driver: replays a stream of simulation requests against a server.

Requests arrive at their (Poisson) arrival times on the wall clock and wait
in a queue. Under the ``fifo`` policy the head of the queue is submitted as
soon as the server admits it (its device footprint fits the memory budget
left by the running requests) and nothing passes it. Under the ``fit``
policy (backfilling) requests behind a head that does not fit are submitted
too when they fit, within a look-ahead window; the head can be passed in at
most ``max_bypass`` rounds, after which admission waits for it again, so no
request waits for ever. A request larger than the whole budget is rejected
by the server and dropped from the queue. The server advances everything
running in rounds of a few steps (continuous batching: requests join and
leave between rounds while the others keep stepping). A request's time to
completion runs from its arrival to the end of the round in which its last
step ran.

The server is anything with the ``GPUServer`` interface (``submit`` returning
a request id, None when it does not fit now, or -1 when it can never fit;
``advance``, ``poll``, ``request``, ``result``, ``release``, ``stats``), so
the queueing logic is tested on the host with a stand-in.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Callable, Dict, List, Optional

import numpy as np

from . import inputs


@dataclasses.dataclass
class Completed:
    spec: inputs.RequestSpec
    rid: int
    arrival: float      # seconds after the stream started
    admitted: float
    done: float
    points: int
    steps: int

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclasses.dataclass
class StreamReport:
    completed: List[Completed]
    makespan: float            # first arrival to last completion (seconds)
    particle_steps: int        # over the completed requests
    max_running: int
    max_queue: int
    rejected: int = 0          # requests larger than the whole budget
    policy: str = "fifo"

    def percentile(self, q: float) -> float:
        return float(np.percentile([c.latency for c in self.completed], q)) if self.completed else float("nan")

    def summary(self) -> Dict[str, float]:
        return {"requests": len(self.completed), "p50_s": self.percentile(50), "p99_s": self.percentile(99),
                "mean_s": float(np.mean([c.latency for c in self.completed])) if self.completed else float("nan"),
                "makespan_s": self.makespan, "particle_steps": self.particle_steps,
                "throughput": self.particle_steps / self.makespan if self.makespan > 0 else 0.0,
                "max_running": self.max_running, "max_queue": self.max_queue, "rejected": self.rejected,
                "policy": self.policy}


def run_stream(server, specs: List[inputs.RequestSpec], round_steps: int = 20,
               make_case: Callable[[inputs.RequestSpec], inputs.Case] = inputs.serving_case,
               on_complete: Optional[Callable[[Completed], None]] = None,
               clock: Callable[[], float] = time.perf_counter, sleep: Callable[[float], None] = time.sleep,
               release: bool = True, policy: str = "fifo", lookahead: int = 32,
               max_bypass: int = 8) -> StreamReport:
    """Replays ``specs`` (sorted by arrival) against ``server`` until every
    request has completed or been rejected. ``on_complete`` sees each
    finished request while its results are still held by the server (they
    are released after it, unless ``release`` is False). ``policy`` is
    ``fifo`` or ``fit`` (see the module docstring)."""
    if policy not in ("fifo", "fit"):
        raise ValueError(f"unknown admission policy {policy}")
    t0 = clock()
    queue: List[inputs.RequestSpec] = []
    cases: Dict[int, inputs.Case] = {}   # cases built for the look-ahead window, by spec index
    meta: Dict[int, tuple] = {}
    done: List[Completed] = []
    i = 0
    running = 0
    max_running = 0
    max_queue = 0
    rejected = 0
    head_bypassed = 0                    # rounds in which the current head was passed
    while i < len(specs) or queue or running > 0:
        now = clock() - t0
        while i < len(specs) and specs[i].arrival <= now:
            queue.append(specs[i])
            i += 1
        max_queue = max(max_queue, len(queue))
        # admission: the head first; under `fit`, later requests of the
        # window too while the head has not been passed too often
        k = 0
        passed_head = False
        while k < len(queue) and k < (lookahead if policy == "fit" else 1):
            spec = queue[k]
            case = cases.get(spec.index)
            if case is None:
                case = cases[spec.index] = make_case(spec)
            rid = server.submit(case, spec.steps)
            if rid is not None and rid < 0:      # larger than the whole budget
                rejected += 1
                cases.pop(spec.index, None)
                queue.pop(k)
                if k == 0:
                    head_bypassed = 0
                continue
            if rid is None:
                if k == 0 and (policy == "fifo" or head_bypassed >= max_bypass):
                    break
                k += 1
                continue
            queue.pop(k)
            cases.pop(spec.index, None)
            meta[rid] = (spec, clock() - t0, case.n_points)
            running += 1
            if k == 0:
                head_bypassed = 0
            else:
                passed_head = True
        if passed_head:
            head_bypassed += 1
        max_running = max(max_running, running)
        if running == 0:
            if i < len(specs):
                sleep(max(0.0, specs[i].arrival - (clock() - t0)))
            continue
        server.advance(round_steps)
        finished = server.poll()
        t_done = clock() - t0
        for rid in finished:
            spec, t_adm, pts = meta.pop(rid)
            c = Completed(spec, rid, spec.arrival, t_adm, t_done, pts, spec.steps)
            done.append(c)
            running -= 1
            if on_complete is not None:
                on_complete(c)
            if release:
                server.release(rid)
    makespan = (max(c.done for c in done) - specs[0].arrival) if done else 0.0
    return StreamReport(done, makespan, int(sum(c.points * c.steps for c in done)), max_running, max_queue, rejected,
                        policy)
