"""Host logic of the serving driver (mpm_3d_b200.serving.run_stream) with a
stand-in server on a virtual clock: arrival-order admission under a memory
budget, requests joining and leaving between rounds, completion times, the
rejection of requests larger than the whole budget, and the backfilling
policy (requests that fit pass a head that does not, a bounded number of
times)."""
import numpy as np

from mpm_3d_b200 import inputs
from mpm_3d_b200.serving import run_stream


class FakeCase:
    def __init__(self, spec):
        self.n_points = 100 * spec.n


class FakeServer:
    """Admits while the points of the running requests fit `budget` (and
    rejects a request larger than the whole budget, as the GPU server does);
    every advance takes `sec_per_step` virtual seconds per step."""

    def __init__(self, budget, clock, sec_per_step=0.001):
        self.budget = budget
        self.clock = clock
        self.sec = sec_per_step
        self.running = {}
        self.finished = []
        self.next_id = 0
        self.admit_order = []
        self.max_reserved = 0

    def submit(self, case, steps):
        if case.n_points > self.budget:
            return -1
        used = sum(c for c, _ in self.running.values())
        if used + case.n_points > self.budget:
            return None
        rid = self.next_id
        self.next_id += 1
        self.running[rid] = (case.n_points, steps)
        self.admit_order.append(rid)
        self.max_reserved = max(self.max_reserved, used + case.n_points)
        return rid

    def advance(self, k):
        self.clock.t += k * self.sec
        for rid in list(self.running):
            pts, left = self.running[rid]
            left -= k
            if left <= 0:
                del self.running[rid]
                self.finished.append(rid)
            else:
                self.running[rid] = (pts, left)

    def poll(self):
        out, self.finished = self.finished, []
        return out

    def release(self, rid):
        pass


class VClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


def _specs():
    return inputs.serving_stream(rate=200.0, duration=0.5, seed=11, n_range=(4, 40), steps_range=(10, 200))


def test_all_requests_complete_in_arrival_order_under_the_budget():
    specs = _specs()
    clk = VClock()
    srv = FakeServer(budget=6000, clock=clk)
    rep = run_stream(srv, specs, round_steps=10, make_case=FakeCase, clock=clk, sleep=clk.sleep)
    assert len(rep.completed) == len(specs)
    # admission follows arrival order (first in, first admitted)
    admitted = sorted(rep.completed, key=lambda c: c.rid)
    assert [c.spec.index for c in admitted] == sorted(s.index for s in specs)
    # nothing ran beyond the budget
    assert srv.max_reserved <= 6000
    for c in rep.completed:
        assert c.admitted >= c.arrival - 1e-12
        assert c.done >= c.admitted
        # a request needs at least its own steps of virtual time
        assert c.done - c.admitted >= c.steps * srv.sec - 10 * srv.sec - 1e-9
    s = rep.summary()
    assert s["p99_s"] >= s["p50_s"] > 0
    assert s["particle_steps"] == sum(100 * sp.n * sp.steps for sp in specs)


def test_larger_budget_means_shorter_latency():
    specs = _specs()
    out = []
    for budget in (4000, 30000):
        clk = VClock()
        srv = FakeServer(budget=budget, clock=clk)
        rep = run_stream(srv, specs, round_steps=10, make_case=FakeCase, clock=clk, sleep=clk.sleep)
        out.append(rep.percentile(99))
    assert out[1] < out[0]


def test_stream_is_seeded_poisson():
    a = inputs.serving_stream(rate=100.0, duration=60.0, seed=1004)
    b = inputs.serving_stream(rate=100.0, duration=60.0, seed=1004)
    assert [x.arrival for x in a] == [x.arrival for x in b]
    gaps = np.diff([x.arrival for x in a])
    assert abs(len(a) - 6000) < 300                 # ~rate * duration
    assert abs(gaps.mean() - 0.01) < 0.001           # exponential gaps, mean 1/rate
    frac = sum(x.kind == "contact" for x in a) / len(a)
    assert 0.07 < frac < 0.13
    ns = np.array([x.n for x in a])
    assert ns.min() >= 16 and ns.max() <= 128


def test_request_larger_than_the_budget_is_rejected():
    specs = _specs()
    big = max(specs, key=lambda s: s.n)
    clk = VClock()
    srv = FakeServer(budget=100 * big.n - 1, clock=clk)   # the largest request can never fit
    rep = run_stream(srv, specs, round_steps=10, make_case=FakeCase, clock=clk, sleep=clk.sleep)
    n_big = sum(s.n == big.n for s in specs)
    assert rep.rejected == n_big
    assert len(rep.completed) == len(specs) - n_big
    assert big.index not in {c.spec.index for c in rep.completed}


def _blocked_head_stream():
    """A large request arrives first behind a running medium one, then a
    stream of small ones that fit beside the medium one but not beside the
    large one."""
    specs = []
    mk = lambda i, t, n, steps: inputs.RequestSpec(index=i, arrival=t, kind="block", n=n, steps=steps, mu=0.0, seed=i)
    specs.append(mk(0, 0.0, 30, 400))     # medium, runs first
    specs.append(mk(1, 0.001, 50, 100))   # large: waits for the medium one
    for i in range(2, 40):
        specs.append(mk(i, 0.001 + 0.001 * i, 5, 20))
    return specs


def test_backfill_lets_small_requests_pass_a_blocked_head():
    specs = _blocked_head_stream()
    lat = {}
    for policy in ("fifo", "fit"):
        clk = VClock()
        srv = FakeServer(budget=6000, clock=clk)
        rep = run_stream(srv, specs, round_steps=10, make_case=FakeCase, clock=clk, sleep=clk.sleep, policy=policy,
                         max_bypass=1000)
        assert len(rep.completed) == len(specs) and rep.policy == policy
        lat[policy] = {c.spec.index: c.latency for c in rep.completed}
    small = range(2, 40)
    assert np.median([lat["fit"][i] for i in small]) < 0.5 * np.median([lat["fifo"][i] for i in small])


def test_backfill_bounds_how_often_the_head_is_passed():
    specs = _blocked_head_stream()
    ahead = {}
    for max_bypass in (2, 1000):
        clk = VClock()
        srv = FakeServer(budget=6000, clock=clk)
        rep = run_stream(srv, specs, round_steps=10, make_case=FakeCase, clock=clk, sleep=clk.sleep, policy="fit",
                         max_bypass=max_bypass)
        assert len(rep.completed) == len(specs)
        order = [c.spec.index for c in sorted(rep.completed, key=lambda c: (c.admitted, c.rid))]
        ahead[max_bypass] = order.index(1)   # requests admitted before the large head
    # with a bound of two rounds only the small requests of those rounds pass
    # the head; without one, every small request that arrives before the
    # medium request leaves does
    assert ahead[2] < ahead[1000]
    assert ahead[1000] == len(specs) - 1
