"""The deterministic FP64 form (MPMGPU_MODE_FP64_DETERMINISTIC).

Nodal sums are pre-rounded into two levels whose partial sums are exact in
any order (kernels_fp64.cuh, make_split / presplit), so the result cannot
depend on the order of the atomics, on the point storage order (re-binning
interval) or on the other jobs of a batch: runs are compared bit for bit.
Against the oracle it meets the FP64 tolerance of the plain form (1e-10).
"""
import numpy as np
import pytest

import bridge  # noqa: F401  (oracle build fixture in test_gpu_parity)
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUBatch, GPUExplicitUSL
from test_gpu_parity import CASES, _step_parity
from util import bits_equal

pytestmark = pytest.mark.gpu

POINT = ["x", "u", "x_t", "T", "v", "active"]


@pytest.fixture(scope="module", autouse=True)
def restated_lib():
    bridge.build_restated()


@pytest.mark.parametrize("name", ["collision_3d_touching", "column_collapse_s16", "block_drop_2d", "collision_2d",
                                  "wall_exit_2d"])
def test_deterministic_parity_with_oracle(name):
    _step_parity(name, mode="fp64_deterministic")


def _run(case, steps, sort_interval):
    sim = GPUExplicitUSL(case, mode="fp64_deterministic", sort_interval=sort_interval, keep_debug=True)
    sim.step(steps)
    pts = [{f: sim.points(b, f) for f in POINT} for b in range(len(case.bodies))]
    nodes = [{f: sim.nodes(b, f) for f in ("m", "mx_t", "f", "x_t")} for b in range(len(case.bodies))]
    sim.close()
    return pts, nodes


def _same(a, b):
    for x, y in zip(a, b):
        for f in x:
            if not bits_equal(x[f], y[f]):
                return f
    return None


@pytest.mark.parametrize("make,steps", [(lambda: inputs.two_body_collision_3d(16, steps=25, gap=0.01), 25),
                                        (lambda: inputs.column_collapse_3d(scale=8, steps=20), 20),
                                        (lambda: inputs.two_body_collision_2d(20, steps=60), 60)])
def test_bit_reproducible_across_runs_and_point_orders(make, steps):
    case = make()
    p1, n1 = _run(case, steps, 32)
    p2, n2 = _run(case, steps, 32)
    assert _same(p1, p2) is None and _same(n1, n2) is None, "two identical runs differ"
    # re-binning every 3 steps stores the points in other orders: the
    # atomics then add in other orders, and the bits must not change
    p3, n3 = _run(case, steps, 3)
    assert _same(p1, p3) is None, f"point field {_same(p1, p3)} depends on the point order"
    assert _same(n1, n3) is None, f"node field {_same(n1, n3)} depends on the point order"


def test_plain_fp64_is_not_bit_reproducible_but_deterministic_is():
    """The check above has teeth: in the plain FP64 form the same comparison
    sees the atomics' order (at least one bit of one field differs)."""
    case = inputs.column_collapse_3d(scale=8, steps=20)
    runs = []
    for si in (32, 3):
        sim = GPUExplicitUSL(case, mode="fp64", sort_interval=si)
        sim.step(20)
        runs.append([{f: sim.points(0, f) for f in ("x", "x_t", "T")}])
        sim.close()
    assert _same(runs[0], runs[1]) is not None


def test_job_alone_and_in_a_batch_are_the_same_bits():
    cases = inputs.block_drop_ensemble(count=5, seed=9, n_range=(10, 24), steps=30)
    alone = []
    for c in cases:
        sim = GPUExplicitUSL(c, mode="fp64_deterministic")
        sim.step(30)
        alone.append([{f: sim.points(0, f) for f in POINT}])
        sim.close()
    batch = GPUBatch(dim=3, mode="fp64_deterministic")
    jobs = [batch.add(c) for c in cases]
    batch.step(30)
    for j, a in zip(jobs, alone):
        got = [{f: batch.points(j, 0, f) for f in POINT}]
        assert _same(got, a) is None, f"job {j}: {_same(got, a)} differs alone and in the batch"
    batch.close()
