"""Parity with the oracle on the benchmark configurations themselves, at
their full sizes.

The other parity tests run reduced grids and point counts; these run the
seeded configurations the benchmark measures, through the C ABI, against
the C restatement of the reference (oracle/mpm_oracle.c, pinned bit for bit
to the reference's own sources by tests/test_oracle.py), per step, with the
FP64 tolerance of every parity test (1e-10 relative per field, util.py):

* the 2D block drop (144 points, 20x20 grid) for all of its 2000 steps;
* the two-body collision at full size (524,288 points, 128^3 grid,
  ContactHuang mu = 0.4, DefaultDriver gravity) for 3 steps. As configured,
  its cubes start 0.15 m apart and close at 2 m/s, so they do not meet
  within the configuration's 1000 steps; a variant with the second cube one
  cell from the first exercises the contact normal and force at the same
  size;
* the column collapse at full size (3,145,728 points, 256x256x128 grid) for
  2 steps; the oracle keeps the reference's COO triplets (about 10 GB for
  this body), so the case is skipped with its reason on a host with less
  than 24 GB of memory available;
* jobs of the 512-job block-drop ensemble stepped inside the full FP64
  batch (one launch per stage over every job), compared per step for their
  first 10 steps with the same jobs run alone by the oracle.
"""
import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUBatch, GPUExplicitUSL
from util import FP64_TOL, assert_close, field_floor

pytestmark = pytest.mark.gpu

POINT_FIELDS = ["x", "u", "x_t", "mx_t", "T", "L", "v", "active"]
NODE_FIELDS = ["m", "mx_t", "f", "x_t", "u", "diff_x_t"]


@pytest.fixture(scope="module", autouse=True)
def restated_lib():
    bridge.build_restated()


def _available_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def _per_step_parity(case, steps, node_fields=NODE_FIELDS):
    ref = bridge.RestatedJob(case)
    gpu = GPUExplicitUSL(case, keep_debug=True)
    worst = {}
    contact_nodes = 0
    for s in range(steps):
        ref.step(1)
        gpu.step(1)
        for b in range(len(case.bodies)):
            for f in POINT_FIELDS:
                e = assert_close(gpu.points(b, f), ref.points(b, f), FP64_TOL, f"{case.name} step {s} body {b} {f}",
                                 field_floor(case, f))
                worst[f] = max(worst.get(f, 0.0), e)
            for f in node_fields:
                e = assert_close(gpu.nodes(b, f), ref.nodes(b, f), FP64_TOL, f"{case.name} step {s} body {b} node {f}")
                worst["n_" + f] = max(worst.get("n_" + f, 0.0), e)
        for c in range(len(case.contacts)):
            assert_close(gpu.contact(c, "force"), ref.contact(c, "force"), FP64_TOL, f"{case.name} step {s} contact force")
            m1 = ref.nodes(case.contacts[c].b1, "m")[:, 0]
            m2 = ref.nodes(case.contacts[c].b2, "m")[:, 0]
            both = (m1 > 0) & (m2 > 0)
            contact_nodes = max(contact_nodes, int(both.sum()))
            if both.any():
                assert_close(gpu.contact(c, "normal")[both], ref.contact(c, "normal")[both], FP64_TOL,
                             f"{case.name} step {s} contact normal")
    gpu.close()
    print(case.name, case.n_points, "points", {k: f"{v:.1e}" for k, v in worst.items()})
    return contact_nodes


def test_block_drop_2d_all_2000_steps():
    case = inputs.block_drop_2d()
    assert case.n_points == 144 and case.steps == 2000
    _per_step_parity(case, case.steps)


def test_two_body_collision_full_size():
    case = inputs.two_body_collision_3d(128)
    assert case.n_points == 524288
    assert _per_step_parity(case, 3) == 0      # 0.15 m apart: no node carries both bodies yet


def test_two_body_collision_full_size_in_contact():
    case = inputs.two_body_collision_3d(128, gap=1.0 / 128)
    assert case.n_points == 524288
    assert _per_step_parity(case, 3) > 1000    # the contact rules act on the shared nodes


def test_column_collapse_full_size():
    need = 24.0
    if _available_gb() < need:
        pytest.skip(f"the oracle's COO triplets of the full column need about {need:.0f} GB of host memory; "
                    f"{_available_gb():.0f} GB available")
    case = inputs.column_collapse_3d(1)
    assert case.n_points == 3145728
    _per_step_parity(case, 2)


def test_ensemble_jobs_inside_the_full_fp64_batch():
    cases = inputs.block_drop_ensemble(512, seed=1003)
    sample = list(range(0, 512, 64))    # 8 jobs spread over the draw
    b = GPUBatch(dim=3, mode="fp64")
    jobs = [b.add(c) for c in cases]
    refs = {i: bridge.RestatedJob(cases[i]) for i in sample}
    worst = 0.0
    for s in range(10):
        b.step(1)
        for i in sample:
            refs[i].step(1)
            for f in ("x", "u", "x_t", "T", "v", "active"):
                e = assert_close(b.points(jobs[i], 0, f), refs[i].points(0, f), FP64_TOL,
                                 f"ensemble job {i} step {s} {f}", field_floor(cases[i], f))
                worst = max(worst, e)
    b.close()
    print("ensemble sample", sample, f"worst {worst:.1e}")
