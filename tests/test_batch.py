"""The batched step (mpmgpu_batch_*) against single-job handles.

Every job of a batch must compute what a single-job handle computes for the
same inputs; only the order of the nodal sums differs, so FP64 batch results
match FP64 handle results within the FP64 parity tolerance (1e-10, util.py)
after every job's own step count. Jobs join mid-run, stop at their own step
counts, leave, and reuse freed node-block ranges; the autotuner leaves the
jobs' state untouched. The mixed form (FP32 point state, FP64 nodal sums) is
compared with the FP64 form within 1e-4 relative error, the bound the mixed
form is held to.
"""
import numpy as np
import pytest

from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUBatch, GPUExplicitUSL
from util import FP64_TOL, rel_err, field_floor

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
FIELDS = ["x", "x_t", "T", "v"]


def _solo(case, steps, mode="fp64"):
    sim = GPUExplicitUSL(case, mode=mode)
    sim.step(steps)
    out = [{f: sim.points(b, f) for f in FIELDS} for b in range(len(case.bodies))]
    sim.close()
    return out


def _from_batch(batch, job, case):
    return [{f: batch.points(job, b, f) for f in FIELDS} for b in range(len(case.bodies))]


def _compare(case, got, ref, tol, what):
    worst = 0.0
    for b in range(len(case.bodies)):
        for f in FIELDS:
            e = rel_err(got[b][f], ref[b][f], field_floor(case, f))
            worst = max(worst, e)
            assert e <= tol, f"{what}: body {b} field {f}: relative error {e:.3e} > {tol:.1e}"
    return worst


def _cases():
    ens = inputs.block_drop_ensemble(count=4, seed=7, n_range=(8, 20), steps=30, side_range=(0.2, 0.35))
    coll = inputs.two_body_collision_3d(16, steps=20, gap=0.01)
    col = inputs.column_collapse_3d(scale=16, steps=12)
    return ens + [coll, col]


def test_batch_matches_single_handles():
    cases = _cases()
    batch = GPUBatch(dim=3, mode="fp64")
    jobs = [batch.add(c) for c in cases]
    batch.step(max(c.steps for c in cases) + 5)
    batch.synchronize()
    for j, c in zip(jobs, cases):
        done, left = batch.state(j)
        assert (done, left) == (c.steps, 0), (c.name, done, left)
        _compare(c, _from_batch(batch, j, c), _solo(c, c.steps), FP64_TOL, c.name)
    batch.close()


def test_jobs_join_mid_run_and_stop_at_their_counts():
    cases = _cases()
    batch = GPUBatch(dim=3, mode="fp64")
    a = batch.add(cases[0])              # 30 steps
    batch.step(7)
    b = batch.add(cases[4])              # collision, 20 steps, joins at step 7
    c = batch.add(cases[1], steps=9)     # stops after 9 of its own steps
    batch.step(40)
    batch.synchronize()
    assert batch.state(a) == (30, 0)
    assert batch.state(b) == (20, 0)
    assert batch.state(c) == (9, 0)
    _compare(cases[0], _from_batch(batch, a, cases[0]), _solo(cases[0], 30), FP64_TOL, "joined first")
    _compare(cases[4], _from_batch(batch, b, cases[4]), _solo(cases[4], 20), FP64_TOL, "joined at step 7")
    _compare(cases[1], _from_batch(batch, c, cases[1]), _solo(cases[1], 9), FP64_TOL, "stopped at 9")
    batch.close()


def test_remove_and_reuse_block_ranges():
    cases = _cases()
    batch = GPUBatch(dim=3, mode="fp64")
    a = batch.add(cases[0])
    b = batch.add(cases[1])
    batch.step(5)
    batch.remove(a)
    jobs_before, _, _ = batch.counts()
    assert jobs_before == 1
    c = batch.add(cases[2])              # takes the freed range
    batch.step(40)
    batch.synchronize()
    _compare(cases[2], _from_batch(batch, c, cases[2]), _solo(cases[2], cases[2].steps), FP64_TOL, "reused range")
    _compare(cases[1], _from_batch(batch, b, cases[1]), _solo(cases[1], cases[1].steps), FP64_TOL, "neighbour")
    batch.close()


def test_table_launch_with_many_items_per_cta():
    """More than four bodies: one launch over the body table, and more work
    items than CTAs, so every CTA walks several items (its table-entry
    slots alternate)."""
    col = inputs.column_collapse_3d(scale=2, steps=6)
    tiny = inputs.block_drop_ensemble(count=4, seed=5, n_range=(8, 10), steps=6)
    cases = [col] + tiny
    batch = GPUBatch(dim=3, mode="fp64")
    jobs = [batch.add(c) for c in cases]
    batch.step(6)
    batch.synchronize()
    for j, c in zip(jobs, cases):
        _compare(c, _from_batch(batch, j, c), _solo(c, c.steps), FP64_TOL, c.name)
    batch.close()


def test_graph_replay_matches_direct_launches():
    cases = _cases()[:3]
    runs = []
    for graph in (True, False):
        batch = GPUBatch(dim=3, mode="fp64", graph=graph)
        jobs = [batch.add(c) for c in cases]
        batch.step(40)
        runs.append([_from_batch(batch, j, c) for j, c in zip(jobs, cases)])
        batch.close()
    for c, g, d in zip(cases, runs[0], runs[1]):
        _compare(c, g, d, FP64_TOL, c.name)


def test_autotune_keeps_the_state():
    cases = _cases()
    batch = GPUBatch(dim=3, mode="fp64")
    jobs = [batch.add(c) for c in cases]
    batch.step(3)
    cap = batch.autotune(steps=4)
    assert cap in (128, 256, 512, 1024)
    assert batch.points_per_item() == cap
    batch.step(40)
    batch.synchronize()
    for j, c in zip(jobs, cases):
        assert batch.state(j) == (c.steps, 0)
        _compare(c, _from_batch(batch, j, c), _solo(c, c.steps), FP64_TOL, c.name)
    batch.close()


@pytest.mark.parametrize("cap", [256, 512, 1024])
def test_mixed_batch_within_1e4_of_fp64(cap):
    cases = _cases()
    batch = GPUBatch(dim=3, mode="mixed", points_per_item=cap)
    jobs = [batch.add(c) for c in cases]
    batch.step(40)
    batch.synchronize()
    for j, c in zip(jobs, cases):
        _compare(c, _from_batch(batch, j, c), _solo(c, c.steps), MIXED_TOL, f"mixed {c.name}")
    batch.close()


def test_mixed_single_handle_within_1e4_of_fp64():
    for c in [inputs.two_body_collision_3d(16, steps=20, gap=0.01), inputs.column_collapse_3d(scale=8, steps=20)]:
        _compare(c, _solo(c, c.steps, mode="mixed"), _solo(c, c.steps), MIXED_TOL, f"mixed {c.name}")


def test_mixed_2d_single_handle():
    c = inputs.block_drop_2d()
    _compare(c, _solo(c, 200, mode="mixed"), _solo(c, 200), MIXED_TOL, "mixed 2D block drop")


def test_mixed_neohookean_and_boundaries_within_1e4_of_fp64():
    """The adjacent material and boundaries in the mixed form (FP32 point
    state and deformation gradient, FP64 nodal sums): a neo-Hookean
    collision and a block on a frictional floor, against FP64."""
    coll = inputs.two_body_collision_3d(16, steps=20, gap=0.01)
    for b in coll.bodies:
        b.material_class = "CompressibleNeohookeanElasticity"
    slide = inputs.sliding_block(3, "CartesianFrictionalBox", mu=0.3, n_cells=12, steps=20)
    for c in (coll, slide):
        _compare(c, _solo(c, c.steps, mode="mixed"), _solo(c, c.steps), MIXED_TOL, f"mixed {c.name}")


def test_mixed_sand_within_1e4_of_fp64():
    """Sand_SachithLocal in the mixed form (FP32 point state, stress and
    plastic strain; FP64 nodal sums) against FP64: the 2D and 3D granular
    columns, with their elastic, plastic-return and zero-stress points."""
    for c in (inputs.sand_column(2, steps=80), inputs.sand_column(3, n_cells=12, steps=30)):
        _compare(c, _solo(c, c.steps, mode="mixed"), _solo(c, c.steps), MIXED_TOL, f"mixed {c.name}")
