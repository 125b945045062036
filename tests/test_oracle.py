"""Pins the oracle.

1. The C restatement (oracle/mpm_oracle.c) reproduces, bit for bit, the golden
   fixtures written by the reference's own sources (tests/golden/make_golden.py).
2. Where the reference build is present (oracle/_ref/libmpmref_parity.so),
   the restatement matches it bit for bit step by step on fresh seeded cases.
"""
import os
import tempfile

import numpy as np
import pytest

import bridge
from golden.make_golden import NODE_FIELDS, POINT_FIELDS, golden_cases, point_fields
from mpm_3d_b200 import inputs
from util import bits_equal

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", autouse=True)
def restated_lib():
    bridge.build_restated()


@pytest.mark.parametrize("name", sorted(golden_cases()))
def test_restated_matches_golden(name):
    case, snaps = golden_cases()[name]
    gold = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    assert list(gold["snaps"]) == snaps
    job = bridge.RestatedJob(case)
    job.build_map()
    for b in range(len(case.bodies)):
        node, pt, val = job.map(b)
        gnode, gpt, grad = job.grad_map(b)
        assert np.array_equal(node, gold[f"map_b{b}_node"]) and np.array_equal(pt, gold[f"map_b{b}_point"])
        assert np.array_equal(gnode, node) and np.array_equal(gpt, pt)
        assert bits_equal(val, gold[f"map_b{b}_S"])
        assert bits_equal(grad, gold[f"map_b{b}_grad"])
    done = 0
    for s in snaps:
        job.step(s - done)
        done = s
        for b in range(len(case.bodies)):
            for f in point_fields(case.bodies[b]):
                assert bits_equal(job.points(b, f), gold[f"s{s}_b{b}_p_{f}"]), f"{name} step {s} point {f}"
            for f in NODE_FIELDS:
                assert bits_equal(job.nodes(b, f), gold[f"s{s}_b{b}_n_{f}"]), f"{name} step {s} node {f}"
        for c in range(len(case.contacts)):
            for f in ("normal", "force"):
                assert bits_equal(job.contact(c, f), gold[f"s{s}_c{c}_{f}"]), f"{name} step {s} contact {f}"


def test_golden_cases_exercise_contact():
    gold = np.load(os.path.join(GOLDEN, "collision_3d_touching.npz"))
    force = gold["s6_c0_force"]
    assert (np.abs(force).sum(axis=1) > 0).sum() > 10
    gold = np.load(os.path.join(GOLDEN, "wall_collision_2d_reflected.npz"))
    assert (np.abs(gold["s15_c0_force"]).sum(axis=1) > 0).sum() > 0


def test_golden_cases_exercise_their_classes():
    """The fixtures of the adjacent classes are not trivially equal to the
    defaults: friction slows the sliding block more than the slip wall, and
    the neo-Hookean stress departs from the linear one."""
    friction = np.load(os.path.join(GOLDEN, "sliding_2d_frictional.npz"))
    first, last = friction["s1_b0_p_x_t"][:, 0], friction["s15_b0_p_x_t"][:, 0]
    assert last.mean() < 0.9 * first.mean()
    neo = np.load(os.path.join(GOLDEN, "collision_2d_neohookean.npz"))["s40_b0_p_T"]
    lin = np.load(os.path.join(GOLDEN, "collision_2d.npz"))["s40_b0_p_T"]
    assert np.abs(neo - lin).max() > 1e-3 * np.abs(lin).max()


needs_ref = pytest.mark.skipif(not bridge.available("libmpmref_parity.so"),
                               reason="reference build oracle/_ref/libmpmref_parity.so not present")


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_restated_matches_reference_seeded(seed):
    """Random small ensemble instances: restatement == reference every step."""
    case = inputs.block_drop_ensemble(count=1, seed=100 + seed, n_range=(8, 14), steps=12,
                                      side_range=(0.3, 0.5))[0]
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(case.steps):
        ref.step(1)
        job.step(1)
        for f in POINT_FIELDS:
            assert bits_equal(job.points(0, f), ref.points(0, f)), f"seed {seed} step {s} point {f}"
        for f in NODE_FIELDS:
            assert bits_equal(job.nodes(0, f), ref.nodes(0, f)), f"seed {seed} step {s} node {f}"


@needs_ref
def test_restated_matches_reference_wall_exit():
    """A block thrown out of a domain without a boundary: corners cross the
    wall (point-sampled fallback rows), then points leave and are deactivated."""
    case = inputs.block_drop_2d()
    for body in case.bodies:
        body.x_t[:, 0] = 60.0
        body.boundary = False
    case.dt = 5e-4
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(25):
        ref.step(1)
        job.step(1)
        for f in POINT_FIELDS:
            assert bits_equal(job.points(0, f), ref.points(0, f)), f"step {s} point {f}"
    assert ref.points(0, "active").sum() < case.bodies[0].n


@needs_ref
@pytest.mark.parametrize("dim,boundary", [(2, "CartesianSmoothBox"), (2, "CartesianFrictionalBox"),
                                          (3, "CartesianSmoothBox"), (3, "CartesianFrictionalBox")])
def test_restated_matches_reference_boundaries(dim, boundary):
    """A block sliding along the floor with the smooth (slip) and the
    frictional box: restatement == reference every step."""
    case = inputs.sliding_block(dim, boundary, mu=0.3, n_cells=8 if dim == 3 else 16, steps=15)
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(case.steps):
        ref.step(1)
        job.step(1)
        for f in POINT_FIELDS:
            assert bits_equal(job.points(0, f), ref.points(0, f)), f"{boundary} step {s} point {f}"
        for f in NODE_FIELDS:
            assert bits_equal(job.nodes(0, f), ref.nodes(0, f)), f"{boundary} step {s} node {f}"


@needs_ref
@pytest.mark.parametrize("dim", [2, 3])
def test_restated_matches_reference_reflected_contact(dim):
    """Two blocks colliding on the floor with ContactHuang_ReflectedBoundary:
    restatement == reference every step (points and contact forces)."""
    case = inputs.wall_collision(dim, n_cells=16 if dim == 2 else 8, steps=15)
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(case.steps):
        ref.step(1)
        job.step(1)
        for b in range(2):
            for f in POINT_FIELDS:
                assert bits_equal(job.points(b, f), ref.points(b, f)), f"step {s} body {b} point {f}"
        assert bits_equal(job.contact(0, "force"), ref.contact(0, "force")), f"step {s} contact force"


def _neohookean(case):
    for body in case.bodies:
        body.material_class = "CompressibleNeohookeanElasticity"
    case.name += "_neohookean"
    return case


@needs_ref
@pytest.mark.parametrize("make", [lambda: _neohookean(inputs.block_drop_2d()),
                                  lambda: _neohookean(inputs.two_body_collision_3d(8, steps=12, gap=0.02))],
                         ids=["block_drop_2d", "collision_3d"])
def test_restated_matches_reference_neohookean(make):
    """CompressibleNeohookeanElasticity (deformation gradient, neo-Hookean
    stress): restatement == reference every step."""
    case = make()
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(12):
        ref.step(1)
        job.step(1)
        for b in range(len(case.bodies)):
            for f in POINT_FIELDS:
                assert bits_equal(job.points(b, f), ref.points(b, f)), f"step {s} body {b} point {f}"


@needs_ref
@pytest.mark.parametrize("make,steps", [(lambda: inputs.sand_column(2, steps=300), 300),
                                        (lambda: inputs.sand_column(2, steps=40, density_pressure=True, mu_2=0.8), 40),
                                        (lambda: inputs.sand_column(3, n_cells=12, steps=40), 40)],
                         ids=["column_2d", "column_2d_mu2_density", "column_3d"])
def test_restated_matches_reference_sand(make, steps):
    """Sand_SachithLocal (trial stress, local mu(I) return, zero stress below
    the critical density or in tension, gammap): restatement == reference
    every step. The density-pressure column dilates through the critical
    density (its stress switches off) within these steps."""
    case = make()
    d = tempfile.mkdtemp()
    ref = bridge.ReferenceJob(inputs.write_case(case, d))
    job = bridge.RestatedJob(case)
    for s in range(steps):
        ref.step(1)
        job.step(1)
        for f in POINT_FIELDS + ["gammap", "gammap_dot"]:
            assert bits_equal(job.points(0, f), ref.points(0, f)), f"step {s} point {f}"
        for f in NODE_FIELDS:
            assert bits_equal(job.nodes(0, f), ref.nodes(0, f)), f"step {s} node {f}"


def _cpdi_off(case):
    case.cpdi = 0
    case.name += "_cpdi_off"
    return case


@needs_ref
@pytest.mark.parametrize("make", [inputs.block_drop_2d, lambda: _cpdi_off(inputs.block_drop_2d()),
                                  lambda: inputs.two_body_collision_3d(8, steps=12, gap=0.02)],
                         ids=["block_drop_2d", "block_drop_2d_cpdi_off", "collision_3d"])
def test_point_element_history_changes_nothing(make):
    """DefaultPoints with use_elem (point-int-props {1}, default_points.cpp:86-95)
    passes an element hint to the grid, which CartesianLinear ignores (the
    Grid defaults fall back to the plain lookups, mpm_objects.hpp:263-274):
    the reference with the option on equals the restatement bit for bit."""
    case = make()
    ref = bridge.ReferenceJob(inputs.write_case(case, tempfile.mkdtemp(), point_int_props=(1,)))
    job = bridge.RestatedJob(case)
    for s in range(12):
        ref.step(1)
        job.step(1)
        for b in range(len(case.bodies)):
            for f in POINT_FIELDS:
                assert bits_equal(job.points(b, f), ref.points(b, f)), f"step {s} body {b} point {f}"
