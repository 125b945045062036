"""Parity of the CUDA path (through the C ABI) with the oracle, step by step.

The oracle is the C restatement in oracle/mpm_oracle.c, which is bit-exact
with the reference's own sources (tests/test_oracle.py pins it). Tolerance:
max |gpu - oracle| / max |oracle| <= 1e-10 per field after every step; the
S / gradS connectivity from mpmgpu_dump_map must be bit-identical.
"""
import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL
from util import FP64_TOL, assert_close, bits_equal

pytestmark = pytest.mark.gpu

POINT_FIELDS = ["x", "u", "x_t", "mx_t", "T", "L", "v", "active"]
NODE_FIELDS = ["m", "mx_t", "f", "x_t", "u", "diff_x_t"]


def _cpdi_off_2d():
    c = inputs.block_drop_2d()
    c.cpdi = 0
    c.name = "block_drop_2d_cpdi_off"
    return c


def _explicit_contact_3d():
    c = inputs.two_body_collision_3d(16, steps=10, gap=0.01)
    c.contact_spec = 0
    c.name += "_explicit"
    return c


def _wall_exit_2d():
    c = inputs.block_drop_2d()
    for body in c.bodies:
        body.x_t[:, 0] = 60.0
        body.boundary = False
    c.dt = 5e-4
    c.name = "wall_exit_2d"
    return c


CASES = {
    "wall_exit_2d": (_wall_exit_2d, 25),
    "block_drop_2d": (inputs.block_drop_2d, 120),
    "block_drop_2d_cpdi_off": (_cpdi_off_2d, 40),
    "collision_2d": (lambda: inputs.two_body_collision_2d(20, steps=60), 60),
    "collision_3d_touching": (lambda: inputs.two_body_collision_3d(16, steps=15, gap=0.01), 15),
    "collision_3d_explicit": (_explicit_contact_3d, 8),
    "column_collapse_s16": (lambda: inputs.column_collapse_3d(scale=16, steps=15), 15),
    "collision_3d_zero_gravity": (lambda: inputs.two_body_collision_3d(16, steps=8, gap=0.01, gravity=(0.0, 0.0, 0.0)), 8),
}


def _ensure_oracle():
    bridge.build_restated()


@pytest.mark.parametrize("name", sorted(CASES))
def test_step_parity(name):
    _ensure_oracle()
    make, steps = CASES[name]
    case = make()
    ref = bridge.RestatedJob(case)
    gpu = GPUExplicitUSL(case, keep_debug=True)
    worst = {}
    for s in range(steps):
        ref.step(1)
        gpu.step(1)
        for b in range(len(case.bodies)):
            for f in POINT_FIELDS:
                e = assert_close(gpu.points(b, f), ref.points(b, f), FP64_TOL, f"{name} step {s} body {b} point {f}")
                worst[f] = max(worst.get(f, 0.0), e)
            for f in NODE_FIELDS:
                e = assert_close(gpu.nodes(b, f), ref.nodes(b, f), FP64_TOL, f"{name} step {s} body {b} node {f}")
                worst["n_" + f] = max(worst.get("n_" + f, 0.0), e)
        for c in range(len(case.contacts)):
            assert_close(gpu.contact(c, "force"), ref.contact(c, "force"), FP64_TOL, f"{name} step {s} contact force")
            m1 = ref.nodes(case.contacts[c].b1, "m")[:, 0]
            m2 = ref.nodes(case.contacts[c].b2, "m")[:, 0]
            both = (m1 > 0) & (m2 > 0)
            if both.any():
                assert_close(gpu.contact(c, "normal")[both], ref.contact(c, "normal")[both], FP64_TOL,
                             f"{name} step {s} contact normal")
    print(name, {k: f"{v:.1e}" for k, v in worst.items()})


@pytest.mark.parametrize("name", sorted(CASES))
def test_map_bit_exact(name):
    _ensure_oracle()
    make, steps = CASES[name]
    case = make()
    ref = bridge.RestatedJob(case)
    gpu = GPUExplicitUSL(case, keep_debug=True)
    for s in (0, min(steps, 5)):
        if s:
            ref.step(s)
            gpu.step(s)
        ref.build_map()
        for b in range(len(case.bodies)):
            node, pt, val, grad = gpu.map(b)
            rn, rp, rv = ref.map(b)
            gn, gp, gg = ref.grad_map(b)
            assert np.array_equal(node, rn) and np.array_equal(pt, rp), f"{name}: S connectivity differs"
            assert bits_equal(val, rv), f"{name}: S values differ"
            assert np.array_equal(node, gn) and np.array_equal(pt, gp), f"{name}: gradS connectivity differs"
            assert bits_equal(grad, gg), f"{name}: gradS values differ"
