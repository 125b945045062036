"""Parity of the CUDA path (through the C ABI) with the oracle, step by step.

The oracle is the C restatement in oracle/mpm_oracle.c, which is bit-exact
with the reference's own sources (tests/test_oracle.py pins it). Tolerance:
max |gpu - oracle| / max(max |oracle|, physical floor) <= 1e-10 per field
after every step (util.field_floor); the S / gradS connectivity of
mpmgpu_dump_map must be bit-identical for identical positions.
"""
import copy

import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL
from util import FP64_TOL, assert_close, bits_equal, field_floor

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


def _spinning_block_2d():
    """Block drop with a rigid spin, so stress and velocity gradient are
    physical from the first step (free fall alone leaves them at round-off)."""
    c = inputs.block_drop_2d()
    b = c.bodies[0]
    cx = b.x[:, :2].mean(0)
    b.x_t[:, 0] = -(b.x[:, 1] - cx[1]) * 20.0
    b.x_t[:, 1] = (b.x[:, 0] - cx[0]) * 20.0 - 1.0
    c.name = "spinning_block_2d"
    return c


def _dense_cells_3d():
    """A regular block plus two crowded cells of an 8^3 grid: 600 points of
    one window class in one cell (more than the 255 a class count of the
    binning's per-cell histogram holds, so that cell keeps arrival order; its
    bin also exceeds one work item) and 400 points spread over all classes
    in another."""
    rng = np.random.default_rng(11)
    h = 1.0 / 8
    block = inputs.block_points((2 * h, 2 * h, 2 * h), (6, 6, 6), (h, h, h), 1000.0, (0.3, -0.2, 0.1),
                                name="block", E=1e5, nu=0.3)
    vol = h ** 3 / 8
    one_class = np.array([5, 5, 5]) * h + rng.uniform(0.2, 0.8, size=(600, 3)) * h
    all_classes = np.array([5, 2, 5]) * h + rng.uniform(0.01, 0.99, size=(400, 3)) * h
    x = np.vstack([block.x, one_class, all_classes])
    n = x.shape[0]
    x_t = np.vstack([block.x_t, rng.uniform(-0.2, 0.2, size=(1000, 3))])
    body = inputs.Body(name="dense", m=np.full(n, 1000 * vol), v=np.full(n, vol), x=x, x_t=x_t,
                       active=np.ones(n, np.int32), E=1e5, nu=0.3)
    return inputs.Case(name="dense_cells_3d", dim=3, L=(1.0, 1.0, 1.0), N=(8, 8, 8), dt=1e-4, steps=10,
                       bodies=[body])


def _neohookean(case):
    for body in case.bodies:
        body.material_class = "CompressibleNeohookeanElasticity"
    case.name += "_neohookean"
    return case


CASES = {
    "dense_cells_3d": (_dense_cells_3d, 10),
    "spinning_block_2d_neohookean": (lambda: _neohookean(_spinning_block_2d()), 60),
    "collision_3d_neohookean": (lambda: _neohookean(inputs.two_body_collision_3d(16, steps=15, gap=0.01)), 15),
    "sliding_3d_neohookean": (lambda: _neohookean(inputs.sliding_block(3, "CartesianSmoothBox", n_cells=12,
                                                                       steps=30)), 30),
    "sliding_2d_smooth_box": (lambda: inputs.sliding_block(2, "CartesianSmoothBox", n_cells=16, steps=60), 60),
    "sliding_2d_frictional_box": (lambda: inputs.sliding_block(2, "CartesianFrictionalBox", mu=0.3, n_cells=16,
                                                               steps=60), 60),
    "sliding_3d_smooth_box": (lambda: inputs.sliding_block(3, "CartesianSmoothBox", n_cells=12, steps=30), 30),
    "wall_collision_2d_reflected": (lambda: inputs.wall_collision(2, n_cells=16, steps=40), 40),
    "wall_collision_3d_reflected": (lambda: inputs.wall_collision(3, n_cells=12, steps=20), 20),
    "sliding_3d_frictional_box": (lambda: inputs.sliding_block(3, "CartesianFrictionalBox", mu=0.3, n_cells=12,
                                                               steps=30), 30),
    "wall_exit_2d": (_wall_exit_2d, 25),
    "block_drop_2d": (inputs.block_drop_2d, 120),
    "spinning_block_2d": (_spinning_block_2d, 120),
    "block_drop_2d_cpdi_off": (_cpdi_off_2d, 40),
    "collision_2d": (lambda: inputs.two_body_collision_2d(20, steps=60), 60),
    "collision_3d_touching": (lambda: inputs.two_body_collision_3d(16, steps=15, gap=0.01), 15),
    "collision_3d_explicit": (_explicit_contact_3d, 8),
    "column_collapse_s16": (lambda: inputs.column_collapse_3d(scale=16, steps=15), 15),
    "collision_3d_zero_gravity": (lambda: inputs.two_body_collision_3d(16, steps=8, gap=0.01, gravity=(0.0, 0.0, 0.0)),
                                  8),
    # Sand_SachithLocal: elastic, plastic-return and zero-stress points from
    # the first tens of steps; with the pressure from the density the column
    # dilates below the critical density from the 8th step on, where the
    # stress switches off discontinuously, so that case stops before it
    "sand_column_2d": (lambda: inputs.sand_column(2, steps=80), 80),
    "sand_column_3d": (lambda: inputs.sand_column(3, n_cells=12, steps=30), 30),
    "sand_column_2d_mu2_density": (lambda: inputs.sand_column(2, steps=6, density_pressure=True, mu_2=0.8), 6),
}


def _point_fields(body):
    extra = ["gammap", "gammap_dot"] if body.material and body.material_class == "Sand_SachithLocal" else []
    return POINT_FIELDS + extra


@pytest.fixture(scope="module", autouse=True)
def restated_lib():
    bridge.build_restated()


def _step_parity(name, sort_interval=0, mode="fp64", kernel=None, autotune=False):
    make, steps = CASES[name]
    case = make()
    ref = bridge.RestatedJob(case)
    gpu = GPUExplicitUSL(case, keep_debug=True, sort_interval=sort_interval, mode=mode, kernel=kernel)
    if autotune:
        # the trials run from snapshots: the state after tuning is the state before it
        form, cap = gpu.autotune(steps=2)
        assert gpu.kernel() == (form, cap)
    worst = {}
    for s in range(steps):
        ref.step(1)
        gpu.step(1)
        for b in range(len(case.bodies)):
            for f in _point_fields(case.bodies[b]):
                e = assert_close(gpu.points(b, f), ref.points(b, f), FP64_TOL, f"{name} step {s} body {b} point {f}",
                                 field_floor(case, f))
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
def test_step_parity(name):
    _step_parity(name)


CASES_3D = sorted(n for n in CASES if "3d" in n)
KERNEL_FORMS = [("staged", 512), ("staged", 256), ("point_per_thread", 128), ("point_per_thread", 256)]


@pytest.mark.parametrize("kernel", KERNEL_FORMS, ids=lambda k: f"{k[0]}{k[1]}")
@pytest.mark.parametrize("name", CASES_3D)
def test_step_parity_kernel_forms(name, kernel):
    """3D jobs run on the one-point-per-thread kernel with 512 points per
    item by default (test_step_parity); every other kernel form and size
    must meet the same parity."""
    _step_parity(name, kernel=kernel)


@pytest.mark.parametrize("name", ["collision_3d_touching", "spinning_block_2d"])
def test_step_parity_after_autotune(name):
    """mpmgpu_autotune on a single handle: whatever it keeps, the steps after
    it meet the parity from the unchanged initial state."""
    _step_parity(name, autotune=True)


@pytest.mark.parametrize("name", ["collision_3d_touching", "wall_exit_2d", "spinning_block_2d", "dense_cells_3d"])
def test_step_parity_frequent_rebinning(name):
    """Re-binning every 2 steps permutes the point storage; results must not
    change (downloads come back in the original point order)."""
    _step_parity(name, sort_interval=2)


def _assert_same_map(gpu, ref, b, what):
    node, pt, val, grad = gpu.map(b)
    rn, rp, rv = ref.map(b)
    gn, gp, gg = ref.grad_map(b)
    assert np.array_equal(node, rn) and np.array_equal(pt, rp), f"{what}: S connectivity differs"
    assert bits_equal(val, rv), f"{what}: S values differ"
    assert np.array_equal(node, gn) and np.array_equal(pt, gp), f"{what}: gradS connectivity differs"
    assert bits_equal(grad, gg), f"{what}: gradS values differ"
    return len(node)


def _with_positions(case, gpu):
    """A copy of the case whose points sit where the GPU has moved them
    (volumes stay the initial ones: extent is never updated)."""
    moved = copy.deepcopy(case)
    for b, body in enumerate(moved.bodies):
        body.x = gpu.points(b, "x").copy()
        body.active = gpu.points(b, "active")[:, 0].astype(np.int32)
    return moved


@pytest.mark.parametrize("name", sorted(CASES))
def test_map_bit_exact(name):
    make, steps = CASES[name]
    case = make()
    gpu = GPUExplicitUSL(case, keep_debug=True)
    ref = bridge.RestatedJob(case)
    ref.build_map()
    for b in range(len(case.bodies)):
        _assert_same_map(gpu, ref, b, f"{name} initial")
    gpu.step(min(steps, 5))
    moved = _with_positions(case, gpu)
    ref2 = bridge.RestatedJob(moved)
    ref2.build_map()
    for b in range(len(case.bodies)):
        _assert_same_map(gpu, ref2, b, f"{name} after steps")


def _edge_case_2d(cpdi):
    """Points on special positions of a 20x20 grid on 1x1 m: exactly on a
    node (0/0 gradient of the point-sampled map), a hi corner exactly on the
    upper wall (no element for that corner), a point exactly on the wall
    (no element at all), a point outside (deactivated) and a near-wall point
    whose corners leave the domain (point-sampled fallback)."""
    h = 0.05
    vol = (h / 2) ** 2
    a = 0.5 * (0.5 * np.sqrt(vol))
    x_corner_at_wall = 1.0 - a
    while x_corner_at_wall + a < 1.0:
        x_corner_at_wall = np.nextafter(x_corner_at_wall, 2.0)
    while x_corner_at_wall + a > 1.0:
        x_corner_at_wall = np.nextafter(x_corner_at_wall, 0.0)
    pts = [
        (0.25, 0.25),                 # on a node
        (x_corner_at_wall, 0.4),      # hi corner exactly at x = L
        (1.0, 0.6),                   # on the wall
        (1.2, 0.3),                   # outside
        (0.003, 0.7),                 # corners cross x = 0
        (0.5 + 1e-17, 0.5),           # at a node within rounding
        (0.3125, 0.4375),             # regular interior point
    ]
    x = np.zeros((len(pts), 3))
    x[:, :2] = np.array(pts)
    n = len(pts)
    body = inputs.Body(name="edge", m=np.full(n, 1000 * vol), v=np.full(n, vol), x=x, x_t=np.zeros((n, 3)),
                       active=np.ones(n, np.int32), E=1e5, nu=0.3)
    return inputs.Case(name=f"edge_2d_cpdi{cpdi}", dim=2, L=(1.0, 1.0), N=(20, 20), dt=1e-4, steps=1,
                       bodies=[body], cpdi=cpdi)


@pytest.mark.parametrize("cpdi", [0, 1])
def test_map_edge_positions(cpdi):
    case = _edge_case_2d(cpdi)
    gpu = GPUExplicitUSL(case, keep_debug=True)
    ref = bridge.RestatedJob(case)
    ref.build_map()
    count = _assert_same_map(gpu, ref, 0, f"edge cpdi={cpdi}")
    assert count > 0
    assert np.array_equal(gpu.points(0, "active"), ref.points(0, "active"))
    assert ref.points(0, "active")[3, 0] == 0
