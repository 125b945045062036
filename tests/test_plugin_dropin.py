"""Drop-in check of the GPUExplicitUSL Solver plugin.

The reference's own Configurator, Job, DefaultBody/DefaultPoints/DefaultNodes,
material, boundary and contact objects (compiled from its sources by
oracle/Makefile) run the same .cfg twice: once with
`solver { class = "ExplicitUSL" }` and once with `class = "GPUExplicitUSL"`
(mpm_3d_b200/plugin, registered next to it as a maintainer would). The GPU
run's host arrays, written back by the plugin, must match the reference
solver within the FP64 parity tolerance.
"""
import tempfile

import pytest

import bridge
from mpm_3d_b200 import inputs
from util import FP64_TOL, assert_close, field_floor

needs_gpu_harness = pytest.mark.skipif(not bridge.available("libmpmref_gpu.so"),
                                       reason="oracle/_ref/libmpmref_gpu.so not built (needs the reference tree)")


@needs_gpu_harness
def test_plugin_configures_from_a_reference_config():
    """Config parsing and Job::init with the plugin need no GPU: device set-up
    is deferred to the first step."""
    case = inputs.block_drop_2d()
    cfg = inputs.write_case(case, tempfile.mkdtemp(), solver_class="GPUExplicitUSL")
    job = bridge.ReferenceJob(cfg, build="gpu")
    assert job.nbodies == 1 and job.n_points(0) == 144
    cfg = inputs.write_case(case, tempfile.mkdtemp(), solver_class="GPUExplicitUSL", point_int_props=(1,))
    assert bridge.ReferenceJob(cfg, build="gpu").n_points(0) == 144
    sand = inputs.sand_column(2, steps=5, density_pressure=True, mu_2=0.8)
    job = bridge.ReferenceJob(inputs.write_case(sand, tempfile.mkdtemp(), solver_class="GPUExplicitUSL"), build="gpu")
    assert job.points(0, "gammap").shape == (sand.bodies[0].n, 1)


def _neohookean(case):
    for body in case.bodies:
        body.material_class = "CompressibleNeohookeanElasticity"
    case.name += "_neohookean"
    return case


CASES = {
    "block_drop_2d": (inputs.block_drop_2d, 30),
    "collision_2d": (lambda: inputs.two_body_collision_2d(20, steps=20), 20),
    "collision_3d_touching": (lambda: inputs.two_body_collision_3d(16, steps=8, gap=0.01), 8),
    "sliding_2d_frictional_box": (lambda: inputs.sliding_block(2, "CartesianFrictionalBox", mu=0.3, n_cells=16,
                                                               steps=20), 20),
    "sliding_3d_smooth_box": (lambda: inputs.sliding_block(3, "CartesianSmoothBox", n_cells=12, steps=10), 10),
    "wall_collision_2d_reflected": (lambda: inputs.wall_collision(2, n_cells=16, steps=20), 20),
    "collision_3d_neohookean": (lambda: _neohookean(inputs.two_body_collision_3d(16, steps=8, gap=0.01)), 8),
    "sand_column_2d": (lambda: inputs.sand_column(2, steps=30), 30),
}


def _material_fields(body):
    # Sand_SachithLocal's frame fields, which the plugin writes back into the material
    return ("gammap", "gammap_dot") if body.material_class == "Sand_SachithLocal" else ()


@needs_gpu_harness
@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_matches_reference_solver(name):
    make, steps = CASES[name]
    case = make()
    ref = bridge.ReferenceJob(inputs.write_case(case, tempfile.mkdtemp()), build="parity")
    gpu = bridge.ReferenceJob(inputs.write_case(case, tempfile.mkdtemp(), solver_class="GPUExplicitUSL"), build="gpu")
    for s in range(steps):
        ref.step(1)
        gpu.step(1)
        for b in range(len(case.bodies)):
            for f in ("x", "u", "x_t", "mx_t", "T", "L", "v", "active", "b") + _material_fields(case.bodies[b]):
                assert_close(gpu.points(b, f), ref.points(b, f), FP64_TOL, f"{name} step {s} point {f}",
                             field_floor(case, f))
            for f in ("m", "mx_t", "f", "x_t", "u", "diff_x_t"):
                assert_close(gpu.nodes(b, f), ref.nodes(b, f), FP64_TOL, f"{name} step {s} node {f}")
        for c in range(len(case.contacts)):
            assert_close(gpu.contact(c, "force"), ref.contact(c, "force"), FP64_TOL, f"{name} step {s} contact")


@needs_gpu_harness
@pytest.mark.gpu
@pytest.mark.parametrize("form,tol", [(1, FP64_TOL), (2, 1e-4)])
def test_dropin_forms_from_the_config(form, tol):
    """The form is the fourth solver int-property: 1 deterministic FP64
    (same tolerance as FP64), 2 mixed FP32/FP64 (1e-4)."""
    case = inputs.two_body_collision_3d(16, steps=8, gap=0.01)
    ref = bridge.ReferenceJob(inputs.write_case(case, tempfile.mkdtemp()), build="parity")
    gpu = bridge.ReferenceJob(inputs.write_case(case, tempfile.mkdtemp(), solver_class="GPUExplicitUSL",
                                                solver_extra=(0, form)), build="gpu")
    ref.step(8)
    gpu.step(8)
    for b in range(len(case.bodies)):
        for f in ("x", "u", "x_t", "T", "v"):
            assert_close(gpu.points(b, f), ref.points(b, f), tol, f"form {form} point {f}", field_floor(case, f))
