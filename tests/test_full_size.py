"""The forms at the configurations' full sizes, through properties that do
not depend on the size (the oracle runs the small cases step by step in
test_gpu_parity.py; at these sizes it would take minutes per step).

For the 3D column collapse (3,145,728 points on 256x256x128) and the 3D
two-body collision (524,288 points on 128^3, ContactHuang), after 100
steps:
* the deterministic FP64 form gives the same bits whether the points are
  re-binned every step or every 8 steps (a different point order each
  time);
* plain FP64 agrees with deterministic FP64 within the FP64 parity
  tolerance (1e-10 relative, util.py): they differ only in the order of the
  nodal sums;
* after the configuration's full step count (500 and 1000), the mixed form
  (FP32 point state, FP64 nodal sums) agrees with FP64 within 1e-4
  relative;
* the nodal mass of every body sums to the mass of its active points
  (the shape functions of a point sum to one), within 1e-12 relative.
"""
import numpy as np
import pytest

from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL
from util import FP64_TOL, assert_close, bits_equal, field_floor

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4
FIELDS = ["x", "x_t", "T", "v"]

# (case, steps compared between the FP64 forms, steps of the mixed-form
# comparison: the configuration's full step count)
CASES = {
    "column_collapse": (lambda: inputs.column_collapse_3d(scale=1, steps=500), 100, 500),
    "collision_3d": (lambda: inputs.two_body_collision_3d(128, steps=1000), 100, 1000),
}


def _run(case, steps, mode, sort_interval=0, keep_debug=False):
    sim = GPUExplicitUSL(case, mode=mode, sort_interval=sort_interval, keep_debug=keep_debug)
    sim.step(steps)
    out = [{f: sim.points(b, f) for f in FIELDS} for b in range(len(case.bodies))]
    mass = None
    if keep_debug:
        mass = [(float(sim.nodes(b, "m").sum()),
                 float((sim.points(b, "m")[:, 0] * (sim.points(b, "active")[:, 0] != 0)).sum()))
                for b in range(len(case.bodies))]
    sim.close()
    return out, mass


@pytest.mark.parametrize("name", sorted(CASES))
def test_full_size_forms(name):
    make, steps, full_steps = CASES[name]
    case = make()
    det_a, _ = _run(case, steps, "fp64_deterministic", sort_interval=1)
    det_b, _ = _run(case, steps, "fp64_deterministic", sort_interval=8)
    for b in range(len(case.bodies)):
        for f in FIELDS:
            assert bits_equal(det_a[b][f], det_b[b][f]), f"{name}: deterministic {f} of body {b} depends on the binning"
    fp64, mass = _run(case, steps, "fp64", keep_debug=True)
    for b in range(len(case.bodies)):
        for f in FIELDS:
            assert_close(fp64[b][f], det_a[b][f], FP64_TOL, f"{name}: FP64 vs deterministic, body {b} {f}",
                         field_floor(case, f))
    for b, (nodal, points) in enumerate(mass):
        assert points > 0.0
        assert abs(nodal - points) <= 1e-12 * points, f"{name}: body {b} nodal mass {nodal!r} vs points {points!r}"
    fp64_full, _ = _run(case, full_steps, "fp64")
    mixed, _ = _run(case, full_steps, "mixed")
    worst = {}
    for b in range(len(case.bodies)):
        for f in FIELDS:
            e = assert_close(mixed[b][f], fp64_full[b][f], MIXED_TOL, f"{name}: mixed vs FP64, body {b} {f}",
                             field_floor(case, f))
            worst[f] = max(worst.get(f, 0.0), e)
    print(f"{name}: mixed vs FP64 after {full_steps} steps", {f: f"{e:.1e}" for f, e in worst.items()})
