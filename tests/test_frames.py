"""The frame write-back in two halves (mpmgpu_frame_begin, mpmgpu_frame_*).

mpmgpu_frame_begin queues copies of every field behind the steps queued so
far and returns; the frame_* calls give each field as it stood then, in the
layout of the mpmgpu_download_* calls, even while later steps run. Checked
against the one-field downloads taken at the same step of a second run:
within the FP64 parity tolerance in the plain form (the two runs differ
only in the order of the atomics' sums), bit for bit in the deterministic
form.
"""
import numpy as np
import pytest

from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL, MpmGpuError, NODE_FIELDS
from util import FP64_TOL, bits_equal, field_floor, rel_err

pytestmark = pytest.mark.gpu

POINT_FIELDS = ["x", "u", "x_t", "mx_t", "T", "L", "v", "active", "m", "extent"]


@pytest.mark.parametrize("make", [lambda: inputs.two_body_collision_3d(16, steps=10, gap=0.01),
                                  lambda: inputs.sand_column(2, steps=10)], ids=["collision_3d", "sand_2d"])
def test_frame_equals_downloads_at_its_step_while_later_steps_run(make):
    case = make()
    sim = GPUExplicitUSL(case, keep_debug=True)
    sim.step(4)
    sim.frame_begin()                    # the state after 4 steps
    sim.step(3)                          # queued behind the frame's copies
    pts = {(b, f): sim.frame_points(b, f) for b in range(len(case.bodies)) for f in POINT_FIELDS}
    if case.bodies[0].material_class == "Sand_SachithLocal":
        pts.update({(0, f): sim.frame_points(0, f) for f in ("gammap", "gammap_dot")})
    nodes = {(b, f): sim.frame_nodes(b, f) for b in range(len(case.bodies)) for f in NODE_FIELDS}
    cont = {(c, f): sim.frame_contact(c, f) for c in range(len(case.contacts)) for f in ("normal", "force")}
    sim.close()
    # the same case stepped 4 times, read with the one-field downloads
    ref = GPUExplicitUSL(case, keep_debug=True)
    ref.step(4)
    moved = False
    for (b, f), got in pts.items():
        want = ref.points(b, f)
        assert got.shape == want.shape
        # the two runs differ only in the order of the atomics' sums:
        # compare with the FP64 parity tolerance
        assert rel_err(got, want, field_floor(case, f)) <= FP64_TOL, f"point {f} body {b}"
        moved |= f == "x" and not np.array_equal(got, case.bodies[b].x)
    assert moved
    for (b, f), got in nodes.items():
        assert rel_err(got, ref.nodes(b, f)) <= FP64_TOL, f"node {f} body {b}"
    for (c, f), got in cont.items():
        want = ref.contact(c, f)
        if f == "normal":
            # the normal acts only where both bodies have mass; elsewhere it
            # normalises round-off
            m1 = ref.nodes(case.contacts[c].b1, "m")[:, 0]
            m2 = ref.nodes(case.contacts[c].b2, "m")[:, 0]
            both = (m1 > 0) & (m2 > 0)
            assert both.any()
            got, want = got[both], want[both]
        assert rel_err(got, want) <= FP64_TOL, f"contact {f}"
    ref.close()


def test_frame_in_deterministic_form_is_bit_identical_to_downloads():
    case = inputs.two_body_collision_3d(16, steps=6, gap=0.01)
    a = GPUExplicitUSL(case, keep_debug=True, mode="fp64_deterministic")
    a.step(3)
    a.frame_begin()
    a.step(2)
    got = {f: a.frame_points(0, f) for f in ("x", "x_t", "T", "v")}
    gn = a.frame_nodes(1, "mx_t")
    a.close()
    b = GPUExplicitUSL(case, keep_debug=True, mode="fp64_deterministic")
    b.step(3)
    for f, g in got.items():
        assert bits_equal(g, b.points(0, f)), f
    assert bits_equal(gn, b.nodes(1, "mx_t"))
    b.close()


def test_frame_reads_need_a_frame():
    case = inputs.two_body_collision_3d(16, steps=2, gap=0.01)
    sim = GPUExplicitUSL(case, keep_debug=True)
    sim.step(1)
    with pytest.raises(MpmGpuError, match="no frame"):
        sim.frame_points(0, "x")
    sim.close()
