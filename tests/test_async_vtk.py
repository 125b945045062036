"""The AsyncVTK serializer plugin (mpm_3d_b200/plugin/async_vtk.cpp) writes
the same frame files as the reference's own DefaultVTK, byte for byte.

Both serializers run inside the reference's Job (oracle/Makefile compiles
the reference's default_vtk.cpp and registers it as "ReferenceDefaultVTK"
next to "AsyncVTK"), on the reference's ExplicitUSL, with a frame every few
steps. AsyncVTK formats its frames on a writer thread; destroying the job
writes the queued ones.
"""
import os
import tempfile

import pytest

import bridge
from mpm_3d_b200 import inputs

needs_ref = pytest.mark.skipif(not bridge.available("libmpmref_parity.so"),
                               reason="reference build oracle/_ref/libmpmref_parity.so not present")


def _wall_exit_2d():
    """Points leave the domain and turn inactive: the zero rules of the
    writers apply to them."""
    c = inputs.block_drop_2d()
    for body in c.bodies:
        body.x_t[:, 0] = 60.0
        body.boundary = False
    c.dt = 5e-4
    c.name = "wall_exit_2d"
    return c


CASES = {
    "block_drop_2d": (inputs.block_drop_2d, 20),
    "collision_2d": (lambda: inputs.two_body_collision_2d(20, steps=20), 20),
    "collision_3d_touching": (lambda: inputs.two_body_collision_3d(8, steps=10, gap=0.02), 10),
    "sand_column_2d": (lambda: inputs.sand_column(2, steps=20), 20),
    "wall_exit_2d": (_wall_exit_2d, 25),
    # 49,152 points on 139,425 nodes: arrays large enough to be formatted in
    # chunks on several threads
    "column_3d_s4": (lambda: inputs.column_collapse_3d(scale=4, steps=10), 10),
}


def _frames(case, steps, serializer, every=5, int_props=()):
    d = tempfile.mkdtemp()
    frames = os.path.join(d, "frames")
    os.makedirs(frames)
    cfg = inputs.write_case(case, d, serializer_class=serializer, frame_dir=frames,
                            sample_rate=1.0 / (every * case.dt), serializer_int_props=int_props)
    job = bridge.ReferenceJob(cfg)
    job.step(steps)
    job.close()
    out = {}
    for name in sorted(os.listdir(frames)):
        with open(os.path.join(frames, name), "rb") as f:
            out[name] = f.read()
    return out


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_async_vtk_writes_the_reference_frames(name):
    make, steps = CASES[name]
    ref = _frames(make(), steps, "ReferenceDefaultVTK")
    got = _frames(make(), steps, "AsyncVTK")
    case = make()
    # a frame at the first step and then every 5 steps: two files per body
    assert len(ref) == 2 * len(case.bodies) * -(-steps // 5)
    assert sorted(got) == sorted(ref)
    for fname in ref:
        assert got[fname] == ref[fname], f"{name}: {fname} differs"
    sample = ref[sorted(f for f in ref if f.startswith("fpd"))[-1]].decode()
    assert "TENSORS cauchy_stress double" in sample and "SCALARS density double 1" in sample
    if case.contacts:
        nodes = ref[sorted(f for f in ref if f.startswith("fnd"))[-1]].decode()
        assert "VECTORS contact_normal_" in nodes
    if case.bodies[0].material_class == "Sand_SachithLocal":
        assert "SCALARS gammap double 1" in sample


@needs_ref
def test_async_vtk_with_one_pending_frame_and_a_frame_every_step():
    """maxPending = 1: writeFrame waits for the writer at every frame; the
    files are still the reference's."""
    case = inputs.two_body_collision_2d(20, steps=12)
    ref = _frames(inputs.two_body_collision_2d(20, steps=12), 12, "ReferenceDefaultVTK", every=1)
    got = _frames(case, 12, "AsyncVTK", every=1, int_props=(1,))
    assert len(ref) >= 2 * 2 * 11 and sorted(got) == sorted(ref)
    for fname in ref:
        assert got[fname] == ref[fname], fname
