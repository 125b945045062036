"""Frames written through the GPU solver plugin.

The reference's Job runs the same configuration twice: once with its own
ExplicitUSL and its own DefaultVTK serializer (default_vtk.cpp, compiled into
the oracle harness as "ReferenceDefaultVTK"), and once with GPUExplicitUSL
(mpm_3d_b200/plugin), whose write-back queues the frame's copies behind the
step and the driver's next step behind them, and AsyncVTK, which formats the
frames on a writer thread. Both runs must write the same files: the same
names, the same lines of text outside the arrays (titles, headers, array
names, connectivity), and in every array the same numbers up to the
printing of 6 significant digits on top of the FP64 parity tolerance (a
value the two runs differ in by a rounding can print with its last digit
one apart). As in the parity tests, the tolerance of a field that can be
pure round-off (the velocity gradient and stress of a body in free fall) is
taken relative to its physical scale (util.field_floor), and the contact
normal, which at nodes of one body normalises round-off, is compared in
its layout only (the parity tests compare it where both bodies have mass).
"""
import os
import re
import tempfile

import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from util import field_floor

pytestmark = pytest.mark.gpu

needs_gpu_harness = pytest.mark.skipif(not bridge.available("libmpmref_gpu.so"),
                                       reason="oracle/_ref/libmpmref_gpu.so not built (needs the reference tree)")

# lines that open a section (a SCALARS section's LOOKUP_TABLE line belongs to it)
HEADER = re.compile(r"^(SCALARS|VECTORS|TENSORS|POINT_DATA|CELL_DATA|POINTS|CELLS|CELL_TYPES|DATASET|ASCII|#)")


def _frames(case, steps, solver, serializer, every):
    d = tempfile.mkdtemp()
    frames = os.path.join(d, "frames")
    os.makedirs(frames)
    cfg = inputs.write_case(case, d, solver_class=solver, serializer_class=serializer, frame_dir=frames,
                            sample_rate=1.0 / (every * case.dt))
    job = bridge.ReferenceJob(cfg, build="gpu")
    job.step(steps)
    job.close()
    out = {}
    for name in sorted(os.listdir(frames)):
        with open(os.path.join(frames, name)) as f:
            out[name] = f.read().splitlines()
    return out


def _sections(lines):
    """Splits a legacy VTK file into (header line, data lines) sections."""
    secs = []
    cur = None
    for ln in lines:
        if HEADER.match(ln) or cur is None:
            cur = (ln, [])
            secs.append(cur)
        elif ln.startswith("LOOKUP_TABLE"):
            assert not cur[1], "a LOOKUP_TABLE line after data"
        else:
            cur[1].append(ln)
    return secs


# physical scale of the arrays a frame holds, by name (util.field_floor)
FLOOR_FIELD = {"velocity_gradient": "L", "cauchy_stress": "T", "pressure": "T", "velocity": "x_t",
               "diff_velocity": "x_t", "displacement": "u", "gammap": "gammap", "gammap_dot": "gammap_dot"}


def _compare(fname, ref, got, case, tol=1e-10, digits=1e-5):
    rs, gs = _sections(ref), _sections(got)
    assert [h for h, _ in rs] == [h for h, _ in gs], f"{fname}: section headers differ"
    for (h, rd), (_, gd) in zip(rs, gs):
        assert len(rd) == len(gd), f"{fname} {h}: line counts differ"
        if not rd:
            continue
        try:
            a = np.array([float(x) for ln in rd for x in ln.split()])
            b = np.array([float(x) for ln in gd for x in ln.split()])
        except ValueError:
            assert rd == gd, f"{fname} {h}: text differs"
            continue
        assert a.shape == b.shape, f"{fname} {h}: token counts differ"
        parts = h.split()
        name = parts[1] if len(parts) > 1 and parts[0] in ("SCALARS", "VECTORS", "TENSORS") else ""
        if name.startswith("contact_normal"):
            continue
        scale = float(np.abs(a).max()) if a.size else 0.0
        if name in FLOOR_FIELD:
            scale = max(scale, field_floor(case, FLOOR_FIELD[name]))
        bound = tol * scale + digits * np.maximum(np.abs(a), np.abs(b))
        bad = np.abs(a - b) > bound
        assert not bad.any(), (f"{fname} {h}: {int(bad.sum())} values differ, e.g. {a[bad][:3]} vs {b[bad][:3]}")


CASES = {
    "collision_2d": (lambda: inputs.two_body_collision_2d(20, steps=20), 20, 5),
    "collision_3d_touching": (lambda: inputs.two_body_collision_3d(16, steps=12, gap=0.01), 12, 1),
    "sand_column_2d": (lambda: inputs.sand_column(2, steps=20), 20, 5),
}


@needs_gpu_harness
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_solver_with_async_vtk_writes_the_reference_frames(name):
    make, steps, every = CASES[name]
    ref = _frames(make(), steps, "ExplicitUSL", "ReferenceDefaultVTK", every)
    got = _frames(make(), steps, "GPUExplicitUSL", "AsyncVTK", every)
    case = make()
    # (the frame condition compares the accumulated time with frames / rate,
    # so a rounding can skip a frame; both runs apply it the same way)
    assert len(ref) >= 2 * len(case.bodies) * (steps // every - 1)
    assert sorted(got) == sorted(ref)
    for fname in ref:
        _compare(fname, ref[fname], got[fname], case)
