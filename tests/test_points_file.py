"""The library's parallel .points reader (mpmgpu_points_file_read, host
only) against the reference's DefaultPoints::readFromFile: the same values
bit for bit, on the files the generators write and on hand-formatted lines
(CRLF endings, a trailing space, exponents, a fractional active flag), and
errors with the line number where the reference would stop reading."""
import os
import tempfile

import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import MpmGpuError, read_points_file
from util import bits_equal

needs_ref = pytest.mark.skipif(not bridge.available("libmpmref_parity.so"),
                               reason="reference build oracle/_ref/libmpmref_parity.so not present")

CASES = {
    "block_drop_2d": inputs.block_drop_2d,
    "column_collapse_s8": lambda: inputs.column_collapse_3d(scale=8, steps=1),
    "collision_3d": lambda: inputs.two_body_collision_3d(16, steps=1, gap=0.01),
}


def _write(case):
    d = tempfile.mkdtemp()
    cfg = inputs.write_case(case, d)
    files = [os.path.join(d, f"{case.name}_{bi}_{b.name}.points") for bi, b in enumerate(case.bodies)]
    return cfg, files


def _ref_points(cfg, nbodies):
    ref = bridge.ReferenceJob(cfg)
    out = [{f: ref.points(b, f) for f in ("m", "v", "x", "x_t", "active")} for b in range(nbodies)]
    ref.close()
    return out


def _same(got, ref):
    m, v, x, xt, active = got
    assert bits_equal(m, ref["m"][:, 0]) and bits_equal(v, ref["v"][:, 0])
    assert bits_equal(x, ref["x"]) and bits_equal(xt, ref["x_t"])
    assert np.array_equal(active, ref["active"][:, 0].astype(np.int32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_reads_the_generated_files(name):
    case = CASES[name]()
    _, files = _write(case)
    for body, path in zip(case.bodies, files):
        m, v, x, xt, active = read_points_file(path, case.dim, threads=4)
        assert bits_equal(m, body.m) and bits_equal(v, body.v) and bits_equal(x, body.x) and bits_equal(xt, body.x_t)
        assert np.array_equal(active, body.active)
        one = read_points_file(path, case.dim, threads=1)
        assert all(bits_equal(a, b) for a, b in zip(one[:4], (m, v, x, xt)))


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES))
def test_same_values_as_the_reference_reader(name):
    case = CASES[name]()
    cfg, files = _write(case)
    ref = _ref_points(cfg, len(case.bodies))
    for b, path in enumerate(files):
        _same(read_points_file(path, case.dim), ref[b])


@needs_ref
def test_hand_formatted_lines_as_the_reference_reads_them():
    case = inputs.block_drop_2d()
    cfg, files = _write(case)
    body = case.bodies[0]
    lines = [f"{body.n}\r\n"]
    for i in range(body.n):
        vals = [body.m[i], body.v[i], body.x[i, 0], body.x[i, 1], body.x_t[i, 0], body.x_t[i, 1]]
        if i % 4 == 0:
            text = " ".join(f"{v:.17e}" for v in vals) + " 1.0\r\n"     # exponents, CRLF
        elif i % 4 == 1:
            text = " ".join(repr(float(v)) for v in vals) + " 1 \n"      # a trailing space
        elif i % 4 == 2:
            text = " ".join(f"{v:.6g}" for v in vals) + " 0.9\n"         # short values, active truncated to 0
        else:
            text = " ".join(repr(float(v)) for v in vals) + " 1\n"
        lines.append(text)
    with open(files[0], "w", newline="") as f:
        f.writelines(lines)
    ref = _ref_points(cfg, 1)[0]
    got = read_points_file(files[0], 2)
    _same(got, ref)
    assert (got[4] == 0).sum() == body.n // 4 + (1 if body.n % 4 > 2 else 0)


@pytest.mark.parametrize("mutate,line", [
    (lambda ls: ls[:3] + [ls[3].replace(" ", "  ", 1)] + ls[4:], 4),   # an empty piece: one column too many
    (lambda ls: ls[:5] + ["0.1 0.2 abc 0.4 0.5 0.6 1\n"] + ls[6:], 6),  # not a number
    (lambda ls: ls[:-1], 145),                                          # a missing line
    (lambda ls: ls[:7] + ["\n"] + ls[8:], 8),                           # an empty line
])
def test_malformed_lines_are_reported(mutate, line):
    case = inputs.block_drop_2d()
    _, files = _write(case)
    with open(files[0]) as f:
        lines = f.readlines()
    with open(files[0], "w") as f:
        f.writelines(mutate(lines))
    with pytest.raises(MpmGpuError, match=f"line {line} "):
        read_points_file(files[0], 2)


def test_2d_lines_with_three_coordinates_are_malformed_as_in_the_reference():
    """DefaultPoints::readFromFile accepts 1 + 1 + DIM + DIM + 1 or
    1 + 1 + GRID_DIM + GRID_DIM + 1 columns (default_points.cpp:150-176); for
    the job types of this path (TYPE 2 and 3, job.hpp:58-71) DIM equals
    GRID_DIM, so a 2D file takes 7 columns only, and a 9-column line ends the
    reference's reading with an error, as it ends this reader's."""
    case = inputs.block_drop_2d()
    _, files = _write(case)
    with open(files[0]) as f:
        lines = f.readlines()
    parts = lines[3].split()
    lines[3] = " ".join(parts[:4] + ["0"] + parts[4:6] + ["0"] + parts[6:]) + "\n"   # x, y, 0, vx, vy, 0
    with open(files[0], "w") as f:
        f.writelines(lines)
    with pytest.raises(MpmGpuError, match="line 4 "):
        read_points_file(files[0], 2)
