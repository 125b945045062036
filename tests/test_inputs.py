"""Seeded input generator: sizes, masses, volumes and exact .points round trip."""
import os
import tempfile

import numpy as np
import pytest

from mpm_3d_b200 import inputs


def test_block_drop_2d_layout():
    c = inputs.block_drop_2d()
    b = c.bodies[0]
    assert b.n == 144 and c.N == (20, 20) and c.steps == 2000 and c.dt == 1e-4
    assert np.allclose(b.m, 0.625) and np.allclose(b.v, 6.25e-4)
    assert np.isclose(b.x[:, 0].min(), 0.3625) and np.isclose(b.x[:, 0].max(), 0.6375)
    assert np.isclose(b.x[:, 1].min(), 0.4625) and np.isclose(b.x[:, 1].max(), 0.7375)
    assert np.all(b.x_t[:, 1] == -1.0) and np.all(b.x_t[:, 0] == 0.0)


def test_two_body_collision_sizes():
    c = inputs.two_body_collision_3d(128)
    assert [b.n for b in c.bodies] == [262144, 262144]
    assert c.contacts[0].mu == 0.4 and c.dt == 2e-5
    h = 1.0 / 128
    assert np.allclose(c.bodies[0].m, 1000.0 * (h / 2) ** 3)
    assert np.allclose(c.bodies[0].x.mean(0), [0.3, 0.5, 0.5])
    assert np.allclose(c.bodies[1].x.mean(0), [0.7, 0.5, 0.5])


def test_column_collapse_counts():
    c = inputs.column_collapse_3d(scale=4)
    assert c.N == (64, 64, 32)
    assert c.bodies[0].n == 32 * 32 * 48
    full = 128 * 128 * 192
    assert full == 3145728
    # jitter within +-1% of h
    h = 2.0 / 64
    x = c.bodies[0].x
    assert x[:, 2].min() > 0 and x[:, 0].min() > 0.75 - 0.01 * h


def test_seeded_determinism():
    a = inputs.block_drop_ensemble(count=3, seed=7)
    b = inputs.block_drop_ensemble(count=3, seed=7)
    for ca, cb in zip(a, b):
        assert ca.N == cb.N and ca.dt == cb.dt
        assert np.array_equal(ca.bodies[0].x, cb.bodies[0].x)


def test_points_file_round_trip_is_exact():
    c = inputs.column_collapse_3d(scale=16)
    d = tempfile.mkdtemp()
    cfg = inputs.write_case(c, d)
    assert os.path.exists(cfg)
    pfile = [f for f in os.listdir(d) if f.endswith(".points")][0]
    m, v, x, xt, act = inputs.read_points_file(os.path.join(d, pfile), 3)
    b = c.bodies[0]
    assert np.array_equal(m, b.m) and np.array_equal(v, b.v)
    assert np.array_equal(x, b.x) and np.array_equal(xt, b.x_t) and np.array_equal(act, b.active)


def test_adjacent_classes_in_written_configs():
    """The boundary, contact and material classes beyond the path's defaults
    reach the .cfg the reference reads, with their properties."""
    slide = inputs.sliding_block(2, "CartesianFrictionalBox", mu=0.25, n_cells=16, steps=5)
    assert inputs.boundary_kind(slide.bodies[0]) == 3
    assert slide.bodies[0].x[:, 1].min() > 0.0 and slide.bodies[0].x[:, 0].min() > 0.0
    coll = inputs.wall_collision(3, n_cells=8, steps=5)
    assert coll.contacts[0].reflected and [inputs.boundary_kind(b) for b in coll.bodies] == [2, 2]
    coll.bodies[0].material_class = "CompressibleNeohookeanElasticity"
    assert inputs.material_kind(coll.bodies[0]) == 1 and inputs.material_kind(coll.bodies[1]) == 0
    d = tempfile.mkdtemp()
    text = open(inputs.write_case(slide, d)).read()
    assert 'boundary-class = "CartesianFrictionalBox"' in text and "boundary-props = {0.25" in text
    text = open(inputs.write_case(coll, d)).read()
    assert 'class = "ContactHuang_ReflectedBoundary"' in text
    assert 'boundary-class = "CartesianSmoothBox"' in text
    assert 'material-class = "CompressibleNeohookeanElasticity"' in text
    assert 'material-class = "IsotropicLinearElasticity"' in text
    plain = inputs.block_drop_2d()
    assert inputs.boundary_kind(plain.bodies[0]) == 1
    plain.bodies[0].boundary = False
    assert inputs.boundary_kind(plain.bodies[0]) == 0
    assert "boundary-class" not in open(inputs.write_case(plain, d)).read()


def test_sand_properties_resolve_as_the_reference_init():
    """Sand_SachithLocal::init (sand_sachithlocal.cpp:57-103): with six
    material-props mu_2 = mu_s and I_0 = 1; with eight they are given."""
    six = inputs.sand_column(2, steps=1)
    props, density = inputs.sand_params(six.bodies[0])
    assert props == (0.01, 0.577, 1650.0, 1000.0, 0.577, 1.0) and not density
    eight = inputs.sand_column(2, steps=1, density_pressure=True, mu_2=0.8)
    props, density = inputs.sand_params(eight.bodies[0])
    assert props == (0.01, 0.577, 1650.0, 1000.0, 0.8, 0.278) and density
    assert inputs.material_kind(eight.bodies[0]) == 2
    bad = inputs.sand_column(2, steps=1)
    bad.bodies[0].material_props = (0.01, 0.577)
    with pytest.raises(ValueError):
        inputs.sand_params(bad.bodies[0])


def test_written_config_carries_material_point_and_serializer_settings(tmp_path):
    case = inputs.sand_column(2, steps=1, density_pressure=True, mu_2=0.8)
    text = open(inputs.write_case(case, str(tmp_path), point_int_props=(1,), serializer_class="AsyncVTK",
                                  frame_dir="frames", sample_rate=250.0)).read()
    assert 'material-class = "Sand_SachithLocal"' in text
    assert "material-props = {10000000.0,0.3,0.01,0.577,1650.0,1000.0,0.8,0.278}" in text
    assert 'material-str-props = {"USE_DENSITY_FOR_PRESSURE"}' in text
    assert "point-int-props = {1}" in text
    assert 'class = "AsyncVTK"' in text and "properties = {250.0}" in text
    assert 'str-properties = {"frames","save","case"}' in text
