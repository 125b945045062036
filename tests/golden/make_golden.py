"""Generates the golden fixtures in this directory from the reference itself.

Runs the reference solver's own hot-path sources, compiled unmodified by
oracle/Makefile (oracle/_ref/libmpmref_parity.so, -ffp-contract=off), on small
seeded cases and stores particle, node and contact fields after selected
steps plus the S / gradS triplets of the first map build. The reference tree
has no golden vectors of its own for this path, so these outputs are the pin
for the C restatement (oracle/mpm_oracle.c) and, through it, for the GPU path.

    make -C oracle REF=/path/to/mpm_3d && python tests/golden/make_golden.py [name ...]

With names, only those fixtures are (re)written.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import bridge  # noqa: E402
from mpm_3d_b200 import inputs  # noqa: E402

POINT_FIELDS = ["x", "u", "x_t", "mx_t", "T", "L", "v", "active"]
NODE_FIELDS = ["m", "mx_t", "f", "x_t", "u", "diff_x_t"]


def golden_cases():
    """name -> (case, snapshot steps)."""
    cpdi_off = inputs.block_drop_2d()
    cpdi_off.cpdi = 0
    cpdi_off.name = "block_drop_2d_cpdi_off"
    explicit = inputs.two_body_collision_3d(16, steps=6, gap=0.01)
    explicit.contact_spec = 0
    explicit.name += "_explicit"
    neohookean = inputs.two_body_collision_2d(20, steps=40)
    for body in neohookean.bodies:
        body.material_class = "CompressibleNeohookeanElasticity"
    neohookean.name += "_neohookean"
    return {
        "block_drop_2d": (inputs.block_drop_2d(), [1, 10, 100]),
        "block_drop_2d_cpdi_off": (cpdi_off, [1, 20]),
        "collision_2d": (inputs.two_body_collision_2d(20, steps=40), [1, 40]),
        "collision_3d_touching": (inputs.two_body_collision_3d(16, steps=6, gap=0.01), [1, 6]),
        "collision_3d_explicit": (explicit, [6]),
        "column_collapse_s16": (inputs.column_collapse_3d(scale=16, steps=10), [10]),
        # the classes beside the path's defaults: boundaries, reflected contact, material
        "sliding_2d_frictional": (inputs.sliding_block(2, "CartesianFrictionalBox", mu=0.3, n_cells=16, steps=15),
                                  [1, 15]),
        "sliding_3d_smooth": (inputs.sliding_block(3, "CartesianSmoothBox", mu=0.3, n_cells=8, steps=15), [15]),
        "wall_collision_2d_reflected": (inputs.wall_collision(2, n_cells=16, steps=15), [1, 15]),
        "collision_2d_neohookean": (neohookean, [1, 40]),
        "sand_column_2d": (inputs.sand_column(2, steps=60), [1, 20, 60]),
        "sand_column_2d_mu2_density": (inputs.sand_column(2, steps=12, density_pressure=True, mu_2=0.8), [12]),
    }


def point_fields(body) -> list:
    """The point fields a body's fixtures hold: the material's frame fields
    beside the points' own."""
    if body.material and body.material_class == "Sand_SachithLocal":
        return POINT_FIELDS + ["gammap", "gammap_dot"]
    return POINT_FIELDS


def run(name, case, snaps):
    d = tempfile.mkdtemp()
    cfg = inputs.write_case(case, d)
    ref = bridge.ReferenceJob(cfg, build="parity")
    out = {}
    ref.build_map()
    for b in range(len(case.bodies)):
        node, pt, val = ref.map(b)
        gnode, gpt, grad = ref.grad_map(b)
        assert np.array_equal(node, gnode) and np.array_equal(pt, gpt)
        out[f"map_b{b}_node"] = node
        out[f"map_b{b}_point"] = pt
        out[f"map_b{b}_S"] = val
        out[f"map_b{b}_grad"] = grad
    done = 0
    for s in snaps:
        ref.step(s - done)
        done = s
        for b in range(len(case.bodies)):
            for f in point_fields(case.bodies[b]):
                out[f"s{s}_b{b}_p_{f}"] = ref.points(b, f)
            for f in NODE_FIELDS:
                out[f"s{s}_b{b}_n_{f}"] = ref.nodes(b, f)
        for c in range(len(case.contacts)):
            for f in ("normal", "force"):
                out[f"s{s}_c{c}_{f}"] = ref.contact(c, f)
    out["snaps"] = np.array(snaps)
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path))


if __name__ == "__main__":
    wanted = set(sys.argv[1:])
    for name, (case, snaps) in golden_cases().items():
        if not wanted or name in wanted:
            run(name, case, snaps)
