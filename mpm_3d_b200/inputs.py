"""Seeded synthetic inputs for the explicit MPM step, in mpm_3d's own formats.

A ``Case`` holds everything one ExplicitUSL run needs: the CartesianLinear grid,
the bodies (points with mass, volume, position, velocity, active flag, an
IsotropicLinearElasticity material and an optional CartesianBox, CartesianSmoothBox
or CartesianFrictionalBox boundary),
ContactHuang pairs, the gravity mode and the time step. ``write_case`` writes it
as a mpm_3d ``.cfg`` plus one ``.points`` file per body, the formats the
reference reads (``src/config/config.cpp:176-528``,
``src/objects/points/default_points.cpp:104-193``); doubles are written with
17 significant digits, so ``std::stod`` reads back the exact same values.

Block layouts follow the reference examples (``examples/blockdrop2D/test2D.points``):
2 points per cell per axis at the quarter points of each cell relative to the
block origin, ``m = rho * (h/2)^D`` and ``V = (h/2)^D``.

The named workloads:

* ``block_drop_2d()``: 2D block drop, 20x20 grid on 1x1 m, 144 points,
  E=1e5, nu=0.3, v=(0,-1), dt=1e-4, 2000 steps.
* ``two_body_collision_3d(n_cells=128)``: two 0.25 m cubes colliding at
  +-1 m/s in a 1 m cube, ContactHuang mu=0.4; 128^3 cells gives 262,144 points
  per body; dt=2e-5, 1000 steps.
* ``column_collapse_3d(scale=1)``: 0.5x0.5x0.75 m column on the floor of a
  2x2x1 m domain at 256x256x128 cells (3,145,728 points), rho=1500,
  +-1% h seeded jitter, dt=1e-5, 500 steps. ``scale`` divides the cell
  counts for smaller parity cases.
* ``block_drop_ensemble(count, seed)``: independent 3D block drops with
  seeded grid size, block size/position, velocity and material, dt from each
  instance's CFL limit.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

__all__ = [
    "Body",
    "Contact",
    "Case",
    "block_points",
    "block_drop_2d",
    "two_body_collision_3d",
    "column_collapse_3d",
    "block_drop_ensemble",
    "RequestSpec",
    "serving_stream",
    "serving_case",
    "write_case",
    "read_points_file",
]


@dataclasses.dataclass
class Body:
    """One DefaultBody: point arrays plus material and boundary settings."""

    name: str
    m: np.ndarray  # (n,) mass
    v: np.ndarray  # (n,) volume
    x: np.ndarray  # (n, 3) position (third column 0 in 2D)
    x_t: np.ndarray  # (n, 3) velocity
    active: np.ndarray  # (n,) int32
    E: float = 1e5
    nu: float = 0.3
    material: bool = True
    # "IsotropicLinearElasticity", "CompressibleNeohookeanElasticity" or
    # "Sand_SachithLocal"
    material_class: str = "IsotropicLinearElasticity"
    # material-props after E and nu (Sand_SachithLocal: grain diameter, mu_s,
    # grains_rho, rho_critical[, mu_2, I_0]) and material-str-props
    material_props: Tuple[float, ...] = ()
    material_str_props: Tuple[str, ...] = ()
    # True or "CartesianBox", "CartesianSmoothBox", "CartesianFrictionalBox";
    # False: no boundary
    boundary: Union[bool, str] = True
    boundary_mu: float = 0.0   # CartesianFrictionalBox friction (boundary-props {mu_f})

    @property
    def n(self) -> int:
        return int(self.m.shape[0])


BOUNDARY_CLASSES = ("CartesianBox", "CartesianSmoothBox", "CartesianFrictionalBox")
MATERIAL_CLASSES = ("IsotropicLinearElasticity", "CompressibleNeohookeanElasticity", "Sand_SachithLocal")
SAND_DENSITY_PRESSURE = "USE_DENSITY_FOR_PRESSURE"


def material_kind(body: "Body") -> int:
    """The C ABI's material code: 0 IsotropicLinearElasticity, 1
    CompressibleNeohookeanElasticity, 2 Sand_SachithLocal."""
    if body.material_class not in MATERIAL_CLASSES:
        raise ValueError(f"unknown material class {body.material_class!r}")
    return MATERIAL_CLASSES.index(body.material_class)


def sand_params(body: "Body") -> Tuple[Tuple[float, ...], bool]:
    """A Sand_SachithLocal body's properties as its init resolves them
    (sand_sachithlocal.cpp:57-103): (grain diameter, mu_s, grains_rho,
    rho_critical, mu_2, I_0), with mu_2 = mu_s and I_0 = 1 unless both are
    given; and whether USE_DENSITY_FOR_PRESSURE is set."""
    p = tuple(float(v) for v in body.material_props)
    if len(p) < 4:
        raise ValueError("Sand_SachithLocal needs E, nu, grain diameter, mu_s, grains_rho and rho_critical")
    if len(p) < 6:
        p = p[:4] + (p[1], 1.0)
    return p[:6], SAND_DENSITY_PRESSURE in body.material_str_props


def boundary_class(body: "Body") -> Optional[str]:
    """The boundary class name of a body, or None."""
    if body.boundary is True:
        return "CartesianBox"
    if not body.boundary:
        return None
    if body.boundary not in BOUNDARY_CLASSES:
        raise ValueError(f"unknown boundary class {body.boundary!r}")
    return str(body.boundary)


def boundary_kind(body: "Body") -> int:
    """The C ABI's boundary code: 0 none, 1 CartesianBox, 2 CartesianSmoothBox,
    3 CartesianFrictionalBox."""
    cls = boundary_class(body)
    return 0 if cls is None else 1 + BOUNDARY_CLASSES.index(cls)


@dataclasses.dataclass
class Contact:
    """ContactHuang between bodies b1 and b2 with friction mu; reflected:
    ContactHuang_ReflectedBoundary (the normal's wall components dropped)."""

    b1: int
    b2: int
    mu: float
    reflected: bool = False


@dataclasses.dataclass
class Case:
    name: str
    dim: int
    L: Tuple[float, ...]
    N: Tuple[int, ...]
    dt: float
    steps: int
    bodies: List[Body]
    contacts: List[Contact] = dataclasses.field(default_factory=list)
    cpdi: int = 1  # ExplicitUSL int-properties[0] (use_gimp)
    contact_spec: int = 1  # ExplicitUSL int-properties[1] (1 = IMPLICIT)
    gravity: Optional[Tuple[float, float, float]] = None  # None = DefaultDriver
    seed: Optional[int] = None

    @property
    def h(self) -> Tuple[float, ...]:
        return tuple(self.L[i] / self.N[i] for i in range(self.dim))

    @property
    def n_points(self) -> int:
        return sum(b.n for b in self.bodies)

    @property
    def n_nodes(self) -> int:
        out = 1
        for i in range(self.dim):
            out *= self.N[i] + 1
        return out


def block_points(lo: Sequence[float], counts: Sequence[int], h: Sequence[float], rho: float,
                 velocity: Sequence[float], jitter: float = 0.0,
                 rng: Optional[np.random.Generator] = None, name: str = "block",
                 E: float = 1e5, nu: float = 0.3) -> Body:
    """A block of 2 points per cell per axis starting at ``lo``.

    ``counts[i]`` points along axis i at ``lo + (j + 1/2) * h/2``; ``jitter`` is a
    fraction of ``h`` for a seeded uniform perturbation per axis.
    """
    dim = len(counts)
    axes = [lo[i] + (np.arange(counts[i], dtype=np.float64) + 0.5) * (h[i] / 2.0) for i in range(dim)]
    # last axis fastest, like examples/collision3D/test3D.points
    grids = np.meshgrid(*axes, indexing="ij")
    pos = np.stack([g.reshape(-1) for g in grids], axis=1)
    n = pos.shape[0]
    if jitter:
        assert rng is not None
        pos = pos + rng.uniform(-jitter, jitter, size=pos.shape) * np.asarray(h[:dim])
    x = np.zeros((n, 3))
    x[:, :dim] = pos
    vol = 1.0
    for i in range(dim):
        vol *= h[i] / 2.0
    xt = np.zeros((n, 3))
    xt[:, :dim] = np.asarray(velocity[:dim], dtype=np.float64)
    return Body(name=name, m=np.full(n, rho * vol), v=np.full(n, vol), x=x, x_t=xt,
                active=np.ones(n, dtype=np.int32), E=E, nu=nu)


def block_drop_2d() -> Case:
    """2D block drop: 20x20 grid on 1x1 m, 0.3x0.3 m block centred at (0.5,0.6)."""
    h = (0.05, 0.05)
    body = block_points((0.35, 0.45), (12, 12), h, 1000.0, (0.0, -1.0), name="block", E=1e5, nu=0.3)
    return Case(name="block_drop_2d", dim=2, L=(1.0, 1.0), N=(20, 20), dt=1e-4, steps=2000, bodies=[body])


def sliding_block(dim: int = 2, boundary: str = "CartesianFrictionalBox", mu: float = 0.3, n_cells: int = 16,
                  steps: int = 200) -> Case:
    """A block resting on the floor (and against the x = 0 wall) of an n^dim
    grid on a 1 m box, thrown along x and pressed into the floor, with the
    given boundary class (and its friction mu for CartesianFrictionalBox):
    the walls' nodes carry mass, so the boundary rules act from the first
    step."""
    h = tuple([1.0 / n_cells] * dim)
    counts = tuple([2 * (n_cells // 4)] * dim)
    lo = tuple([0.0] * dim)
    vel = (2.0, -1.0) if dim == 2 else (2.0, 0.5, -1.0)
    body = block_points(lo, counts, h, 1000.0, vel, name="block", E=1e5, nu=0.3)
    body.boundary = boundary
    body.boundary_mu = mu
    name = f"sliding_block_{dim}d_{boundary}"
    return Case(name=name, dim=dim, L=tuple([1.0] * dim), N=tuple([n_cells] * dim), dt=1e-4, steps=steps,
                bodies=[body])


def wall_collision(dim: int = 2, n_cells: int = 16, steps: int = 100, mu: float = 0.4,
                   reflected: bool = True) -> Case:
    """Two blocks resting on the floor of an n^dim grid on a 1 m box with
    slip walls (CartesianSmoothBox), thrown at each other along x, with
    ContactHuang (reflected: the ContactHuang_ReflectedBoundary variant)
    between them: the contact nodes include floor nodes, where the reflected
    variant drops the normal's floor component."""
    h = tuple([1.0 / n_cells] * dim)
    side = n_cells // 4
    counts = tuple([2 * side] * dim)
    lo1 = tuple([0.25] + [0.0] * (dim - 1))
    lo2 = tuple([0.25 + side * h[0]] + [0.0] * (dim - 1))
    v1 = tuple([1.0] + [0.0] * (dim - 1))
    v2 = tuple([-1.0] + [0.0] * (dim - 1))
    b1 = block_points(lo1, counts, h, 1000.0, v1, name="left", E=1e5, nu=0.3)
    b2 = block_points(lo2, counts, h, 1000.0, v2, name="right", E=1e5, nu=0.3)
    b1.boundary = b2.boundary = "CartesianSmoothBox"
    name = f"wall_collision_{dim}d" + ("_reflected" if reflected else "")
    return Case(name=name, dim=dim, L=tuple([1.0] * dim), N=tuple([n_cells] * dim), dt=1e-4, steps=steps,
                bodies=[b1, b2], contacts=[Contact(0, 1, mu, reflected)])


def two_body_collision_3d(n_cells: int = 128, steps: int = 1000, gravity=None, gap: Optional[float] = None,
                          speed: float = 1.0, mu: float = 0.4) -> Case:
    """Two 0.25 m cubes at (0.3,0.5,0.5) and (0.7,0.5,0.5) moving at +-1 m/s.

    ``gap`` (metres) instead places the second cube that far from the first,
    so that contact engages within the first steps.
    """
    h = (1.0 / n_cells,) * 3
    per_axis = int(round(0.25 / (h[0] / 2.0)))
    lo2 = 0.575 if gap is None else 0.425 + gap
    a = block_points((0.175, 0.375, 0.375), (per_axis,) * 3, h, 1000.0, (speed, 0.0, 0.0), name="cube1", E=1e6,
                     nu=0.3)
    b = block_points((lo2, 0.375, 0.375), (per_axis,) * 3, h, 1000.0, (-speed, 0.0, 0.0), name="cube2", E=1e6, nu=0.3)
    tag = "" if gap is None else "_touching"
    return Case(name=f"two_body_collision_3d_{n_cells}{tag}", dim=3, L=(1.0, 1.0, 1.0), N=(n_cells,) * 3, dt=2e-5,
                steps=steps, bodies=[a, b], contacts=[Contact(0, 1, mu)], gravity=gravity)


def two_body_collision_2d(n_cells: int = 20, steps: int = 200, gap: float = 0.02, mu: float = 0.4) -> Case:
    """2D analogue of the two-body collision, blocks already in contact range."""
    h = (1.0 / n_cells,) * 2
    per_axis = int(round(0.3 / (h[0] / 2.0)))
    a = block_points((0.15, 0.35), (per_axis, per_axis), h, 1000.0, (1.0, 0.5), name="left", E=1e5, nu=0.3)
    b = block_points((0.45 + gap, 0.3), (per_axis, per_axis), h, 1000.0, (-1.0, 0.0), name="right", E=1e5, nu=0.3)
    return Case(name=f"two_body_collision_2d_{n_cells}", dim=2, L=(1.0, 1.0), N=(n_cells, n_cells), dt=1e-4,
                steps=steps, bodies=[a, b], contacts=[Contact(0, 1, mu)])


def sand_column(dim: int = 2, n_cells: int = 20, steps: int = 200, density_pressure: bool = False,
                mu_2: Optional[float] = None) -> Case:
    """A granular column collapsing under gravity on the floor of a 1 m box
    (0.5 m deep in 3D), after the reference's own column-collapse examples
    (examples/columncollapse2D, columncollapse3D): Sand_SachithLocal with
    E = 1e7, nu = 0.3, grain diameter 0.01 m, mu_s = 0.577, grains_rho =
    1650, rho_critical = 1000 (optionally mu_2 and I_0 = 0.278, and
    USE_DENSITY_FOR_PRESSURE), density 1500, CartesianBox, dt = 1e-4. The
    column is 0.2 m wide and 0.4 m tall at the centre of the floor."""
    L = (1.0, 1.0) if dim == 2 else (1.0, 1.0, 0.5)
    N = (n_cells, n_cells) if dim == 2 else (n_cells, n_cells, n_cells // 2)
    h = tuple(L[i] / N[i] for i in range(dim))
    size = (0.2, 0.4) if dim == 2 else (0.2, 0.2, 0.4)
    lo = (0.4, 0.0) if dim == 2 else (0.4, 0.4, 0.0)
    counts = tuple(int(round(size[i] / (h[i] / 2.0))) for i in range(dim))
    body = block_points(lo, counts, h, 1500.0, (0.0,) * dim, name="column", E=1e7, nu=0.3)
    body.material_class = "Sand_SachithLocal"
    body.material_props = (0.01, 0.577, 1650.0, 1000.0) + (() if mu_2 is None else (mu_2, 0.278))
    body.material_str_props = (SAND_DENSITY_PRESSURE,) if density_pressure else ()
    name = f"sand_column_{dim}d" + ("_mu2" if mu_2 is not None else "") + ("_density" if density_pressure else "")
    return Case(name=name, dim=dim, L=L, N=N, dt=1e-4, steps=steps, bodies=[body])


def column_collapse_3d(scale: int = 1, seed: int = 1002, steps: int = 500) -> Case:
    """Column 0.5x0.5x0.75 m on the floor of a 2x2x1 m domain, rho=1500."""
    N = (256 // scale, 256 // scale, 128 // scale)
    h = (2.0 / N[0], 2.0 / N[1], 1.0 / N[2])
    counts = tuple(int(round(s / (hh / 2.0))) for s, hh in zip((0.5, 0.5, 0.75), h))
    rng = np.random.default_rng(seed)
    body = block_points((0.75, 0.75, 0.0), counts, h, 1500.0, (0.0, 0.0, 0.0), jitter=0.01, rng=rng,
                        name="column", E=1e6, nu=0.3)
    return Case(name=f"column_collapse_3d_s{scale}", dim=3, L=(2.0, 2.0, 1.0), N=N, dt=1e-5, steps=steps,
                bodies=[body], seed=seed)


def _cfl_dt(h: float, E: float, nu: float, rho: float, vmax: float, courant: float = 0.3) -> float:
    G = E / (2.0 * (1.0 + nu))
    K = E / (3.0 * (1.0 - 2.0 * nu))
    c = math.sqrt((K + 4.0 * G / 3.0) / rho)
    return courant * h / (c + vmax)


def block_drop_ensemble(count: int = 512, seed: int = 1003, n_range=(16, 96), steps: int = 500,
                        side_range=(0.15, 0.4)) -> List[Case]:
    """Independent 3D block drops drawn from ``seed``.

    Per instance: N log-uniform in ``n_range`` (grid N^3 on a 1 m cube), a cube of
    side uniform in ``side_range`` placed at least one cell from every wall,
    velocity uniform in [-2,2]^3, E log-uniform in [1e4,1e7], nu uniform in
    [0.2,0.45], rho=1000, DefaultDriver gravity, dt = 0.3 h / (c + |v|max).
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        out.append(_block_drop(rng, n, steps, side_range, f"ensemble_{seed}_{k}", seed))
    return out


def _block_drop(rng: np.random.Generator, n: int, steps: int, side_range, name: str, seed: int) -> Case:
    """One block drop on an n^3 grid with the remaining draws from ``rng``."""
    h = 1.0 / n
    side = rng.uniform(*side_range)
    per_axis = max(2, int(round(side / (h / 2.0))))
    side = per_axis * h / 2.0
    lo = [rng.uniform(h, 1.0 - h - side) for _ in range(3)]
    vel = rng.uniform(-2.0, 2.0, size=3)
    E = math.exp(rng.uniform(math.log(1e4), math.log(1e7)))
    nu = rng.uniform(0.2, 0.45)
    body = block_points(lo, (per_axis,) * 3, (h,) * 3, 1000.0, vel, name="block", E=E, nu=nu)
    dt = _cfl_dt(h, E, nu, 1000.0, float(np.abs(vel).max()) * math.sqrt(3.0))
    return Case(name=name, dim=3, L=(1.0, 1.0, 1.0), N=(n, n, n), dt=dt, steps=steps, bodies=[body], seed=seed)


@dataclasses.dataclass
class RequestSpec:
    """One request of a serving stream: its arrival time and the draws that
    make its case (``serving_case``); the arrays are built only when needed."""

    index: int
    arrival: float
    kind: str      # "block" or "contact"
    n: int
    steps: int
    mu: float
    seed: int


def serving_stream(rate: float = 100.0, duration: float = 60.0, seed: int = 1004, n_range=(16, 128),
                   steps_range=(200, 5000), contact_frac: float = 0.1) -> List[RequestSpec]:
    """Poisson arrivals at ``rate`` per second for ``duration`` seconds. Each
    request is a 3D block drop drawn like ``block_drop_ensemble`` with N
    log-uniform in ``n_range`` and a step count log-uniform in
    ``steps_range``; a fraction ``contact_frac`` are instead two-body
    ContactHuang collisions laid out like ``two_body_collision_3d`` at the
    drawn N (mu uniform in [0.1, 0.6], dt scaled with the cell size)."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        kind = "contact" if rng.random() < contact_frac else "block"
        n = int(round(math.exp(rng.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        steps = int(round(math.exp(rng.uniform(math.log(steps_range[0]), math.log(steps_range[1])))))
        mu = float(rng.uniform(0.1, 0.6))
        out.append(RequestSpec(len(out), t, kind, n, steps, mu, int(rng.integers(0, 2**31 - 1))))
    return out


def serving_case(spec: RequestSpec) -> Case:
    """The case of a serving request (deterministic in the spec)."""
    if spec.kind == "contact":
        c = two_body_collision_3d(spec.n, steps=spec.steps, mu=spec.mu)
        c.dt = 2e-5 * 128.0 / spec.n
        c.name = f"request_{spec.index}_contact"
        return c
    rng = np.random.default_rng(spec.seed)
    return _block_drop(rng, spec.n, spec.steps, (0.15, 0.4), f"request_{spec.index}", spec.seed)


def _fmt(v: float) -> str:
    return repr(float(v))


def write_points_file(body: Body, path: str, dim: int) -> None:
    """Writes a ``.points`` file: count, then ``m v x.. x_t.. active`` lines."""
    cols = [body.m[:, None], body.v[:, None], body.x[:, :dim], body.x_t[:, :dim]]
    arr = np.concatenate(cols, axis=1)
    with open(path, "w") as f:
        f.write(f"{body.n}\n")
        for row, act in zip(arr, body.active):
            f.write(" ".join(_fmt(v) for v in row) + f" {int(act)}\n")


def read_points_file(path: str, dim: int) -> Tuple[np.ndarray, ...]:
    """Reads a ``.points`` file; returns (m, v, x (n,3), x_t (n,3), active)."""
    with open(path) as f:
        n = int(f.readline())
        data = np.loadtxt(f, ndmin=2)
    if data.shape[0] != n:
        raise ValueError(f"{path}: header says {n} points, found {data.shape[0]}")
    if data.shape[1] != 3 + 2 * dim:
        raise ValueError(f"{path}: expected {3 + 2 * dim} columns, found {data.shape[1]}")
    x = np.zeros((n, 3))
    xt = np.zeros((n, 3))
    x[:, :dim] = data[:, 2:2 + dim]
    xt[:, :dim] = data[:, 2 + dim:2 + 2 * dim]
    return data[:, 0].copy(), data[:, 1].copy(), x, xt, data[:, -1].astype(np.int32)


def write_case(case: Case, directory: str, solver_class: str = "ExplicitUSL", points_class: str = "DefaultPoints",
               threads: Optional[int] = None, solver_extra: Sequence[int] = (),
               point_int_props: Sequence[int] = (), serializer_class: str = "DefaultVTK",
               frame_dir: str = "output", sample_rate: float = 60.0,
               serializer_int_props: Sequence[int] = ()) -> str:
    """Writes ``<name>.cfg`` and the ``.points`` files; returns the cfg path.
    ``solver_extra`` appends solver int-properties (the GPU solver's
    write-back interval and form); ``point_int_props`` are DefaultPoints'
    int-properties ({1}: the point-element history, use_elem); the
    serializer writes frames to ``frame_dir`` at ``sample_rate`` per
    simulated second (``serializer_int_props``: its int-properties)."""
    os.makedirs(directory, exist_ok=True)
    lines = ["job", "{", f"    dt = {_fmt(case.dt)}", "    t = 0", f"    TYPE = {case.dim}"]
    if threads is not None:
        lines.append(f"    threads = {threads}")
    lines += ["}", "", "serializer", "{", f'    class = "{serializer_class}"', f"    properties = {{{_fmt(sample_rate)}}}",
              f'    str-properties = {{"{frame_dir}","save","case"}}']
    if serializer_int_props:
        lines += ["    int-properties = {" + ",".join(str(v) for v in serializer_int_props) + "}"]
    lines += ["}", ""]
    stop = case.dt * case.steps
    if case.gravity is None:
        lines += ["driver", "{", '    class = "DefaultDriver"', f"    properties = {{{_fmt(stop)}}}", "}", ""]
    else:
        g = ",".join(_fmt(v) for v in case.gravity[:case.dim])
        lines += ["driver", "{", '    class = "UserDefinedGravityDriver"', f"    properties = {{{_fmt(stop)},{g}}}",
                  "}", ""]
    sprops = ",".join(str(v) for v in [case.cpdi, case.contact_spec, *solver_extra])
    lines += ["solver", "{", f'    class = "{solver_class}"', f"    int-properties = {{{sprops}}}", "}", ""]
    lines += ["grid", "{", '    class = "CartesianLinear"',
              "    properties = {" + ",".join(_fmt(case.L[i]) for i in range(case.dim)) + "}",
              "    int-properties = {" + ",".join(str(case.N[i]) for i in range(case.dim)) + "}", "}", ""]
    for bi, body in enumerate(case.bodies):
        pfile = f"{case.name}_{bi}_{body.name}.points"
        write_points_file(body, os.path.join(directory, pfile), case.dim)
        lines += ["body", "{", '    class = "DefaultBody"', f'    name = "{body.name}"', f'    point-file = "{pfile}"',
                  f'    point-class = "{points_class}"', '    node-class = "DefaultNodes"']
        if point_int_props:
            lines += ["    point-int-props = {" + ",".join(str(v) for v in point_int_props) + "}"]
        if body.material:
            props = ",".join(_fmt(v) for v in (body.E, body.nu, *body.material_props))
            lines += [f'    material-class = "{body.material_class}"', f"    material-props = {{{props}}}"]
            if body.material_str_props:
                sp = ",".join(f'"{v}"' for v in body.material_str_props)
                lines += [f"    material-str-props = {{{sp}}}"]
        cls = boundary_class(body)
        if cls is not None:
            lines += [f'    boundary-class = "{cls}"']
            if cls == "CartesianFrictionalBox":
                lines += [f"    boundary-props = {{{_fmt(body.boundary_mu)}}}"]
        lines += ["}", ""]
    for c in case.contacts:
        cclass = "ContactHuang_ReflectedBoundary" if c.reflected else "ContactHuang"
        lines += ["contact", "{", '    name = "contact"', f'    class = "{cclass}"', f"    properties = {{{_fmt(c.mu)}}}",
                  f'    str-properties = {{"{case.bodies[c.b1].name}","{case.bodies[c.b2].name}"}}', "}", ""]
    path = os.path.join(directory, f"{case.name}.cfg")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return path
