"""ctypes binding of the C ABI in include/mpm_b200.h, and ``GPUExplicitUSL``,
the B200 replacement for mpm_3d's ExplicitUSL solver on a ``Case``.

The binding loads ``mpm_3d_b200/lib/libmpm_b200.so`` and fails loudly when it
is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional, Tuple

import numpy as np

from . import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
# MPM_B200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("MPM_B200_LIB", os.path.join(HERE, "lib", "libmpm_b200.so"))

MODES = {"fp64": 0, "fp64_deterministic": 1, "mixed": 2}
# forms of the fused kernel (mpmgpu_kernel_form)
KERNELS = {"staged": 0, "point_per_thread": 1}
KERNEL_NAMES = {v: k for k, v in KERNELS.items()}
POINT_FIELDS = {"x": (0, 3), "u": (1, 3), "x_t": (2, 3), "mx_t": (3, 3), "b": (4, 3), "L": (5, 9), "T": (6, 9),
                "m": (7, 1), "v": (8, 1), "extent": (9, 1), "active": (10, 1), "gammap": (11, 1),
                "gammap_dot": (12, 1)}
NODE_FIELDS = {"m": (0, 1), "mx_t": (1, 3), "f": (2, 3), "x_t": (3, 3), "u": (4, 3), "diff_x_t": (5, 3)}
CONTACT_FIELDS = {"normal": (0, 3), "force": (1, 3)}


class MpmGpuError(RuntimeError):
    pass


class _Config(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("L", ctypes.c_double * 3), ("N", ctypes.c_int * 3), ("dt", ctypes.c_double),
                ("cpdi_spec", ctypes.c_int), ("contact_spec", ctypes.c_int), ("mode", ctypes.c_int),
                ("device", ctypes.c_int), ("keep_debug", ctypes.c_int), ("sort_interval", ctypes.c_int)]


class _BatchConfig(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("mode", ctypes.c_int), ("device", ctypes.c_int),
                ("sort_interval", ctypes.c_int), ("points_per_item", ctypes.c_int), ("no_graph", ctypes.c_int),
                ("keep_debug", ctypes.c_int)]


class _ContactDesc(ctypes.Structure):
    _fields_ = [("body1", ctypes.c_int), ("body2", ctypes.c_int), ("mu", ctypes.c_double), ("reflected", ctypes.c_int)]


class _BodyDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("m", ctypes.c_void_p), ("v", ctypes.c_void_p), ("x", ctypes.c_void_p),
                ("x_t", ctypes.c_void_p), ("active", ctypes.c_void_p), ("has_material", ctypes.c_int),
                ("E", ctypes.c_double), ("nu", ctypes.c_double), ("has_boundary", ctypes.c_int),
                ("u", ctypes.c_void_p), ("T", ctypes.c_void_p), ("boundary_mu", ctypes.c_double),
                ("material_kind", ctypes.c_int), ("material_props", ctypes.c_double * 6),
                ("material_flags", ctypes.c_int)]


def _body_desc(body: "inputs.Body"):
    """mpmgpu_body_desc of a body, and the arrays it points at (keep them alive)."""
    arrs = dict(m=np.ascontiguousarray(body.m, np.float64), v=np.ascontiguousarray(body.v, np.float64),
                x=np.ascontiguousarray(body.x, np.float64), x_t=np.ascontiguousarray(body.x_t, np.float64),
                active=np.ascontiguousarray(body.active, np.int32))
    kind = inputs.material_kind(body)
    desc = _BodyDesc(body.n, _ptr(arrs["m"]).value, _ptr(arrs["v"]).value, _ptr(arrs["x"]).value,
                     _ptr(arrs["x_t"]).value, _ptr(arrs["active"]).value, int(body.material), body.E, body.nu,
                     inputs.boundary_kind(body), None, None, float(body.boundary_mu), kind)
    if body.material and kind == 2:
        props, density = inputs.sand_params(body)
        desc.material_props = (ctypes.c_double * 6)(*props)
        desc.material_flags = int(density)
    return desc, arrs


class _JobDesc(ctypes.Structure):
    _fields_ = [("grid", ctypes.POINTER(_Config)), ("nbodies", ctypes.c_int), ("bodies", ctypes.POINTER(_BodyDesc)),
                ("ncontacts", ctypes.c_int), ("contacts", ctypes.POINTER(_ContactDesc)),
                ("gravity_vector", ctypes.c_int), ("gravity", ctypes.c_double * 3), ("steps", ctypes.c_int64)]


_lib = None


def load() -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m mpm_3d_b200.build` "
                          "(there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.mpmgpu_status_string.restype = ctypes.c_char_p
    lib.mpmgpu_status_string.argtypes = [ctypes.c_int]
    lib.mpmgpu_last_error.restype = ctypes.c_char_p
    lib.mpmgpu_last_error.argtypes = [vp]
    lib.mpmgpu_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(vp)]
    lib.mpmgpu_add_body.argtypes = [vp, ctypes.POINTER(_BodyDesc), ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_add_contact.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_add_contact_reflected.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                 ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_set_gravity.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.mpmgpu_step.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_synchronize.argtypes = [vp]
    for fn in ("mpmgpu_download_points", "mpmgpu_download_nodes", "mpmgpu_download_contact", "mpmgpu_frame_points",
               "mpmgpu_frame_nodes", "mpmgpu_frame_contact"):
        getattr(lib, fn).argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
    lib.mpmgpu_frame_begin.argtypes = [vp]
    lib.mpmgpu_dump_map.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.POINTER(ctypes.c_int64)]
    lib.mpmgpu_dump_map_noalloc.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_int64,
                                            ctypes.POINTER(ctypes.c_int64)]
    lib.mpmgpu_sizes.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    lib.mpmgpu_launch_count.restype = ctypes.c_int64
    lib.mpmgpu_launch_count.argtypes = [vp]
    lib.mpmgpu_stream.restype = vp
    lib.mpmgpu_stream.argtypes = [vp]
    lib.mpmgpu_profile.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_set_wait_limit.argtypes = [vp, ctypes.c_uint32]
    lib.mpmgpu_set_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.mpmgpu_kernel.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_batch_set_kernel.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.mpmgpu_batch_kernel_form.argtypes = [vp]
    lib.mpmgpu_profile_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]
    lib.mpmgpu_destroy.argtypes = [vp]
    i64p = ctypes.POINTER(ctypes.c_int64)
    lib.mpmgpu_batch_create.argtypes = [ctypes.POINTER(_BatchConfig), ctypes.POINTER(vp)]
    lib.mpmgpu_batch_last_error.restype = ctypes.c_char_p
    lib.mpmgpu_batch_last_error.argtypes = [vp]
    lib.mpmgpu_batch_footprint.argtypes = [vp, ctypes.POINTER(_JobDesc), i64p]
    lib.mpmgpu_batch_add_job.argtypes = [vp, ctypes.POINTER(_JobDesc), ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_batch_step.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_batch_synchronize.argtypes = [vp]
    lib.mpmgpu_batch_job_state.argtypes = [vp, ctypes.c_int, i64p, i64p]
    lib.mpmgpu_batch_sizes.argtypes = [vp, ctypes.c_int, ctypes.c_int, i64p, i64p]
    lib.mpmgpu_batch_download_points.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    lib.mpmgpu_batch_download_points_many.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                                      ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    lib.mpmgpu_batch_remove_job.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_batch_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_int), i64p, i64p]
    lib.mpmgpu_batch_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_batch_points_per_item.argtypes = [vp]
    lib.mpmgpu_batch_sort_interval.argtypes = [vp]
    lib.mpmgpu_batch_active_nodes.argtypes = [vp, i64p, i64p]
    lib.mpmgpu_active_nodes.argtypes = [vp, i64p, i64p]
    lib.mpmgpu_batch_profile.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_batch_profile_read.argtypes = [vp, ctypes.c_int, i64p, ctypes.POINTER(ctypes.c_double)]
    lib.mpmgpu_batch_stream.restype = vp
    lib.mpmgpu_batch_stream.argtypes = [vp]
    lib.mpmgpu_batch_launch_count.restype = ctypes.c_int64
    lib.mpmgpu_batch_launch_count.argtypes = [vp]
    lib.mpmgpu_batch_destroy.argtypes = [vp]
    lib.mpmgpu_server_create.argtypes = [ctypes.POINTER(_BatchConfig), ctypes.c_int64, ctypes.POINTER(vp)]
    lib.mpmgpu_server_last_error.restype = ctypes.c_char_p
    lib.mpmgpu_server_last_error.argtypes = [vp]
    lib.mpmgpu_server_submit.argtypes = [vp, ctypes.POINTER(_JobDesc), ctypes.POINTER(ctypes.c_int)]
    lib.mpmgpu_server_footprint.argtypes = [vp, ctypes.POINTER(_JobDesc), i64p]
    lib.mpmgpu_server_advance.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_server_poll.restype = ctypes.c_int
    lib.mpmgpu_server_poll.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    lib.mpmgpu_server_request.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), i64p, i64p]
    lib.mpmgpu_server_result.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp]
    lib.mpmgpu_server_release.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_server_cancel.argtypes = [vp, ctypes.c_int]
    lib.mpmgpu_server_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int), i64p, i64p, i64p]
    lib.mpmgpu_server_clock.restype = ctypes.c_double
    lib.mpmgpu_server_clock.argtypes = [vp]
    lib.mpmgpu_server_destroy.argtypes = [vp]
    lib.mpmgpu_points_file_count.argtypes = [ctypes.c_char_p, i64p]
    lib.mpmgpu_points_file_read.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int64, vp, vp, vp, vp, vp,
                                            ctypes.c_int, i64p]
    _lib = lib
    return lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


def read_points_file(path: str, dim: int, threads: int = 0):
    """Reads a DefaultPoints ``.points`` file with the library's parallel
    reader (mpmgpu_points_file_read; host only, no GPU): returns (m, v,
    x (n,3), x_t (n,3), active), parsed as DefaultPoints::readFromFile does."""
    lib = load()
    n = ctypes.c_int64()
    st = lib.mpmgpu_points_file_count(path.encode(), ctypes.byref(n))
    if st != 0:
        raise MpmGpuError(f"{path}: no point count on the first line (status {st})")
    m = np.zeros(n.value)
    v = np.zeros(n.value)
    x = np.zeros((n.value, 3))
    xt = np.zeros((n.value, 3))
    active = np.zeros(n.value, np.int32)
    bad = ctypes.c_int64()
    st = lib.mpmgpu_points_file_read(path.encode(), dim, n.value, _ptr(m), _ptr(v), _ptr(x), _ptr(xt), _ptr(active),
                                     threads, ctypes.byref(bad))
    if st != 0:
        raise MpmGpuError(f"{path}: unable to read line {bad.value} (status {st})")
    return m, v, x, xt, active


class GPUExplicitUSL:
    """ExplicitUSL on the GPU for one ``inputs.Case`` (the Job's grid, bodies,
    contacts and driver gravity), with the reference's step/frame surface:
    ``step(n)`` advances n steps; ``points``/``nodes``/``contact`` read fields
    in the reference's layout (AoS, original point order, reference node ids).
    """

    def __init__(self, case: inputs.Case, mode: str = "fp64", keep_debug: bool = False, device: int = 0,
                 sort_interval: int = 0, kernel: Optional[Tuple[str, int]] = None):
        self.lib = load()
        self.case = case
        cfg = _Config()
        cfg.dim = case.dim
        for d in range(3):
            cfg.L[d] = case.L[d] if d < case.dim else 0.0
            cfg.N[d] = case.N[d] if d < case.dim else 0
        cfg.dt = case.dt
        cfg.cpdi_spec = case.cpdi
        cfg.contact_spec = case.contact_spec
        cfg.mode = MODES[mode]
        cfg.device = device
        cfg.keep_debug = int(keep_debug)
        cfg.sort_interval = int(sort_interval)
        h = ctypes.c_void_p()
        self._check(self.lib.mpmgpu_create(ctypes.byref(cfg), ctypes.byref(h)), None)
        self.h = h
        for body in case.bodies:
            desc, arrs = _body_desc(body)
            bid = ctypes.c_int()
            self._check(self.lib.mpmgpu_add_body(self.h, ctypes.byref(desc), ctypes.byref(bid)))
        for c in case.contacts:
            cid = ctypes.c_int()
            add = self.lib.mpmgpu_add_contact_reflected if c.reflected else self.lib.mpmgpu_add_contact
            self._check(add(self.h, c.b1, c.b2, c.mu, ctypes.byref(cid)))
        if case.gravity is not None:
            g = (ctypes.c_double * 3)(*(list(case.gravity) + [0.0] * (3 - len(case.gravity))))
            self._check(self.lib.mpmgpu_set_gravity(self.h, 1, g))
        if kernel is not None:
            self.set_kernel(*kernel)
        n_nodes = ctypes.c_int64()
        self._check(self.lib.mpmgpu_sizes(self.h, 0, None, ctypes.byref(n_nodes)))
        self.n_nodes = n_nodes.value

    def _check(self, status: int, h=0):
        if status != 0:
            hh = self.h if h == 0 else h
            msg = self.lib.mpmgpu_status_string(status).decode()
            detail = self.lib.mpmgpu_last_error(hh).decode() if hh else ""
            raise MpmGpuError(f"{msg}: {detail}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpmgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        self._check(self.lib.mpmgpu_step(self.h, n))

    def synchronize(self):
        self._check(self.lib.mpmgpu_synchronize(self.h))

    def launches(self) -> int:
        return int(self.lib.mpmgpu_launch_count(self.h))

    def stream(self) -> int:
        """The cudaStream_t (as an integer) the solver queues its work on."""
        return int(self.lib.mpmgpu_stream(self.h) or 0)

    STAGES = {"g2p2g": 0, "grid": 1, "compact": 2, "rebin": 3}

    def set_kernel(self, form: str, points_per_item: int):
        """Selects the fused kernel's form (KERNELS) and points per work item."""
        self._check(self.lib.mpmgpu_set_kernel(self.h, KERNELS[form], points_per_item))

    def autotune(self, steps: int = 5) -> Tuple[str, int]:
        """Times every available kernel form and points-per-item choice on
        this handle's bodies, then the re-binning interval, and keeps the
        fastest (the state after the call is the state before it)."""
        f = ctypes.c_int()
        c = ctypes.c_int()
        self._check(self.lib.mpmgpu_autotune(self.h, steps, ctypes.byref(f), ctypes.byref(c)))
        return KERNEL_NAMES[f.value], c.value

    def kernel(self) -> Tuple[str, int]:
        f = ctypes.c_int()
        c = ctypes.c_int()
        self._check(self.lib.mpmgpu_kernel(self.h, ctypes.byref(f), ctypes.byref(c)))
        return KERNEL_NAMES[f.value], c.value

    def set_wait_limit(self, polls: int):
        """Poll limit of the fused kernel's waits for bulk copies (2^24 by
        default); a wait that runs out makes the next synchronize raise."""
        self._check(self.lib.mpmgpu_set_wait_limit(self.h, polls))

    def active_nodes(self) -> Tuple[int, int]:
        """(nodes with mass in the last step, per body; drifted point visits)."""
        a = ctypes.c_int64()
        d = ctypes.c_int64()
        self._check(self.lib.mpmgpu_active_nodes(self.h, ctypes.byref(a), ctypes.byref(d)))
        return int(a.value), int(d.value)

    def profile(self, enable: bool = True):
        """Starts (and resets) or stops per-stage CUDA-event timing."""
        self._check(self.lib.mpmgpu_profile(self.h, int(enable)))

    def profile_read(self) -> Dict[str, Tuple[int, float]]:
        """Per stage: (launches, total device milliseconds)."""
        out = {}
        for name, sid in self.STAGES.items():
            n = ctypes.c_int64()
            ms = ctypes.c_double()
            self._check(self.lib.mpmgpu_profile_read(self.h, sid, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (int(n.value), float(ms.value))
        return out

    def points(self, b: int, name: str) -> np.ndarray:
        fid, w = POINT_FIELDS[name]
        out = np.zeros((self.case.bodies[b].n, w))
        self._check(self.lib.mpmgpu_download_points(self.h, b, fid, _ptr(out)))
        return out

    def nodes(self, b: int, name: str) -> np.ndarray:
        fid, w = NODE_FIELDS[name]
        out = np.zeros((self.n_nodes, w))
        self._check(self.lib.mpmgpu_download_nodes(self.h, b, fid, _ptr(out)))
        return out

    def contact(self, c: int, name: str) -> np.ndarray:
        fid, w = CONTACT_FIELDS[name]
        out = np.zeros((self.n_nodes, w))
        self._check(self.lib.mpmgpu_download_contact(self.h, c, fid, _ptr(out)))
        return out

    def frame_begin(self):
        """Queues copies of every field behind the steps queued so far
        (returns at once); frame_points / frame_nodes / frame_contact read
        them as they stood then."""
        self._check(self.lib.mpmgpu_frame_begin(self.h))

    def frame_points(self, b: int, name: str) -> np.ndarray:
        fid, w = POINT_FIELDS[name]
        out = np.zeros((self.case.bodies[b].n, w))
        self._check(self.lib.mpmgpu_frame_points(self.h, b, fid, _ptr(out)))
        return out

    def frame_nodes(self, b: int, name: str) -> np.ndarray:
        fid, w = NODE_FIELDS[name]
        out = np.zeros((self.n_nodes, w))
        self._check(self.lib.mpmgpu_frame_nodes(self.h, b, fid, _ptr(out)))
        return out

    def frame_contact(self, c: int, name: str) -> np.ndarray:
        fid, w = CONTACT_FIELDS[name]
        out = np.zeros((self.n_nodes, w))
        self._check(self.lib.mpmgpu_frame_contact(self.h, c, fid, _ptr(out)))
        return out

    def map(self, b: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """Exact S / gradS triplets of body b at the current positions, in the
        reference's order: (node, point, S value, gradient (k,3))."""
        cnt = ctypes.c_int64()
        self._check(self.lib.mpmgpu_dump_map(self.h, b, None, None, None, None, ctypes.byref(cnt)))
        n = cnt.value
        node = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        val = np.zeros(n)
        grad = np.zeros((n, 3))
        self._check(self.lib.mpmgpu_dump_map(self.h, b, _ptr(node), _ptr(pt), _ptr(val), _ptr(grad),
                                             ctypes.byref(cnt)))
        return node, pt, val, grad

    def map_noalloc(self, b: int, d_node: int, d_point: int, d_s: int, d_grad: int, capacity: int) -> int:
        """Allocation-free triplet export into caller-owned device arrays
        (integer device addresses); returns the triplet count."""
        cnt = ctypes.c_int64()
        self._check(self.lib.mpmgpu_dump_map_noalloc(self.h, b, d_node, d_point, d_s, d_grad, capacity,
                                                     ctypes.byref(cnt)))
        return cnt.value


def _case_config(case: inputs.Case, mode: str = "fp64") -> _Config:
    cfg = _Config()
    cfg.dim = case.dim
    for d in range(3):
        cfg.L[d] = case.L[d] if d < case.dim else 0.0
        cfg.N[d] = case.N[d] if d < case.dim else 0
    cfg.dt = case.dt
    cfg.cpdi_spec = case.cpdi
    cfg.contact_spec = case.contact_spec
    cfg.mode = MODES[mode]
    return cfg


def job_desc(case: inputs.Case, steps: Optional[int] = None):
    """mpmgpu_job_desc of a case, and the arrays it points at (keep them alive)."""
    keep = []
    cfg = _case_config(case)
    bodies = (_BodyDesc * len(case.bodies))()
    for i, body in enumerate(case.bodies):
        bodies[i], arrs = _body_desc(body)
        keep.append(arrs)
    contacts = (_ContactDesc * max(1, len(case.contacts)))()
    for i, c in enumerate(case.contacts):
        contacts[i] = _ContactDesc(c.b1, c.b2, c.mu, int(c.reflected))
    desc = _JobDesc()
    desc.grid = ctypes.pointer(cfg)
    desc.nbodies = len(case.bodies)
    desc.bodies = bodies
    desc.ncontacts = len(case.contacts)
    desc.contacts = contacts
    if case.gravity is not None:
        desc.gravity_vector = 1
        g = list(case.gravity) + [0.0] * (3 - len(case.gravity))
        for d in range(3):
            desc.gravity[d] = g[d]
    desc.steps = int(case.steps if steps is None else steps)
    keep += [cfg, bodies, contacts]
    return desc, keep


class GPUBatch:
    """Many independent ``inputs.Case`` jobs stepped together on one GPU
    (``mpmgpu_batch_*``): one launch per stage for all jobs, the step replayed
    from a CUDA graph. Jobs may be added while others run; each runs its own
    step count and then stops advancing until removed.
    """

    def __init__(self, dim: int = 3, mode: str = "mixed", device: int = 0, sort_interval: int = 0,
                 points_per_item: int = 0, graph: bool = True, keep_debug: bool = False,
                 kernel: Optional[Tuple[str, int]] = None):
        self.lib = load()
        cfg = _BatchConfig(dim, MODES[mode], device, sort_interval, points_per_item, 0 if graph else 1,
                           int(keep_debug))
        h = ctypes.c_void_p()
        st = self.lib.mpmgpu_batch_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise MpmGpuError(f"{self.lib.mpmgpu_status_string(st).decode()}: batch create")
        self.h = h
        self.dim = dim
        self.cases: Dict[int, inputs.Case] = {}
        if kernel is not None:
            self.set_kernel(*kernel)

    def _check(self, status: int):
        if status != 0:
            msg = self.lib.mpmgpu_status_string(status).decode()
            raise MpmGpuError(f"{msg}: {self.lib.mpmgpu_batch_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpmgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _job_desc(self, case: inputs.Case, steps: Optional[int]):
        return job_desc(case, steps)

    def footprint(self, case: inputs.Case, steps: Optional[int] = None) -> int:
        desc, _keep = self._job_desc(case, steps)
        out = ctypes.c_int64()
        self._check(self.lib.mpmgpu_batch_footprint(self.h, ctypes.byref(desc), ctypes.byref(out)))
        return int(out.value)

    def add(self, case: inputs.Case, steps: Optional[int] = None) -> int:
        """Adds a job (runs ``steps``, default ``case.steps``); returns its id."""
        desc, _keep = self._job_desc(case, steps)
        jid = ctypes.c_int()
        self._check(self.lib.mpmgpu_batch_add_job(self.h, ctypes.byref(desc), ctypes.byref(jid)))
        self.cases[jid.value] = case
        return jid.value

    def step(self, n: int = 1):
        self._check(self.lib.mpmgpu_batch_step(self.h, n))

    def synchronize(self):
        self._check(self.lib.mpmgpu_batch_synchronize(self.h))

    def state(self, job: int) -> Tuple[int, int]:
        done = ctypes.c_int64()
        left = ctypes.c_int64()
        self._check(self.lib.mpmgpu_batch_job_state(self.h, job, ctypes.byref(done), ctypes.byref(left)))
        return int(done.value), int(left.value)

    def points(self, job: int, b: int, name: str) -> np.ndarray:
        fid, w = POINT_FIELDS[name]
        out = np.zeros((self.cases[job].bodies[b].n, w))
        self._check(self.lib.mpmgpu_batch_download_points(self.h, job, b, fid, _ptr(out)))
        return out

    def points_many(self, jobs, b: int, name: str, threads: int = 0):
        """One point field of body b of several jobs, copied with one wait
        and converted on host threads (all host threads by default)."""
        fid, w = POINT_FIELDS[name]
        outs = [np.zeros((self.cases[j].bodies[b].n, w)) for j in jobs]
        ids = (ctypes.c_int * len(jobs))(*jobs)
        ptrs = (ctypes.c_void_p * len(jobs))(*[o.ctypes.data for o in outs])
        self._check(self.lib.mpmgpu_batch_download_points_many(self.h, len(jobs), ids, b, fid, ptrs,
                                                               threads or (os.cpu_count() or 1)))
        return outs

    def remove(self, job: int):
        self._check(self.lib.mpmgpu_batch_remove_job(self.h, job))
        self.cases.pop(job, None)

    def counts(self) -> Tuple[int, int, int]:
        """(jobs still stepping, their points, device bytes held)."""
        j = ctypes.c_int()
        p = ctypes.c_int64()
        b = ctypes.c_int64()
        self._check(self.lib.mpmgpu_batch_counts(self.h, ctypes.byref(j), ctypes.byref(p), ctypes.byref(b)))
        return int(j.value), int(p.value), int(b.value)

    def autotune(self, steps: int = 5) -> int:
        cap = ctypes.c_int()
        self._check(self.lib.mpmgpu_batch_autotune(self.h, steps, ctypes.byref(cap)))
        return int(cap.value)

    def points_per_item(self) -> int:
        return int(self.lib.mpmgpu_batch_points_per_item(self.h))

    def kernel_form(self) -> str:
        return KERNEL_NAMES[int(self.lib.mpmgpu_batch_kernel_form(self.h))]

    def set_kernel(self, form: str, points_per_item: int):
        """Selects the fused kernel's form (KERNELS) and points per work item."""
        self._check(self.lib.mpmgpu_batch_set_kernel(self.h, KERNELS[form], points_per_item))

    def sort_interval(self) -> int:
        return int(self.lib.mpmgpu_batch_sort_interval(self.h))

    def active_nodes(self) -> Tuple[int, int]:
        """(nodes with mass in the last step, per body; drifted point visits)."""
        a = ctypes.c_int64()
        d = ctypes.c_int64()
        self._check(self.lib.mpmgpu_batch_active_nodes(self.h, ctypes.byref(a), ctypes.byref(d)))
        return int(a.value), int(d.value)

    STAGES = GPUExplicitUSL.STAGES

    def profile(self, enable: bool = True):
        self._check(self.lib.mpmgpu_batch_profile(self.h, int(enable)))

    def profile_read(self) -> Dict[str, Tuple[int, float]]:
        out = {}
        for name, sid in self.STAGES.items():
            n = ctypes.c_int64()
            ms = ctypes.c_double()
            self._check(self.lib.mpmgpu_batch_profile_read(self.h, sid, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (int(n.value), float(ms.value))
        return out

    def stream(self) -> int:
        return int(self.lib.mpmgpu_batch_stream(self.h) or 0)

    def launches(self) -> int:
        return int(self.lib.mpmgpu_batch_launch_count(self.h))


STATUS_NOMEM = 3
STATUS_STATE = 5


class GPUServer:
    """Continuous batching of simulation requests (``mpmgpu_server_*``):
    ``submit`` admits a case at once if its device footprint fits the budget
    left by the running requests (else returns None: keep it queued and retry
    after ``advance``); ``advance(k)`` steps everything running k steps and
    collects the requests that have run their steps."""

    def __init__(self, budget_bytes: int, dim: int = 3, mode: str = "mixed", device: int = 0, sort_interval: int = 0,
                 points_per_item: int = 0, graph: bool = True):
        self.lib = load()
        cfg = _BatchConfig(dim, MODES[mode], device, sort_interval, points_per_item, 0 if graph else 1, 0)
        h = ctypes.c_void_p()
        st = self.lib.mpmgpu_server_create(ctypes.byref(cfg), int(budget_bytes), ctypes.byref(h))
        if st != 0:
            raise MpmGpuError(f"{self.lib.mpmgpu_status_string(st).decode()}: server create")
        self.h = h
        self.cases: Dict[int, inputs.Case] = {}

    def _check(self, status: int):
        if status != 0:
            msg = self.lib.mpmgpu_status_string(status).decode()
            raise MpmGpuError(f"{msg}: {self.lib.mpmgpu_server_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mpmgpu_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def footprint(self, case: inputs.Case, steps: Optional[int] = None) -> int:
        desc, _keep = job_desc(case, steps)
        out = ctypes.c_int64()
        self._check(self.lib.mpmgpu_server_footprint(self.h, ctypes.byref(desc), ctypes.byref(out)))
        return int(out.value)

    def submit(self, case: inputs.Case, steps: Optional[int] = None) -> Optional[int]:
        desc, _keep = job_desc(case, steps)
        rid = ctypes.c_int()
        st = self.lib.mpmgpu_server_submit(self.h, ctypes.byref(desc), ctypes.byref(rid))
        if st == STATUS_STATE:
            return None
        if st == STATUS_NOMEM:
            return -1   # larger than the whole budget: can never run
        self._check(st)
        self.cases[rid.value] = case
        return rid.value

    def advance(self, steps: int):
        self._check(self.lib.mpmgpu_server_advance(self.h, steps))

    def poll(self, max_ids: int = 4096):
        ids = (ctypes.c_int * max_ids)()
        k = self.lib.mpmgpu_server_poll(self.h, ids, max_ids)
        return [ids[i] for i in range(k)]

    def request(self, rid: int) -> Dict[str, float]:
        st = ctypes.c_int()
        ta = ctypes.c_double()
        td = ctypes.c_double()
        pts = ctypes.c_int64()
        steps = ctypes.c_int64()
        self._check(self.lib.mpmgpu_server_request(self.h, rid, ctypes.byref(st), ctypes.byref(ta), ctypes.byref(td),
                                                   ctypes.byref(pts), ctypes.byref(steps)))
        return {"state": st.value, "t_admit": ta.value, "t_done": td.value, "points": pts.value, "steps": steps.value}

    def result(self, rid: int, b: int, name: str) -> np.ndarray:
        fid, w = POINT_FIELDS[name]
        out = np.zeros((self.cases[rid].bodies[b].n, w))
        self._check(self.lib.mpmgpu_server_result(self.h, rid, b, fid, _ptr(out)))
        return out

    def release(self, rid: int):
        self._check(self.lib.mpmgpu_server_release(self.h, rid))
        self.cases.pop(rid, None)

    def cancel(self, rid: int):
        """Cancels a running request (it leaves the batch at the next step
        boundary; the other requests are unaffected)."""
        self._check(self.lib.mpmgpu_server_cancel(self.h, rid))
        self.cases.pop(rid, None)

    def stats(self) -> Dict[str, int]:
        r = ctypes.c_int()
        res = ctypes.c_int64()
        lp = ctypes.c_int64()
        done = ctypes.c_int64()
        self._check(self.lib.mpmgpu_server_stats(self.h, ctypes.byref(r), ctypes.byref(res), ctypes.byref(lp),
                                                 ctypes.byref(done)))
        return {"running": r.value, "reserved_bytes": res.value, "live_points": lp.value,
                "particle_steps_done": done.value}

    def clock(self) -> float:
        return float(self.lib.mpmgpu_server_clock(self.h))
