"""ctypes bridge to the CPU oracles (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm
of ``bench.py`` import this module; the product (``mpm_3d_b200``) never does.

Two oracles are exposed with the same small interface (``step``, ``points``,
``nodes``, ``contact``, ``map``, ``grad_map``):

* ``ReferenceJob``: the reference's own hot-path sources compiled unmodified
  (``oracle/_ref/libmpmref_parity.so`` or ``libmpmref_timing.so``, built by
  ``oracle/Makefile`` where the reference tree is present), driven through its
  own ``Configurator`` from a ``.cfg`` file.
* ``RestatedJob``: the C restatement ``oracle/mpm_oracle.c``
  (``oracle/_ref/libmpm_oracle.so``), fed from an ``mpm_3d_b200.inputs.Case``.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a: np.ndarray, kind=_dp):
    return a.ctypes.data_as(kind)


def lib_path(name: str) -> str:
    return os.path.join(REF_DIR, name)


def available(name: str) -> bool:
    return os.path.exists(lib_path(name))


_LIBS = {}


def _load(name: str) -> ctypes.CDLL:
    if name not in _LIBS:
        _LIBS[name] = ctypes.CDLL(lib_path(name))
    return _LIBS[name]


class _JobBase:
    _prefix = ""

    def _f(self, fname):
        return getattr(self.lib, self._prefix + fname)

    def _field(self, fname, b, name, count, width):
        # the C side writes `got` packed doubles per entry (got <= width)
        out = np.zeros(count * width, dtype=np.float64)
        got = self._f(fname)(self.h, b, name.encode(), _ptr(out))
        if got < 0:
            raise KeyError(name)
        return out[:count * got].reshape(count, got).copy()


class ReferenceJob(_JobBase):
    """The reference solver compiled from its own sources."""

    _prefix = "ref_"

    def __init__(self, cfg_path: str, build: str = "parity"):
        self.lib = _load(f"libmpmref_{build}.so")
        L = self.lib
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_char_p]
        for fn in ("ref_step", "ref_num_points", "ref_num_nodes", "ref_num_bodies", "ref_get_point_field",
                   "ref_get_node_field", "ref_get_contact_field", "ref_map_size", "ref_grad_map_size",
                   "ref_get_map", "ref_get_grad_map", "ref_build_map", "ref_destroy", "ref_job_dim"):
            getattr(L, fn).argtypes = None
        L.ref_get_time.restype = ctypes.c_double
        h = L.ref_create(cfg_path.encode())
        if not h:
            raise RuntimeError(f"reference failed to configure {cfg_path}")
        self.h = ctypes.c_void_p(h)
        self.nbodies = L.ref_num_bodies(self.h)

    def close(self):
        if self.h is not None:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        self.lib.ref_step(self.h, ctypes.c_int(n))

    def build_map(self):
        self.lib.ref_build_map(self.h)

    def n_points(self, b):
        return self.lib.ref_num_points(self.h, b)

    def n_nodes(self, b=0):
        return self.lib.ref_num_nodes(self.h, b)

    def points(self, b, name):
        return self._field("get_point_field", b, name, self.n_points(b), 9)

    def nodes(self, b, name):
        return self._field("get_node_field", b, name, self.n_nodes(b), 3)

    def contact(self, c, name):
        return self._field("get_contact_field", c, name, self.n_nodes(0), 3)

    def map(self, b):
        n = self.lib.ref_map_size(self.h, b)
        node = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        val = np.zeros(n)
        self.lib.ref_get_map(self.h, b, _ptr(node, _ip), _ptr(pt, _ip), _ptr(val))
        return node, pt, val

    def grad_map(self, b):
        n = self.lib.ref_grad_map_size(self.h, b)
        node = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        g = np.zeros((n, 3))
        self.lib.ref_get_grad_map(self.h, b, _ptr(node, _ip), _ptr(pt, _ip), _ptr(g))
        return node, pt, g


class RestatedJob(_JobBase):
    """The C restatement of the step (oracle/mpm_oracle.c)."""

    _prefix = "oc_"

    def __init__(self, case):
        self.lib = _load("libmpm_oracle.so")
        L = self.lib
        L.oc_create.restype = ctypes.c_void_p
        L.oc_create.argtypes = [ctypes.c_int, _dp, _ip, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.oc_add_body.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, _ip, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oc_add_contact.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.oc_set_gravity.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp]
        L.oc_set_sand.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int]
        for fn in ("oc_step", "oc_num_nodes", "oc_get_point_field", "oc_get_node_field", "oc_get_contact_field",
                   "oc_map_size", "oc_grad_map_size", "oc_get_map", "oc_get_grad_map", "oc_build_map", "oc_destroy"):
            getattr(L, fn).argtypes = None
        Lx = np.array(list(case.L) + [0.0] * (3 - case.dim), dtype=np.float64)
        Nx = np.array(list(case.N) + [0] * (3 - case.dim), dtype=np.int32)
        h = L.oc_create(case.dim, _ptr(Lx), _ptr(Nx, _ip), case.dt, case.cpdi, case.contact_spec)
        if not h:
            raise RuntimeError("oracle allocation failed")
        self.h = ctypes.c_void_p(h)
        self.case = case
        self._keep = []
        from mpm_3d_b200.inputs import boundary_kind, material_kind, sand_params
        for bi, body in enumerate(case.bodies):
            arrs = [np.ascontiguousarray(body.m, np.float64), np.ascontiguousarray(body.v, np.float64),
                    np.ascontiguousarray(body.x, np.float64), np.ascontiguousarray(body.x_t, np.float64),
                    np.ascontiguousarray(body.active, np.int32)]
            L.oc_add_body(self.h, body.n, _ptr(arrs[0]), _ptr(arrs[1]), _ptr(arrs[2]), _ptr(arrs[3]),
                          _ptr(arrs[4], _ip), int(body.material), body.E, body.nu, boundary_kind(body),
                          float(body.boundary_mu), material_kind(body))
            if body.material and material_kind(body) == 2:
                props, density = sand_params(body)
                pa = np.array(props, dtype=np.float64)
                if L.oc_set_sand(self.h, bi, _ptr(pa), len(props), int(density)) != 0:
                    raise RuntimeError("oracle rejected the Sand_SachithLocal properties")
        for c in case.contacts:
            L.oc_add_contact(self.h, c.b1, c.b2, c.mu, int(getattr(c, "reflected", False)))
        if case.gravity is not None:
            g = np.array(list(case.gravity) + [0.0] * (3 - len(case.gravity)), dtype=np.float64)
            L.oc_set_gravity(self.h, 1, _ptr(g))
        self.nbodies = len(case.bodies)

    def close(self):
        if self.h is not None:
            self.lib.oc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        rc = self.lib.oc_step(self.h, ctypes.c_int(n))
        if rc != 0:
            raise RuntimeError("oracle step failed")

    def build_map(self):
        self.lib.oc_build_map(self.h)

    def n_points(self, b):
        return self.case.bodies[b].n

    def n_nodes(self, b=0):
        return self.lib.oc_num_nodes(self.h)

    def points(self, b, name):
        return self._field("get_point_field", b, name, self.n_points(b), 9)

    def nodes(self, b, name):
        return self._field("get_node_field", b, name, self.n_nodes(b), 3)

    def contact(self, c, name):
        return self._field("get_contact_field", c, name, self.n_nodes(0), 3)

    def map(self, b):
        n = self.lib.oc_map_size(self.h, b)
        node = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        val = np.zeros(n)
        self.lib.oc_get_map(self.h, b, _ptr(node, _ip), _ptr(pt, _ip), _ptr(val))
        return node, pt, val

    def grad_map(self, b):
        n = self.lib.oc_grad_map_size(self.h, b)
        node = np.zeros(n, np.int32)
        pt = np.zeros(n, np.int32)
        g = np.zeros((n, 3))
        self.lib.oc_get_grad_map(self.h, b, _ptr(node, _ip), _ptr(pt, _ip), _ptr(g))
        return node, pt, g


def build_restated(force: bool = False) -> Optional[str]:
    """Compiles oracle/mpm_oracle.c into oracle/_ref/libmpm_oracle.so."""
    import subprocess

    out = lib_path("libmpm_oracle.so")
    src = os.path.join(HERE, "mpm_oracle.c")
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    os.makedirs(REF_DIR, exist_ok=True)
    subprocess.check_call(["/usr/bin/gcc", "-std=c99", "-O3", "-ffp-contract=off", "-fPIC", "-shared", "-g", src,
                           "-lm", "-o", out])
    return out
