"""The C ABI library loads and exports every function include/mpm_b200.h
declares; argument errors come back as status codes (no GPU needed)."""
import ctypes
import os
import re

import pytest

from mpm_3d_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mpm_b200.h")).read()
    return sorted(set(re.findall(r"\b(mpmgpu_\w+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return native.load()


def test_header_declares_api():
    names = declared_functions()
    for required in ("mpmgpu_create", "mpmgpu_add_body", "mpmgpu_add_contact", "mpmgpu_set_gravity", "mpmgpu_step",
                     "mpmgpu_download_points", "mpmgpu_download_nodes", "mpmgpu_dump_map", "mpmgpu_destroy"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings(lib):
    for code, word in [(0, "ok"), (1, "invalid argument"), (2, "CUDA error"), (4, "unsupported")]:
        assert lib.mpmgpu_status_string(code).decode() == word


def test_invalid_configs_rejected_before_device_use(lib):
    cfg = native._Config()
    cfg.dim = 4
    cfg.dt = 1e-4
    h = ctypes.c_void_p()
    assert lib.mpmgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == 4
    cfg.dim = 3
    cfg.dt = 0.0
    assert lib.mpmgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    cfg.dt = 1e-4
    cfg.N[0] = 0
    assert lib.mpmgpu_create(ctypes.byref(cfg), ctypes.byref(h)) == 1
    assert lib.mpmgpu_create(None, ctypes.byref(h)) == 1


def test_null_handle_calls_are_argument_errors(lib):
    assert lib.mpmgpu_step(None, 1) == 1
    assert lib.mpmgpu_synchronize(None) == 1
    assert lib.mpmgpu_destroy(None) == 0
    assert lib.mpmgpu_launch_count(None) == 0
