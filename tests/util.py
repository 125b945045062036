"""Shared comparison helpers for the parity tests."""
import numpy as np

# Parity tolerance of the plain FP64 form against the oracle, per step and
# per field: max |gpu - ref| / max |ref| (summation order is the only
# source of difference).
FP64_TOL = 1e-10


def rel_err(got: np.ndarray, ref: np.ndarray) -> float:
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if got.shape != ref.shape:
        raise AssertionError(f"shape {got.shape} != {ref.shape}")
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    diff = float(np.max(np.abs(got - ref))) if ref.size else 0.0
    if scale == 0.0:
        return diff
    return diff / scale


def assert_close(got, ref, tol, what):
    e = rel_err(got, ref)
    assert e <= tol, f"{what}: relative error {e:.3e} > {tol:.1e}"
    return e


def bits_equal(a, b) -> bool:
    """Bitwise equality of two float arrays; NaNs match NaNs at the same
    positions (x86 and CUDA produce different NaN payloads for 0/0)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return bool(np.array_equal(a[~na].view(np.int64), b[~nb].view(np.int64)))
