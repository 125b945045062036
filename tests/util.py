"""Shared comparison helpers for the parity tests."""
import numpy as np

# Parity tolerance of the plain FP64 form against the oracle, per step and
# per field: max |gpu - ref| / max |ref| (summation order is the only
# source of difference).
FP64_TOL = 1e-10


def rel_err(got: np.ndarray, ref: np.ndarray, floor: float = 0.0) -> float:
    """max |got - ref| / max(max |ref|, floor).

    ``floor`` is the field's physical scale for fields that can be pure
    round-off in the reference (the stress and velocity gradient of a block
    in free fall are ~1e-12 noise): differences far below that scale are
    summation-order noise, not disagreement.
    """
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if got.shape != ref.shape:
        raise AssertionError(f"shape {got.shape} != {ref.shape}")
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    scale = max(scale, floor)
    diff = float(np.max(np.abs(got - ref))) if ref.size else 0.0
    if scale == 0.0:
        return diff
    return diff / scale


def assert_close(got, ref, tol, what, floor: float = 0.0):
    e = rel_err(got, ref, floor)
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


def field_floor(case, field: str) -> float:
    """Physical scale of a field for ``rel_err``: the velocity scale is the
    largest initial speed (at least 1 m/s); the velocity-gradient scale is
    that speed over a cell; the stress scale is one step of elastic stress
    at that gradient (E * dt * v / h); a plastic shear rate (gammap_dot)
    has the gradient's scale and a plastic strain (gammap) one step of it."""
    v0 = max(1.0, max(float(np.abs(b.x_t).max()) for b in case.bodies))
    h = min(case.h)
    E = max(b.E for b in case.bodies)
    return {"L": v0 / h, "T": E * case.dt * v0 / h, "x_t": v0, "u": h, "x": min(case.L), "gammap_dot": v0 / h,
            "gammap": case.dt * v0 / h}.get(field, 0.0)
