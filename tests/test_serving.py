"""Serving (mpmgpu_server_*): requests that arrive while others run are
admitted under a memory budget, step together with them and leave when
done; each result equals the same request run alone, within the form's
tolerance (FP64: 1e-10, util.py; mixed: 1e-4)."""
import pytest

from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL, GPUServer
from mpm_3d_b200.serving import run_stream
from util import FP64_TOL, field_floor, rel_err

pytestmark = pytest.mark.gpu

FIELDS = ["x", "x_t", "T", "u"]


def _alone(case, steps, mode):
    sim = GPUExplicitUSL(case, mode=mode)
    sim.step(steps)
    out = [{f: sim.points(b, f) for f in FIELDS} for b in range(len(case.bodies))]
    sim.close()
    return out


@pytest.mark.parametrize("mode,tol", [("fp64", FP64_TOL), ("mixed", 1e-4)])
def test_each_result_is_the_same_alone_and_in_the_mix(mode, tol):
    specs = inputs.serving_stream(rate=60.0, duration=0.25, seed=21, n_range=(8, 16), steps_range=(10, 60),
                                  contact_frac=0.3)
    assert len(specs) >= 8
    # a budget of about three requests: later arrivals queue, then join
    # while earlier ones are still stepping
    server = GPUServer(budget_bytes=1 << 40, mode=mode)
    fp = max(server.footprint(inputs.serving_case(s)) for s in specs)
    server.close()
    server = GPUServer(budget_bytes=3 * fp, mode=mode)
    got = {}

    def keep(c):
        case = server.cases[c.rid]
        got[c.spec.index] = (case, [{f: server.result(c.rid, b, f) for f in FIELDS} for b in range(len(case.bodies))])

    rep = run_stream(server, specs, round_steps=7, on_complete=keep)
    assert len(rep.completed) == len(specs)
    assert rep.max_running >= 2          # requests overlapped on the device
    for spec in specs:
        case, res = got[spec.index]
        ref = _alone(case, spec.steps, mode)
        for b in range(len(case.bodies)):
            for f in FIELDS:
                e = rel_err(res[b][f], ref[b][f], field_floor(case, f))
                assert e <= tol, f"request {spec.index} ({case.name}) body {b} {f}: {e:.3e}"
    server.close()
