"""Failure detection without a GPU fault.

The reference stops the process on any error (stderr and exit(0);
include/signal_handler.hpp:15-31 on SIGINT); this library reports errors as
status codes instead. These tests make each failure happen in an allowed
form and check that it is reported and contained:

* a device-side wait that runs out: the fused kernel's waits for the bulk
  copies of a work item are bounded; with the bound set to zero the wait
  gives up at once, the kernel flags it, lets the copies in flight land and
  returns, and the step reports MPMGPU_ERR_DEVICE. The device stays usable:
  a new handle on it still matches the oracle;
* a serving request larger than the whole memory budget is rejected at
  submission (it could never run);
* a running request is cancelled between rounds; every other request's
  result is unchanged.
"""
import numpy as np
import pytest

import bridge
from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL, GPUServer, MpmGpuError
from util import FP64_TOL, assert_close, field_floor

pytestmark = pytest.mark.gpu

FIELDS = ["x", "x_t", "T", "u"]


def test_wait_that_runs_out_is_reported_and_contained():
    bridge.build_restated()
    case = inputs.block_drop_2d()   # the staged kernel, whose point arrays arrive by bulk copies
    sim = GPUExplicitUSL(case)
    sim.step(3)
    sim.synchronize()
    sim.set_wait_limit(0)
    sim.step(1)
    with pytest.raises(MpmGpuError, match="wait limit"):
        sim.synchronize()
    sim.close()
    # the context is intact: a new handle steps and matches the oracle
    sim = GPUExplicitUSL(case, keep_debug=True)
    ref = bridge.RestatedJob(case)
    sim.step(5)
    ref.step(5)
    sim.synchronize()
    for f in FIELDS:
        assert_close(sim.points(0, f), ref.points(0, f), FP64_TOL, f"after a timed-out handle: {f}",
                     field_floor(case, f))
    sim.close()


def test_request_larger_than_the_budget_is_rejected_at_submission():
    case = inputs.serving_case(inputs.serving_stream(rate=50.0, duration=0.2, seed=5, n_range=(16, 16),
                                                     steps_range=(10, 10))[0])
    probe = GPUServer(budget_bytes=1 << 40)
    fp = probe.footprint(case)
    probe.close()
    server = GPUServer(budget_bytes=fp - 1)
    assert server.submit(case, 10) == -1            # can never fit: rejected
    assert server.stats()["running"] == 0
    server.close()
    server = GPUServer(budget_bytes=fp)
    rid = server.submit(case, 10)
    assert rid is not None and rid >= 0             # fits exactly
    server.close()


def test_cancel_a_running_request_leaves_the_others_unchanged():
    specs = inputs.serving_stream(rate=100.0, duration=0.1, seed=23, n_range=(10, 14), steps_range=(30, 30),
                                  contact_frac=0.0)
    cases = [inputs.serving_case(s) for s in specs[:4]]
    assert len(cases) == 4

    def run(cancel):
        # the deterministic form: the same bits whatever else runs in the batch
        server = GPUServer(budget_bytes=1 << 40, mode="fp64_deterministic")
        rids = [server.submit(c, 30) for c in cases]
        assert all(r is not None and r >= 0 for r in rids)
        server.advance(10)
        if cancel:
            server.cancel(rids[1])
            st = server.request(rids[1])
            assert st["state"] == 5
            with pytest.raises(MpmGpuError):
                server.cancel(rids[1])       # no longer running
        out = {}
        for _ in range(6):
            server.advance(10)
            for rid in server.poll():
                out[rid] = [server.result(rid, 0, f) for f in FIELDS]
        assert rids[1] not in out if cancel else rids[1] in out
        server.close()
        return {i: out[r] for i, r in enumerate(rids) if r in out}

    base = run(False)
    cut = run(True)
    assert sorted(cut) == [0, 2, 3]
    for i in cut:
        for k, f in enumerate(FIELDS):
            assert np.array_equal(cut[i][k], base[i][k]), f"request {i} {f} changed by the cancel"
