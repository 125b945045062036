"""The allocation-free map export, mpmgpu_dump_map_noalloc.

Callers that cannot allocate device memory at the point of the call
(frameworks that own all device memory through their own pools, real-time
loops that forbid cudaMalloc after set-up) read the S / gradS triplets
through this entry point: it keeps its scratch in a static device array of
the library and writes into device arrays the caller already owns. This test
owns those arrays (allocated here with torch), calls the entry point through
the C ABI twice in a row (at the initial positions and after some steps, so
the second call reuses scratch the first call left behind), and checks each
result against the allocating entry point mpmgpu_dump_map, bit for bit, and
that the second call leaves the device's free memory unchanged. It also
checks that a body above the static scratch limit is rejected with an error
instead of being served, and that a call while the handle's stream is being
captured into a CUDA graph is refused without breaking the capture.

The file name makes pytest collect it last, so a run that stops at the first
failure has already run every other test.
"""
import numpy as np
import pytest

from mpm_3d_b200 import inputs
from mpm_3d_b200.native import GPUExplicitUSL, MpmGpuError
from util import bits_equal

pytestmark = pytest.mark.gpu


def _device_buffers(torch, capacity):
    return (torch.empty(capacity, dtype=torch.int32, device="cuda"),
            torch.empty(capacity, dtype=torch.int32, device="cuda"),
            torch.empty(capacity, dtype=torch.float64, device="cuda"),
            torch.empty(3 * capacity, dtype=torch.float64, device="cuda"))


def _noalloc_map(sim, body, bufs, capacity):
    node, pt, s, g = bufs
    n = sim.map_noalloc(body, node.data_ptr(), pt.data_ptr(), s.data_ptr(), g.data_ptr(), capacity)
    return (node[:n].cpu().numpy(), pt[:n].cpu().numpy(), s[:n].cpu().numpy(),
            g[:3 * n].cpu().numpy().reshape(n, 3))


@pytest.mark.parametrize("make", [lambda: inputs.two_body_collision_3d(16, steps=6, gap=0.01),
                                  lambda: inputs.two_body_collision_2d(20, steps=6)],
                         ids=["collision_3d", "collision_2d"])
def test_noalloc_map_matches_allocating_export(make):
    torch = pytest.importorskip("torch")
    case = make()
    sim = GPUExplicitUSL(case)
    capacity = max(b.n for b in case.bodies) * (1 << case.dim) ** 2
    bufs = _device_buffers(torch, capacity)
    for call in range(2):
        if call == 1:
            sim.step(5)
        for b in range(len(case.bodies)):
            want = sim.map(b)
            got = _noalloc_map(sim, b, bufs, capacity)
            assert len(got[0]) == len(want[0]) > 0
            assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
            assert bits_equal(got[2], want[2]) and bits_equal(got[3], want[3])
    sim.close()


def test_noalloc_map_rejects_bodies_above_the_scratch_limit():
    torch = pytest.importorskip("torch")
    case = inputs.two_body_collision_3d(48, steps=1)  # 13,824 points x 64 slots per body > 524,288
    sim = GPUExplicitUSL(case)
    bufs = _device_buffers(torch, 16)
    with pytest.raises(MpmGpuError, match="static scratch limit"):
        _noalloc_map(sim, 0, bufs, 16)
    sim.close()


def test_noalloc_map_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    # 8,000 points per body: 512,000 slots, just under the scratch limit, so
    # that slot buffers taken from cudaMalloc (about 18 MB) would show
    case = inputs.two_body_collision_3d(40, steps=2, gap=0.01)
    sim = GPUExplicitUSL(case)
    capacity = max(b.n for b in case.bodies) * 64
    assert capacity <= 1 << 19
    bufs = _device_buffers(torch, capacity)
    want = sim.map(0)
    first = _noalloc_map(sim, 0, bufs, capacity)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    node, pt, s_, g = bufs
    n = sim.map_noalloc(0, node.data_ptr(), pt.data_ptr(), s_.data_ptr(), g.data_ptr(), capacity)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    assert n == len(want[0]) == len(first[0])
    assert np.array_equal(node[:n].cpu().numpy(), want[0]) and bits_equal(s_[:n].cpu().numpy(), want[2])
    sim.close()


def test_noalloc_map_refuses_a_captured_stream():
    torch = pytest.importorskip("torch")
    case = inputs.two_body_collision_3d(16, steps=2, gap=0.01)
    sim = GPUExplicitUSL(case)
    capacity = max(b.n for b in case.bodies) * 64
    bufs = _device_buffers(torch, capacity)
    want = _noalloc_map(sim, 0, bufs, capacity)
    stream = torch.cuda.ExternalStream(sim.stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        graph.capture_begin()
        try:
            with pytest.raises(MpmGpuError, match="captured"):
                _noalloc_map(sim, 0, bufs, capacity)
        finally:
            graph.capture_end()   # the capture is still valid: it ends without an error
    del graph
    # and the handle still serves the call once the capture is over
    got = _noalloc_map(sim, 0, bufs, capacity)
    assert np.array_equal(got[0], want[0]) and bits_equal(got[2], want[2])
    sim.close()
