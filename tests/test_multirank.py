"""Host side of the N > 1 benchmark path on CPU: two gloo ranks, as torchrun
would start them on two GPUs. Each rank runs its own share of the work (the
ensemble with its own seed; no data crosses ranks); the timing is the
slowest rank's and the points are summed over ranks."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist

    r, w, local = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(w)
        slowest = bench.max_over_ranks(10.0 * (r + 1), w)
        points = bench.sum_over_ranks(1000.0 + r, w)
        # the ensemble of each rank is drawn from its own seed
        first = bench.make_workload("ensemble", r)[0]
        out.put((r, w, slowest, points, first.N[0], first.n_points))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_draw_their_own_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1]
    for r, w, slowest, points, n0, np0 in res:
        assert w == 2
        assert slowest == 20.0          # the slowest rank's time
        assert points == 2001.0         # points of both ranks
    # different seeds per rank: different first jobs
    assert (res[0][4], res[0][5]) != (res[1][4], res[1][5])
