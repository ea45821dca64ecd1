"""bench.py's multi-GPU host logic (one independent replica per rank, the
timed region's length taken as the max over ranks) on two CPU processes
with the gloo backend: the same calls the torchrun launch makes, without a
GPU."""
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


def _rank(rank, ws, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(ws), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    w, r, local = bench.dist_init("gloo")
    try:
        # rank r "took" 10 + 5 r ms for 1000 units
        rate, ms = bench.job_rate(1000, 10.0 + 5.0 * r, w)
        bench.barrier(w)
        out.put((r, w, local, rate, ms))
    finally:
        dist.destroy_process_group()


def test_replica_rate_uses_slowest_rank():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 and x[2] == x[0] for x in res)
    # every rank reports the job: 2 x 1000 units in the slowest rank's 15 ms
    for _, _, _, rate, ms in res:
        assert ms == pytest.approx(15.0)
        assert rate == pytest.approx(2 * 1000 / 15e-3)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.job_rate(500, 20.0, 1) == (pytest.approx(500 / 20e-3), 20.0)
