"""Host logic of `bench.py --gpus N` (replicas, one process per GPU) on CPU:
two `gloo` ranks reduce their timings to the slowest one and compute the
whole-job value the same way; rank discovery from the torchrun variables."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, local, w = bench.env_rank()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        ms = 10.0 + 5.0 * rank                    # rank 1 is the slowest
        t = bench.max_over_ranks(ms, dist, "cpu")
        e = bench.max_over_ranks(1.0 + rank, dist, "cpu")
        q.put((r, local, w, t, e, bench.replica_value(w, 4096.0 * 4096.0, 20, t / 1e3)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, local, world, t, e, v) in enumerate(out):
        assert (rank, local, world) == (r, r, 2)
        assert t == 15.0 and e == 2.0          # the max over ranks, on every rank
        assert v == pytest.approx(2 * 4096 * 4096 * 20 / 0.015)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert bench.replica_value(1, 100.0, 10, 2.0) == 500.0
