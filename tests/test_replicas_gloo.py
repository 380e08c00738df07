"""The multi-GPU harness of bench.py on CPU: replicas only, so the one collective
is the max-over-ranks reduction of the step time; world_size 2 over gloo."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
    got = bench._max_over_ranks(dist, torch, torch.device("cpu"), ms)
    # the reference arm runs on rank 0 only; the others return nothing
    class A:
        config = "c4"
    ref = bench.run_reference(A(), {}, rank, world)
    out.put((rank, got, ref))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2]["impl"] == "reference" and "unavailable" in res[0][2]
    assert res[1][2] is None


def test_single_process_needs_no_group():
    import bench
    assert bench._max_over_ranks(None, torch, torch.device("cpu"), 3.5) == 3.5
    assert bench._init_dist(1) is None
