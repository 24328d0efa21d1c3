"""The multi-GPU form is N independent replicas (no collective on the data
path); the bench's cross-rank steps are the max over ranks of the device time
and the whole-job rate.  Checked here with 2 gloo ranks on the CPU."""
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


def _rank(rank, world, port, q):
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w, r, lr = bench.dist_setup()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, True, torch.device("cpu"))
        dist.barrier()
        q.put((r, w, ms, bench.whole_job_rate(w, 1_000_000, ms)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(90)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[0] for g in got] == [0, 1] and all(g[1] == 2 for g in got)
    assert all(g[2] == 15.0 for g in got)                     # max over ranks
    assert all(abs(g[3] - 2 * 1_000_000 / 15e-3) < 1e-6 for g in got)


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.5, False, None) == 3.5
    assert bench.whole_job_rate(1, 100, 1.0) == 100_000.0
