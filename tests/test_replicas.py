"""Multi-rank host logic of the replicated solve (`sporco_cuda.replicas`),
run as two gloo ranks on the CPU: the job time is the slowest rank's, counts
are summed, the round-robin shard gives every image to exactly one rank."""

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from sporco_cuda import replicas
        r, w = replicas.world()
        ms = 100.0 + 50.0 * rank          # rank 1 is the slow one
        units = 10 * (rank + 1)           # 10 and 20 iterations
        res = {
            "world": (r, w),
            "max": replicas.max_over_ranks(ms),
            "sum": replicas.sum_over_ranks(units),
            "rate": replicas.job_rate(units, ms),
            "shard": replicas.shard(range(7)),
        }
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in range(world):
        res = got[rank]
        assert res["world"] == (rank, world)
        assert res["max"] == 150.0
        assert res["sum"] == 30.0
        assert res["rate"] == pytest.approx(30 / 0.150)
    shards = got[0]["shard"] + got[1]["shard"]
    assert sorted(shards) == list(range(7))
    assert got[0]["shard"] == [0, 2, 4, 6] and got[1]["shard"] == [1, 3, 5]


def test_single_process_defaults():
    from sporco_cuda import replicas
    assert replicas.world() == (0, 1)
    assert replicas.max_over_ranks(3.0) == 3.0
    assert replicas.job_rate(10, 100.0) == pytest.approx(100.0)
    assert replicas.shard([1, 2, 3]) == [1, 2, 3]
