"""Host logic of the multi-GPU bench on CPU: two gloo ranks reduce the
timing (max over ranks) and the work (sum over ranks) as the NCCL ranks do."""
import multiprocessing as mp
import os
import socket


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms, value = bench.aggregate_throughput(10.0 + rank, 100.0 * (rank + 1), world)
        bench.barrier(world)
        q.put((rank, ms, value, bench.max_over_ranks(float(rank), world)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value, mx in got:
        assert ms == 11.0 and mx == 1.0
        assert abs(value - 300.0 / 11e-3) < 1e-6 * value


def test_single_rank_is_local():
    import bench
    assert bench.aggregate_throughput(5.0, 50.0, 1) == (5.0, 50.0 / 5e-3)
