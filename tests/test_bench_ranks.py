"""CPU: the multi-rank path of bench.py with two gloo ranks on 127.0.0.1.

`bench.py --gpus N` under torchrun runs one independent replica per rank (the
operator does not shard); the job's step time is the slowest rank's, taken
with one all-reduce(MAX) -- the only collective of the path.  The reference
arm runs on rank 0 alone; other ranks return without work.
"""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # rank r's replica: step 5 + r ms, e2e 7 - r ms
        got = bench.max_over_ranks([5.0 + rank, 7.0 - rank], world, "cpu")
        queue.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every rank sees the slowest rank's step and e2e times
    assert results[0] == results[1] == [6.0, 7.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:  # the arm must return before touching any of these on rank 1
        def __getattr__(self, name):
            raise AssertionError(f"rank 1 read args.{name}")

    bench.run_reference_arm(Args(), rank=1)
    assert capsys.readouterr().out == ""
