"""The benchmark's multi-GPU path is N independent replicas (one structure
per rank, no collective on the data path): its only collectives are the
barrier and the maximum of the ranks' step times.  Two gloo ranks on the CPU
check that every rank gets the slowest rank's time and that the whole-job
value counts all ranks' grid points over it."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
    got = bench.rank_max(ms, dist, torch.device("cpu"))
    dist.barrier()
    q.put((rank, got, bench.replica_value(1_000_000, world, got)))
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    import multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict((r, (ms, v)) for r, ms, v in (q.get(timeout=120) for _ in ps))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][0] == res[1][0] == 15.0
    # 2 ranks x 1 M grid points in 15 ms: 133.3 M grid points per second.
    assert abs(res[0][1] - 2e6 / 0.015 / 1e6) < 1e-9


def test_single_rank_is_its_own_maximum():
    sys.path.insert(0, ROOT)
    import torch
    import bench
    assert bench.rank_max(3.5, None, torch.device("cpu")) == 3.5
    assert bench.replica_value(2_000_000, 1, 4.0) == 500.0
