"""The replica form's host logic on two gloo ranks (CPU): every rank takes its own seeded stream and
the job reports each latency as the maximum over ranks."""
import os
import socket

import torch.multiprocessing as mp


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        got = bench.max_over_ranks([float(rank), 10.0 - rank, 3.5], dist, device="cpu")
        import svdag.workloads as w

        times, edits, _ = w.c4_stream(500.0, 0.05, seed=4 + rank, levels=12, terrain=w.C0_TERRAIN, rmax=64.0, copy_offset=32)
        q.put((rank, got, len(edits), [tuple(e.center) for e in edits[:3]]))
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] == [1.0, 10.0, 3.5]
    assert res[0][3] != res[1][3]  # each replica replays its own stream
