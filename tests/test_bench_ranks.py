"""The multi-rank host logic of bench.py on CPU: two gloo ranks reduce their timings (max)
and counts (sum), and draw disjoint, reproducible shards of the batched droplet solves."""
import datetime
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, ROOT)
        import bench

        mx = bench.max_over_ranks(1.5 + rank, world)
        sm = bench.sum_over_ranks(10.0 * (rank + 1), world)
        shard = [(d["N"], d["c3"], d["n"]) for d in bench.batch_solves(8, rank=rank)]
        q.put((rank, mx, sm, shard))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_shard():
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            rank, mx, sm, shard = q.get(timeout=120)
            out[rank] = (mx, sm, shard)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert out[0][0] == out[1][0] == 2.5
    assert out[0][1] == out[1][1] == 30.0
    s0, s1 = out[0][2], out[1][2]
    assert len(s0) == len(s1) == 8 and not set(s0) & set(s1)
    sys.path.insert(0, ROOT)
    import bench

    assert s0 == [(d["N"], d["c3"], d["n"]) for d in bench.batch_solves(8, rank=0)]
    assert all(20 <= N <= 2000 and -3.2 <= c3 <= -2.8 and n in (32, 64, 128) for N, c3, n in s0 + s1)


def test_single_rank_reductions_are_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, 1) == 3.25 and bench.sum_over_ranks(7.0, 1) == 7.0
