"""The replica (multi-rank) path of bench.py on the CPU: world size 2 over gloo.
Each rank takes a disjoint slice of the query stream per step, and the timed
totals are reduced to their maximum over the ranks."""
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slices = [bench.rank_slice(600, step, 32, rank, world) for step in range(4)]
        times = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist)
        out.put((rank, slices, times))
    finally:
        dist.destroy_process_group()


def test_two_ranks_disjoint_slices_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r, (sl, t)) for r, sl, t in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for step in range(4):
        a, b = set(res[0][0][step]), set(res[1][0][step])
        assert len(a) == len(b) == 32 and not (a & b)
    assert res[0][1] == res[1][1] == [2.0, 10.0]
