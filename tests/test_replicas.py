"""The multi-process (replicas) path of bench.py on CPU: two gloo ranks at 127.0.0.1.

bench.py --gpus N runs N independent replicas; the only cross-rank steps are the barrier
and the reduction of the timed results (slowest rank's time, summed pairs), and only rank
0 prints.  This checks those host-side steps without a GPU.
"""
import datetime
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        out = bench.reduce_over_ranks(100.0 + 10 * rank, 200.0 - rank, 200, 200 + rank)

        class Args:
            workload, steps, warmup = "c2", 1, 0

        buf = io.StringIO()
        if rank != 0:  # a non-zero rank of the reference arm returns without work or output
            with redirect_stdout(buf):
                bench.run_reference(Args, rank, world)
        q.put((rank, out, buf.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, out, printed in res:
        assert out == (110.0, 200.0, 400, 401)  # max of times, sum of pairs, on every rank
        assert printed == ""
