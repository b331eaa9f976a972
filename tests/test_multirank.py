"""The N-GPU host logic of bench.py on CPU: two ranks over gloo (127.0.0.1).
Every rank holds the same scene replica and traces its own seeded rays; the
timed value is the slowest rank's time (an all-reduce MAX) and the job's
throughput counts all ranks' rays; the reference arm runs on rank 0 alone."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import torch.distributed as dist
    from datetime import timedelta

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    ms = bench.max_over_ranks(1.5 + rank, world, "cpu")
    tris, rays = bench.make_workload(rank, n_tris=512, n_rays=1024)
    out.put((rank, ms, tris.sum(dtype=np.float64), rays[:, [0, 1, 2, 4, 5, 6]].sum(dtype=np.float64)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_their_own_rays():
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
    (r0, ms0, t0, y0), (r1, ms1, t1, y1) = res
    assert ms0 == ms1 == 2.5          # the max over ranks, on every rank
    assert t0 == t1                   # one scene replica on every rank
    assert y0 != y1                   # each rank its own rays


def test_single_rank_time_is_its_own():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference_arm(None)  # other ranks exit without work or output
    assert buf.getvalue() == ""
