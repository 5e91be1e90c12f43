"""The N > 1 path of bench.py on CPU: two gloo ranks (world_size 2).

bench.py --gpus N runs one rank per GPU as replicas: every rank evaluates its
own K states on the same geometry, with no data-path collective; the job's
step time is the max over ranks and the value is the units all ranks
processed divided by it.  These tests run that host logic with the gloo
backend on 127.0.0.1 (no GPU): the max-over-ranks reduction, distinct
per-rank moment seeds, the aggregate rate, and that the reference arm prints
only on rank 0.
"""

import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        my_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.reduce_max_over_ranks(my_ms, dist, "cpu")
        seed = bench.rank_moment_seed(314159, rank)
        rate = bench.whole_job_rate(1000, world, ms)
        seeds = [None] * world
        dist.all_gather_object(seeds, seed)
        out.put((rank, ms, rate, seeds))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_step_time_and_aggregate():
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    port = _free_port()
    q = mp.Queue()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate, seeds in results:
        assert ms == 15.0                       # max over ranks
        assert rate == pytest.approx(2 * 1000 / 15e-3)
        assert len(set(seeds)) == 2             # each rank its own states
    assert results[0][3] == results[1][3]


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    args = bench.parse_args()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.reference_arm(args)
    assert buf.getvalue() == ""
