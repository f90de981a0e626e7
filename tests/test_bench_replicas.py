"""bench.py's multi-GPU bookkeeping on CPU: two gloo ranks stand in for two
GPUs.  Each replica reports its own device time; the job takes the slowest
rank's time (max over ranks) and the whole-job rate counts every replica's
cells."""
import importlib.util
import os
import socket

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(REPO, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        b = _bench()
        ms = [10.0, 12.5][rank]           # this replica's device time for the timed steps
        b.barrier(dist, 0)
        mx = b.reduce_max(dist, ms, 0)
        out.put((rank, mx, b.whole_job_rate(1000, 4, world, mx)))
        b.barrier(dist, 0)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_replicas_take_max_over_ranks():
    torch = pytest.importorskip("torch")
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, rate in res:
        assert mx == 12.5
        # 2 replicas x 1000 cells x 4 steps in 12.5 ms
        assert rate == pytest.approx(2 * 1000 * 4 / 12.5e-3)
