"""The multi-rank path of bench.py on CPU: two gloo ranks on 127.0.0.1, the
max-over-ranks timing and the whole-job rate its JSON line reports; and a
rank whose peer never joins ends with an error (short timeout), not a hang."""
import datetime
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    ms = [12.5, 40.0][rank]  # rank 1 is the slow one
    worst = bench.max_over_ranks(ms, dist, "cpu")
    rate = bench.whole_job_rate(world, 1e9, worst)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, worst, rate))


def test_two_gloo_ranks_report_the_slowest_rank_and_the_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for _, worst, rate in got:
        assert worst == 40.0                                   # max over ranks, on every rank
        assert rate == pytest.approx(2 * 1e9 / 0.040 / 1e9)   # both ranks' units / slowest time


def _lonely(port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    try:
        dist.init_process_group("gloo", rank=0, world_size=2,
                                timeout=datetime.timedelta(seconds=3))
        q.put("joined")
    except Exception as e:  # the peer never comes: an error, not a hang
        q.put(type(e).__name__)


def test_a_rank_whose_peer_never_joins_gets_an_error_not_a_hang():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_free_port(), q))
    p.start()
    p.join(timeout=120)
    assert p.exitcode == 0
    assert q.get(timeout=10) != "joined"
