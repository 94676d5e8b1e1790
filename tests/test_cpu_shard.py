"""Block sharding on CPU: the shard plan (Z order, contiguous ranges, halo
blocks, exchange lists) and one halo exchange over two and three gloo ranks.

The reference partitions its ordered leaf list into contiguous ranges, one
per MPI rank (src/FFV/Solver.cpp:306-381), and exchanges guide faces between
ranks.  Here every rank must end an exchange holding, in each halo block,
exactly the owner's interior of that block, so that the unchanged in-kernel
exchange sees the unsharded grid's neighbours.
"""
import ctypes
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

import ffvgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("ranks", [1, 2, 3, 4])
def test_shard_plan_partitions_and_lists(ranks):
    g = ffvgpu.SphereGrid(3)
    d = g.desc()
    nbr = np.zeros((g.nb, 6), np.int32)
    ids = np.zeros((g.nb, 6, 4), np.int32)
    ffvgpu.lib().ffvgpu_grid_neighbors(d, nbr.ctypes.data, ids.ctypes.data)
    shards = [ffvgpu.Shard(d, ranks, r) for r in range(ranks)]
    z = shards[0].zorder
    assert sorted(z.tolist()) == list(range(g.nb))
    sizes = [s.owned for s in shards]
    assert sum(sizes) == g.nb and max(sizes) - min(sizes) <= 1
    start = 0
    for r, S in enumerate(shards):
        # owned: the r-th contiguous range of the Z order, in Z order
        assert S.local[:S.owned].tolist() == z[start:start + S.owned].tolist()
        assert (S.owner[S.local[:S.owned]] == r).all()
        start += S.owned
        # halo: exactly the other ranks' face neighbours of owned blocks
        need = set()
        for b in S.local[:S.owned]:
            for f in range(6):
                k = nbr[b, f]
                n = 4 if k == 3 else (0 if k == 0 else 1)
                need |= {int(x) for x in ids[b, f, :n] if S.owner[x] != r}
        assert set(S.local[S.owned:].tolist()) == need
        # the local description's table maps owned blocks' neighbours to local ids
        ld = S.desc()
        assert ld.num_blocks == S.owned + S.halo
        i32p = ctypes.POINTER(ctypes.c_int32)
        kind = np.ctypeslib.as_array(ctypes.cast(ld.neighbor_kind, i32p),
                                     shape=(ld.num_blocks * 6,)).reshape(-1, 6)
        lid = np.ctypeslib.as_array(ctypes.cast(ld.neighbor_ids, i32p),
                                    shape=(ld.num_blocks * 24,)).reshape(-1, 6, 4)
        for l in range(S.owned):
            b = S.local[l]
            assert (kind[l] == nbr[b]).all()
            for f in range(6):
                n = 4 if nbr[b, f] == 3 else (0 if nbr[b, f] == 0 else 1)
                assert (S.local[lid[l, f, :n]] == ids[b, f, :n]).all()
        assert (kind[S.owned:] == 0).all()
    # what r sends to p is what p receives from r, in the same order
    for r, S in enumerate(shards):
        for p, T in enumerate(shards):
            if p == r:
                continue
            assert (S.local[S.send[p]] == T.local[T.recv[r]]).all()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    sys.path.insert(0, os.path.join(ROOT, "ffv-hc_b200"))
    import torch
    import torch.distributed as dist
    import ffvgpu as fg
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    g = fg.SphereGrid(3)
    S = fg.Shard(g.desc(), world, rank)
    xg = np.random.default_rng(11).standard_normal((g.nb, 4096))  # the same on every rank
    x = torch.zeros((S.owned + S.halo, 4096), dtype=torch.float64)
    x[:S.owned] = torch.from_numpy(xg[S.local[:S.owned]])
    fg.halo_exchange(dist, S, x)
    ok = bool(np.array_equal(x.numpy(), xg[S.local]))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, ok, S.halo))


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_over_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert all(ok for _, ok, _ in got), got
    assert all(h > 0 for _, _, h in got)
