"""Multi-rank plumbing on CPU (gloo, world size 2): frames shard across ranks with
no data-path collective; timing takes the max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mvs_b200 import dist


def test_shard_covers_all_items_once():
    for n in [0, 1, 7, 48, 49]:
        for ws in [1, 2, 3, 8]:
            got = [i for r in range(ws) for i in dist.shard(n, r, ws)]
            assert got == list(range(n))
            sizes = [len(dist.shard(n, r, ws)) for r in range(ws)]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    r, w = dist.init("gloo")
    items = list(dist.shard(5, r, w))
    dist.barrier()
    t = dist.max_over_ranks(1.0 + r)
    total = dist.sum_over_ranks(len(items))
    dist.finish()
    q.put((r, items, t, total))


def test_two_rank_gloo_sharding_and_max_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][1] == [0, 1, 2] and out[1][1] == [3, 4]
    assert all(o[2] == 2.0 for o in out)
    assert all(o[3] == 5 for o in out)
