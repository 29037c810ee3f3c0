"""World-size-2 gloo run of the multi-rank host logic (sharding, max over
ranks, result gather).  CPU only; the scan itself needs no collective."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from redrock_b200 import synth
        from redrock_b200.shard import gather_results, max_over_ranks, shard_targets
        from redrock_b200.targets import from_synth
        tg = from_synth(synth.make_targets(9, seed=4, drop_camera_frac=0.3))
        mine = shard_targets(tg, world, rank)
        t = max_over_ranks([1.0 + rank, 10.0 - rank])
        res = gather_results({x.id: rank for x in mine})
        q.put((rank, [x.id for x in mine], t, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_reduce_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, ids, t, res = q.get(timeout=120)
        out[r] = (ids, t, res)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids0, ids1 = out[0][0], out[1][0]
    assert set(ids0).isdisjoint(ids1) and len(ids0) + len(ids1) == 9
    assert abs(len(ids0) - len(ids1)) <= 2
    assert out[0][1] == [2.0, 10.0] and out[1][1] == [2.0, 10.0]
    merged = out[0][2]
    assert out[1][2] is None and sorted(merged) == sorted(ids0 + ids1)
    assert all(merged[i] == 0 for i in ids0) and all(merged[i] == 1 for i in ids1)
