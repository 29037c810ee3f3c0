"""zfind with a communicator on the GPU: two ranks (processes) each scan and
refine their own shard of the targets on cuda:0 -- their kernels are
independent, so sharing one GPU is fine -- and rank 0 gathers and finalises.
The gathered table must equal the one-process zfind bit for bit (every
per-target computation is the same; only the process that runs it
differs).  Objects travel over a gloo group (redrock_b200.shard.TorchComm)."""
import os
import socket

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    from redrock_b200 import synth
    tg = synth.make_targets(9, seed=43, amp=2.0, drop_camera_frac=0.2, first_id=7000)
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4}
    tset = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            tset.append(ts)
    return tg, tset


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        from redrock_b200 import targets as T, templates as TM
        from redrock_b200.shard import TorchComm
        from redrock_b200.zfind import zfind
        tg, tset = _inputs()
        comm = TorchComm()
        dtg = T.DistTargetsCopy(T.from_synth(tg), comm=comm)
        dwave = dtg.wavegrids()
        dts = [TM.DistTemplate(TM.from_synth(ts), dwave, comm=comm) for ts in tset]
        ids = list(dtg.local_target_ids())
        _, zfit = zfind(dtg, dts, nminima=3)
        q.put((rank, ids, zfit))
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_equal_one_process():
    import torch.multiprocessing as mp
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.zfind import zfind
    tg, tset = _inputs()
    dtg = T.DistTargetsCopy(T.from_synth(tg))
    dts = [TM.DistTemplate(TM.from_synth(ts), dtg.wavegrids()) for ts in tset]
    _, ref = zfind(dtg, dts, nminima=3)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, ids, zf = q.get(timeout=600)
        out[r] = (ids, zf)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0][0] and out[1][0] and set(out[0][0]).isdisjoint(out[1][0])
    assert out[1][1] is None
    zf = out[0][1]
    assert list(zf.keys()) == list(ref.keys())
    for k in zf:
        np.testing.assert_array_equal(zf[k], ref[k], err_msg=k)
