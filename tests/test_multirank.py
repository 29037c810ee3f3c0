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


# ---------------------------------------------------------------------------
# zfind with a communicator: each rank scans and refines its own targets,
# rank 0 gathers and finalises (redrock zfind.py:416-456).  The GPU stages
# are replaced by deterministic stand-ins here, so this checks the host
# plumbing on CPU: sharding, the collective calls every rank makes, the
# gather and the finalised table against a one-process run.
# ---------------------------------------------------------------------------
class _Tmpl:
    def __init__(self, spectype, subtype, nb, z):
        self.template_type = spectype
        self._rrtype = spectype
        self.sub_type = subtype
        self.full_type = spectype if not subtype else f"{spectype}:::{subtype}"
        self.nbasis = nb
        self.redshifts = z
        self.method = "PCA"


class _DT:
    def __init__(self, tm):
        self.template = tm


def _fake_scan(targets, templates, mp_procs=1):
    import numpy as np
    out = {}
    for t in targets.local():
        out[t.id] = {}
        for dt in templates:
            z = dt.template.redshifts
            rng = np.random.default_rng(int(t.id) * 7 + len(dt.template.full_type))
            out[t.id][dt.template.full_type] = dict(
                redshifts=z, zchi2=rng.uniform(100, 200, len(z)), penalty=np.zeros(len(z)),
                zcoeff=rng.normal(size=(len(z), dt.template.nbasis)))
    return out


def _fake_fitz(chi2_list, redshifts, targets, template, nminima=3, **kw):
    import numpy as np
    out = []
    for c, t in zip(chi2_list, targets):
        ii = np.argsort(c)[:nminima]
        n = len(ii)
        out.append(dict(z=redshifts[ii][:, None], zerr=np.full((n, 1), 1e-4),
                        zwarn=np.zeros((n, 1), dtype=int), chi2=c[ii][:, None],
                        zz=np.tile(redshifts[:3], (n, 1)), zzchi2=np.tile(c[:3], (n, 1)),
                        coeff=np.ones((n, template.nbasis)) * t.id,
                        fitmethod=np.full((n, 1), "PCA"),
                        npixels=np.full((n, 1), sum(len(s.wave) for s in t.spectra))))
    return out


def _zfind_worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from redrock_b200 import synth, zfind as Z
        from redrock_b200.shard import TorchComm
        from redrock_b200.targets import DistTargetsCopy, from_synth
        Z.calc_zchi2_targets = _fake_scan
        Z._fitz.fitz_targets = _fake_fitz
        Z.GridLayout = type("L", (), {"from_dwave": staticmethod(lambda d: None)})
        Z.RowPack = type("R", (), {"from_targets": staticmethod(lambda t, l: None)})
        tg = from_synth(synth.make_targets(7, seed=6, drop_camera_frac=0.3))
        tmpls = [_DT(_Tmpl("GALAXY", "", 4, np.linspace(0.1, 1.0, 40))),
                 _DT(_Tmpl("STAR", "K", 3, np.linspace(-0.001, 0.001, 20)))]
        comm = TorchComm()
        dtg = DistTargetsCopy(tg, comm=comm)
        local_ids = list(dtg.local_target_ids())
        allres, allzfit = Z.zfind(dtg, tmpls, nminima=3)
        single = None
        if rank == 0:
            single = Z.zfind(DistTargetsCopy(tg), tmpls, nminima=3)[1]
        # one target for two ranks: rank 1 has none, and still makes every
        # collective call
        one = DistTargetsCopy(tg[:1], comm=comm)
        _, zf1 = Z.zfind(one, tmpls, nminima=3)
        n1 = None if zf1 is None else len(zf1["targetid"])
        q.put((rank, local_ids, allzfit, single, None if allres is None else sorted(allres),
               len(one.local_target_ids()), n1))
    finally:
        dist.destroy_process_group()


def test_two_rank_zfind_gathers_on_rank0():
    import numpy as np
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_zfind_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        r, ids, zf, single, keys, nlocal1, n1 = q.get(timeout=180)
        out[r] = (ids, zf, single, keys, nlocal1, n1)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ids0, ids1 = out[0][0], out[1][0]
    assert ids0 and ids1 and set(ids0).isdisjoint(ids1) and len(ids0) + len(ids1) == 7
    assert out[1][1] is None and out[1][3] is None
    zf, single = out[0][1], out[0][2]
    assert out[0][3] == sorted(ids0 + ids1)
    assert list(zf.keys()) == list(single.keys())
    for k in zf:
        np.testing.assert_array_equal(zf[k], single[k], err_msg=k)
    assert out[0][4] + out[1][4] == 1 and min(out[0][4], out[1][4]) == 0
    assert out[0][5] == 6 and out[1][5] is None   # 3 minima x 2 templates
