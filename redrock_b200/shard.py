"""Multi-GPU plumbing for the scan: one process per GPU, targets sharded.

Targets are independent units (redrock distributes them over MPI ranks with
``distribute_work``, utils.py:185-227, and GPU ranks rebin all redshifts,
templates.py:558-563); the scan needs no collective.  The only cross-rank
steps are the max-over-ranks timing reduction and the final gather of
per-target results to rank 0 (redrock's zfind.py:416-454), both through
torch.distributed (NCCL on GPUs, gloo on CPUs).
"""

from __future__ import annotations

import torch
import torch.distributed as dist

from .targets import distribute_work


class TorchComm:
    """The mpi4py-style communicator redrock's distributed objects expect
    (``rank``, ``size``, ``bcast``, ``allgather``, ``gather``, ``barrier``)
    over a torch.distributed process group.  Python objects travel through
    a gloo group (host memory), made from the default group's ranks unless
    one is given, so large result dicts never pass through GPU buffers."""

    def __init__(self, group=None):
        if group is None:
            group = dist.new_group(backend="gloo") \
                if dist.get_backend() != "gloo" else dist.group.WORLD
        self.group = group

    @property
    def rank(self):
        return dist.get_rank(self.group)

    @property
    def size(self):
        return dist.get_world_size(self.group)

    def bcast(self, obj, root=0):
        buf = [obj]
        dist.broadcast_object_list(buf, src=root, group=self.group)
        return buf[0]

    def allgather(self, obj):
        out = [None] * self.size
        dist.all_gather_object(out, obj, group=self.group)
        return out

    def gather(self, obj, root=0):
        out = [None] * self.size if self.rank == root else None
        dist.gather_object(obj, out, dst=root, group=self.group)
        return out

    def barrier(self):
        dist.barrier(group=self.group)


def rank_world():
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def target_weights(targets, templates=None):
    """Work per target ~ pixels x (sum over templates of nz * nbasis)."""
    per_pix = 1
    if templates:
        per_pix = sum(len(t.redshifts) * t.nbasis for t in templates)
    return {t.id: per_pix * sum(len(s.wave) for s in t.spectra) for t in targets}


def shard_targets(targets, world, rank, templates=None):
    """This rank's targets, balanced by the weighted greedy rule."""
    ids = [t.id for t in targets]
    dist_ids = distribute_work(world, ids, weights=target_weights(targets, templates))
    mine = set(dist_ids[rank])
    return [t for t in targets if t.id in mine]


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks."""
    rank, world = rank_world()
    if world == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def gather_results(local, dst=0):
    """Merge per-rank dict[targetid] -> results on rank dst (others get None)."""
    rank, world = rank_world()
    if world == 1:
        return dict(local)
    parts = [None] * world if rank == dst else None
    dist.gather_object(local, parts, dst=dst)
    if rank != dst:
        return None
    out = {}
    for p in parts:
        out.update(p)
    return out
