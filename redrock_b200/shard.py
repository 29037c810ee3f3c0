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
