"""Tile-shape autotuner for the fused scan.

A fused-scan tile is 32 targets (one per lane) x 8 ZT redshifts (8 warps, ZT
per thread) x 24-pixel stages, and the persistent CTAs take the tiles in an
order over (target block, redshift tile) set by ``block_group``.  The lane
and warp counts are fixed by the register file (each thread keeps its Gram
matrices in FP64 registers, 255 registers per thread, so 8 warps per SM) and
the stage by the shared memory holding a block's packed rows; the free
dimensions are ZT for the small bases, whose sweep is bound by shared-memory
traffic (several redshifts per thread share each packed-row load), and the
tile order.  Compiled choices: nbasis 4 -> ZT 1, 2, 3; nbasis 5 -> ZT 1, 2
(rr_scan_options); tile orders: target blocks fastest (tiles running
together share basis windows) or groups of 4 blocks with all their redshift
tiles (packed rows reused while in L2).

``tune(pack, bases)`` times the fused launch (CUDA events around the kernel
alone, after one untimed run) for each candidate of every small-basis
template present, keeps the fastest, and caches it per workload signature
(grids, each small template's nbasis and redshift count, number of target
blocks rounded up to a power of two).  ``choice`` returns the cached choice
(or None).  Tuning runs the scan of the small templates a few times, so it
belongs outside timed regions; the scan's results do not depend on the
choice beyond rounding order within a thread (the tests check bit equality).
"""

from __future__ import annotations

import torch

CANDIDATES = {4: (1, 2, 3), 5: (1, 2)}
# tile orders (rr_scan_options.block_group): target blocks fastest, or all
# redshift tiles of 4 target blocks (their packed rows, 4 x 24.5 MB on DESI
# grids, fit in the 126 MB L2) before the next 4
BLOCK_GROUPS = (0, 4)
_cache = {}


def _key(pack, bases):
    small = tuple(sorted((b.nbasis, b.nz) for b in bases if b.nbasis in CANDIDATES))
    nb = 1
    while nb < pack.nblock:
        nb *= 2
    return (pack.layout.signature, small, nb)


def choice(pack, bases):
    return _cache.get(_key(pack, bases))


def tune(pack, bases, repeats=1):
    """Time the candidates and cache the fastest ZT per small nbasis."""
    from .engine import run_fused
    key = _key(pack, bases)
    if key in _cache:
        return _cache[key]
    best = {}
    for nb, cands in CANDIDATES.items():
        sub = [b for b in bases if b.nbasis == nb]
        if not sub:
            continue
        times = {}
        for zt in cands:
            run_fused(pack, sub, tiles={nb: zt})   # untimed (first launch of a variant)
            ev = []
            for _ in range(repeats):
                run_fused(pack, sub, tiles={nb: zt}, kernel_events=ev)
            torch.cuda.synchronize()
            times[zt] = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        best[nb] = min(times, key=times.get)
        best[f"ms_{nb}"] = {zt: round(t, 3) for zt, t in times.items()}
    # tile order, timed on the templates without a ZT choice (GALAXY's
    # nbasis 10: the bulk of the scan), else on all of them
    groups = [g for g in BLOCK_GROUPS if g == 0 or g < pack.nblock]
    if len(groups) > 1:
        sub = [b for b in bases if b.nbasis not in CANDIDATES] or list(bases)
        zt = {nb: best[nb] for nb in CANDIDATES if nb in best}
        times = {}
        for g in groups:
            tiles = dict(zt, block_group=g)
            run_fused(pack, sub, tiles=tiles)
            ev = []
            for _ in range(repeats):
                run_fused(pack, sub, tiles=tiles, kernel_events=ev)
            torch.cuda.synchronize()
            times[g] = sum(a.elapsed_time(b) for a, b in ev) / len(ev)
        best["block_group"] = min(times, key=times.get)
        best["ms_block_group"] = {g: round(t, 3) for g, t in times.items()}
    _cache[key] = best
    return best


def tiles_of(best):
    """The run_fused ``tiles`` argument of a tune() result."""
    if not best:
        return None
    out = {nb: zt for nb, zt in best.items() if isinstance(nb, int)}
    if "block_group" in best:
        out["block_group"] = best["block_group"]
    return out
