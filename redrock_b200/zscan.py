"""Drop-in redshift-scan functions (redrock 0.22 zscan.py) on the GPU.

  calc_zchi2          zscan.py:807-889   all targets x all z in one fused
                                         launch (rr_zscan_fused)
  calc_zchi2_targets  zscan.py:910-1105  every template in the same launch
  calc_zchi2_batch    zscan.py:626-781   one target, plain kernel chain
                                         (rr_zchi2_batch_plain)
  calc_zchi2_one      zscan.py:213-243   one z (plain chain with nz = 1)
  calc_negOII_penalty zscan.py:783-800
  spectral_data       zscan.py:192-209

Inputs are redrock's own objects (or the mirrors in redrock_b200.targets /
redrock_b200.templates); outputs are the same numpy arrays with the same
shapes.  Device copies of packed targets and template bases are cached by
the identity of the objects they came from; after changing a Target's or a
DistTemplate's arrays in place, call ``clear_caches()``.  Error conventions follow redrock: all-zero weights give HUGE_CHI2
rows with zero coefficients; an exactly singular normal matrix gives
HUGE_CHI2 at that z; an unrecognised solve method gives HUGE_CHI2
everywhere.  Non-negative / bounded solvers (NMF, NNLS, BVLS) run on the
GPU too, through the plain chain's device solvers.
"""

from __future__ import annotations

import sys

import numpy as np
import torch

from . import _lib
from .device import to_device, to_numpy
from .engine import (DeviceBasis, GridLayout, IdCache, PlainTarget, ScanResult, TargetBatch,
                     TargetPack, resolve_y, run_fused, run_plain)
from .templates import oii_sums, solve_code, solve_code_of

HUGE_CHI2 = 9999999.0

_pack_cache = IdCache(64)
_basis_cache = IdCache(32)
# zfind(graph=True): the captured device plan of the last target batch
_plan_cache = IdCache(1)


def clear_caches():
    """Drop the device copies of packed targets and template bases, and
    zfind's captured plan (needed after a caller modifies those objects'
    arrays in place)."""
    _pack_cache.clear()
    _basis_cache.clear()
    _plan_cache.clear()


def spectral_data(spectra):
    weights = np.concatenate([s.ivar for s in spectra])
    flux = np.concatenate([s.flux for s in spectra])
    return (weights, flux, weights * flux)


def calc_negOII_penalty(OIItemplate, coeff):
    """penalty[nz] = max(0, -sum over the [OII] window of the model)."""
    coeff_t = coeff if isinstance(coeff, torch.Tensor) else to_device(coeff)
    s = to_device(np.asarray(OIItemplate, dtype=np.float64).sum(axis=1))
    nz, nb = coeff_t.shape
    out = torch.empty(nz, dtype=torch.float64, device=coeff_t.device)
    from .device import ptr, stream_handle
    rc = _lib.lib().rr_negoii_penalty(ptr(coeff_t.contiguous()), nz, nb, ptr(s), ptr(out),
                                      stream_handle())
    _lib.check(rc, "rr_negoii_penalty")
    return out if isinstance(coeff, torch.Tensor) else out.cpu().numpy()


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def _layout_for(dtemplate, targets):
    lay = getattr(dtemplate, "layout", None)
    if isinstance(lay, GridLayout):
        return lay
    data = dtemplate.local.data
    waves = {}
    for t in targets:
        for s in t.spectra:
            waves.setdefault(s.wavehash, s.wave)
    return GridLayout((k, v.shape[1], waves.get(k)) for k, v in data.items())


def _device_basis(dtemplate, layout):
    b = getattr(dtemplate, "basis", None)
    if isinstance(b, DeviceBasis):
        return b
    tmpl = dtemplate.template

    def make():
        return DeviceBasis.from_tdata(dtemplate.local.data, layout,
                                      redshifts=dtemplate.local.redshifts, oii=oii_sums(tmpl),
                                      method=solve_code(tmpl))
    return _basis_cache.get(("dt", id(dtemplate), layout.signature), [dtemplate], make)


def _pack(targets, layout):
    def make():
        p = TargetPack.from_targets(targets, layout)
        torch.cuda.current_stream().synchronize()
        p.check()
        return p
    return _pack_cache.get(("pack", layout.signature, len(targets)), targets, make)


# ---------------------------------------------------------------------------
# fused scan
# ---------------------------------------------------------------------------
CHUNK_TARGETS = 224   # targets per pipelined chunk (7 target blocks)
# batches of at least LARGE_BATCH targets use CHUNK_TARGETS_LARGE: fewer
# chunks, so fewer last-wave tails and y GEMM padding (5000 DESI-like
# targets, end to end: 2583 ms per call at 448 and at 640, 2607 ms at 224,
# 2636 ms at 1024)
LARGE_BATCH = 2048
CHUNK_TARGETS_LARGE = 448
AUTOTUNE = True       # time the small-basis tile shapes once per workload signature
FIRST_CHUNK = 64      # a small first chunk gets the GPU started early
# (64 / 224 measured best of 32-64 / 128-468 for 500 DESI-like targets:
# 304.6 ms per end-to-end step against 315.3 ms for 32 / 128)


def _bases_for(dtemplates, layout):
    bases = []
    for dt in dtemplates:
        b = _device_basis(dt, layout)
        if b.layout.signature != layout.signature:
            # templates built on other grids: re-layout through the dict view
            b = DeviceBasis.from_tdata(dt.local.data, layout, redshifts=dt.local.redshifts,
                                       oii=oii_sums(dt.template), method=solve_code(dt.template))
        bases.append(b)
    return bases


def _chunk_bounds(n, chunk):
    if n <= 2 * chunk:
        return [(0, n)]
    bounds = [(0, min(FIRST_CHUNK, chunk))]
    while bounds[-1][1] < n:
        i0 = bounds[-1][1]
        bounds.append((i0, min(n, i0 + chunk)))
    return bounds


_side_streams = {}
_lane_streams = {}


def _side_stream():
    d = torch.cuda.current_device()
    if d not in _side_streams:
        _side_streams[d] = torch.cuda.Stream()
    return _side_streams[d]


def _lane_stream():
    d = torch.cuda.current_device()
    if d not in _lane_streams:
        _lane_streams[d] = torch.cuda.Stream()
    return _lane_streams[d]


class HostResult:
    """One template's results in pinned host memory (numpy views)."""

    def __init__(self, ntarget, basis):
        self.t = [torch.empty((ntarget, basis.nz), dtype=torch.float64, pin_memory=True),
                  torch.empty((ntarget, basis.nz, basis.nbasis), dtype=torch.float64,
                              pin_memory=True),
                  torch.empty((ntarget, basis.nz), dtype=torch.float64, pin_memory=True)]
        self.zchi2, self.zcoeff, self.penalty = (x.numpy() for x in self.t)


# solve methods the fused scan handles; NNLS / BVLS templates (their chi2 is
# the direct residual of a bounded solve) go through the plain chain
_FUSED_METHODS = (_lib.RR_SOLVE_PCA, _lib.RR_SOLVE_UNSUPPORTED)


def _plain_scan(targets, basis, layout):
    """One template with a bounded solve: the plain per-target chain for
    every target (calc_zchi2's loop, zscan.py:853-887), results on the
    device like the fused scan's."""
    res = ScanResult(len(targets), basis, torch.device("cuda", torch.cuda.current_device()))
    for i, t in enumerate(targets):
        w = np.concatenate([s.ivar for s in t.spectra])
        if w.sum() == 0:
            res.zchi2[i] = HUGE_CHI2
            res.zcoeff[i] = 0.0
            continue
        pt = PlainTarget(t.spectra, layout)
        zc, co = run_plain(pt, basis, method=basis.method)
        res.zchi2[i] = zc
        res.zcoeff[i] = co
        if basis.oii is not None:
            res.penalty[i] = calc_negOII_penalty_sums(basis.oii, co)
        pt._status.check("rr_zchi2_batch_plain_ex")
    return res


def calc_negOII_penalty_sums(oii_sums_dev, coeff_t):
    """calc_negOII_penalty from the per-basis window sums (device)."""
    from .device import ptr, stream_handle
    nz, nb = coeff_t.shape
    out = torch.empty(nz, dtype=torch.float64, device=coeff_t.device)
    rc = _lib.lib().rr_negoii_penalty(ptr(coeff_t.contiguous()), nz, nb, ptr(oii_sums_dev),
                                      ptr(out), stream_handle())
    _lib.check(rc, "rr_negoii_penalty")
    return out


_copy_streams = {}


def _pack_overlapped(sub, layout, st, main):
    """TargetPack of one chunk whose host-to-device copies run on a copy
    stream, so that they overlap the previous chunk's scan instead of
    queueing behind it on the chunk's compute stream ``main``; the pack
    kernel (launched on ``main``) waits for them.  The copy stream does not
    wait for ``main``: its buffers are new allocations, and record_stream
    keeps them from reuse until the kernels on ``main`` that read them are
    done."""
    d = torch.cuda.current_device()
    if d not in _copy_streams:
        _copy_streams[d] = torch.cuda.Stream()
    cs = _copy_streams[d]
    batch = TargetBatch(sub, layout)
    with torch.cuda.stream(cs):
        dbatch = batch.to_device()
    for name in ("descs", "segs", "first", "rows", "rdata", "roffs", "ivar", "flux"):
        getattr(dbatch, name).record_stream(main)
    ev = torch.cuda.Event()
    ev.record(cs)
    main.wait_event(ev)
    return TargetPack(dbatch, status=st)


class _NoGC:
    """Python's cyclic collector paused for the duration of the pipelined
    scan: a full collection (hundreds of ms with a large heap) in the middle
    would leave the GPU idle waiting for the next chunk's launches.  The
    objects made meanwhile are collected afterwards as usual."""

    def __enter__(self):
        import gc
        self._was = gc.isenabled()
        gc.disable()

    def __exit__(self, *exc):
        import gc
        if self._was:
            gc.enable()
        return False


def scan_device(targets, dtemplates, chunk=None, host=False, on_host_ready=None):
    """Fused scan of every target against every template (see
    _scan_device), with the cyclic garbage collector paused."""
    with _NoGC():
        out = _scan_device(targets, dtemplates, chunk=chunk, host=host,
                           on_host_ready=on_host_ready)
    # bases built asynchronously (DistTemplate) report device errors here
    for dt in dtemplates:
        chk = getattr(dt, "check", None)
        if callable(chk):
            chk()
    return out


def _scan_device(targets, dtemplates, chunk=None, host=False, on_host_ready=None):
    """Fused scan of every target against every template.

    Returns a list (one entry per template) of results with zchi2 (T, nz),
    zcoeff (T, nz, nbasis), penalty (T, nz): device ScanResult objects, or
    with host=True HostResult numpy arrays.  Large target lists are
    processed in chunks (a small first one, then CHUNK_TARGETS): the host
    packing and upload of chunk k + 1 run while the GPU scans chunk k, and
    with host=True chunk k's results are copied to pinned host memory on a
    side stream while chunk k + 1 runs.  on_host_ready(hout) (host=True) is
    called once the GPU has the first two chunks queued, with the host
    result arrays (filled as the copies land, complete when this returns),
    so that the caller can build its views of them meanwhile.
    """
    layout = _layout_for(dtemplates[0], targets)
    all_bases = _bases_for(dtemplates, layout)
    plain_ix = [i for i, b in enumerate(all_bases) if b.method not in _FUSED_METHODS]
    if plain_ix:
        fused_ix = [i for i in range(len(all_bases)) if i not in plain_ix]
        out = [None] * len(all_bases)
        if fused_ix:
            part = scan_device(targets, [dtemplates[i] for i in fused_ix], chunk=chunk, host=host)
            for i, r in zip(fused_ix, part):
                out[i] = r
        for i in plain_ix:
            r = _plain_scan(targets, all_bases[i], layout)
            if host:
                h = HostResult(len(targets), all_bases[i])
                for dst, src in zip(h.t, (r.zchi2, r.zcoeff, r.penalty)):
                    dst.copy_(src)
                r = h
            out[i] = r
        return out
    bases = all_bases
    chunk = chunk or (CHUNK_TARGETS_LARGE if len(targets) >= LARGE_BATCH else CHUNK_TARGETS)
    from .device import StatusWord
    st = StatusWord()
    bounds = _chunk_bounds(len(targets), chunk)
    main = torch.cuda.current_stream()
    # consecutive chunks alternate between two compute streams, so that a
    # chunk's packing, y GEMMs and first scan launch need not wait for the
    # previous chunk's last tiles: its CTAs take the SMs that the other
    # chunk's last tile wave leaves idle (each chunk has its own outputs,
    # tile counters and scratch, allocated on its own stream)
    lanes = [main] if len(bounds) == 1 else [main, _lane_stream()]
    if len(lanes) > 1:
        # what the chunks share is made on main first: the bases and their
        # INT8 digit planes for the y GEMM (cached on each basis)
        yv = _lib.YGEMM_VARIANTS[resolve_y(None, layout)]
        if yv in _lib.I8_VARIANTS:
            kpad = int(_lib.lib().rr_ygemm_kpad(layout.pix_stride))
            for b in bases:
                b.i8_digits(kpad, variant=yv)
        ev0 = torch.cuda.Event()
        ev0.record(main)
        lanes[1].wait_event(ev0)
    side = _side_stream() if host else None
    hout = [HostResult(len(targets), b) for b in bases] if host else None
    parts = []
    keep = []
    for k, (i0, i1) in enumerate(bounds):
        sub = targets[i0:i1]
        cs = lanes[k % len(lanes)]
        with torch.cuda.stream(cs):
            if len(bounds) == 1:
                pack = _pack(sub, layout)
            else:
                pack = _pack_cache.get(("chunk", layout.signature, i0, len(sub)), sub,
                                       lambda: _pack_overlapped(sub, layout, st, cs))
            tiles = None
            if AUTOTUNE:
                from . import autotune
                tiles = autotune.tiles_of(autotune.choice(pack, bases)
                                          or autotune.tune(pack, bases))
            res, _ = run_fused(pack, bases, status=st, tiles=tiles)
        keep.append((pack, res))
        if host:
            ev = torch.cuda.Event()
            ev.record(cs)
            side.wait_event(ev)
            with torch.cuda.stream(side):
                for h, r in zip(hout, res):
                    for dst, src in zip(h.t, (r.zchi2, r.zcoeff, r.penalty)):
                        dst[i0:i1].copy_(src, non_blocking=True)
            if on_host_ready is not None and len(keep) == min(2, len(bounds)):
                on_host_ready(hout)
        else:
            parts.append(res)
    if len(lanes) > 1:
        ev1 = torch.cuda.Event()
        ev1.record(lanes[1])
        main.wait_event(ev1)
        # device results of the lane's chunks are read on main from here on
        for k, (_, res) in enumerate(keep):
            if k % 2:
                for r in res:
                    for t in (r.zchi2, r.zcoeff, r.penalty):
                        t.record_stream(main)
    main.synchronize()
    if host:
        side.synchronize()
    st.check("rr_zscan_fused")
    if host:
        return hout
    if len(parts) == 1:
        return parts[0]
    out = []
    for it in range(len(bases)):
        r = parts[0][it]
        r.zchi2 = torch.cat([p[it].zchi2 for p in parts])
        r.zcoeff = torch.cat([p[it].zcoeff for p in parts])
        r.penalty = torch.cat([p[it].penalty for p in parts])
        out.append(r)
    return out


def calc_zchi2(target_ids, target_data, dtemplate, progress=None, use_gpu=False):
    """chi2 vs redshift of every target for one template (zscan.py:807)."""
    ntargets = len(target_ids)
    nz = len(dtemplate.local.redshifts)
    nbasis = dtemplate.template.nbasis
    if ntargets == 0:
        return np.zeros((0, nz)), np.zeros((0, nz, nbasis)), np.zeros((0, nz))
    res = scan_device(list(target_data), [dtemplate], host=True)[0]
    zchi2, zcoeff, pen = res.zchi2, res.zcoeff, res.penalty
    if dtemplate.comm is None and progress is not None:
        for _ in range(ntargets):
            progress.put(1)
    return zchi2, zcoeff, pen


def calc_zchi2_targets(targets, templates, mp_procs=1, use_gpu=True):
    """All templates for all local targets in one fused launch (zscan.py:910).

    Results are keyed by the id of each target object in ``targets.local()``.
    (redrock pairs ``local_target_ids()`` -- sorted by number of spectra --
    with ``local()`` in input order, zscan.py:1008-1019, which attaches a
    target's chi2 to another target when spectrum counts differ; keying by
    the object's own id gives redrock's answer whenever redrock's pairing is
    consistent.)
    """
    am_root = targets.comm is None or targets.comm.rank == 0
    data = list(targets.local())
    tids = [t.id for t in data]
    results = {tid: {} for tid in targets.local_target_ids()}
    if am_root:
        print("Computing redshifts")
        sys.stdout.flush()
    if len(tids) == 0:
        return results

    def fill(out):
        # views of the pinned host results, built while the GPU scans
        for t, r in zip(templates, out):
            ft = t.template.full_type
            zc, co, pe = r.zchi2, r.zcoeff, r.penalty
            z = t.template.redshifts
            for i, tid in enumerate(tids):
                results.setdefault(tid, {})[ft] = dict(redshifts=z, zchi2=zc[i], penalty=pe[i],
                                                       zcoeff=co[i])
    done = []
    out = scan_device(data, list(templates), host=True,
                      on_host_ready=lambda hout: (fill(hout), done.append(True)))
    if not done:
        fill(out)
    return results


# ---------------------------------------------------------------------------
# plain per-target path
# ---------------------------------------------------------------------------
def _plain_layout(spectra, tdata):
    waves = {}
    for s in spectra:
        waves.setdefault(s.wavehash, s.wave)
    keys = list(dict.fromkeys(s.wavehash for s in spectra))
    return GridLayout((k, tdata[k].shape[-2], waves[k]) for k in keys)


def calc_zchi2_batch(spectra, tdata, weights, flux, wflux, nz, nbasis,
                     solve_matrices_algorithm=None, solver_args=None, use_gpu=False,
                     fullprecision=True, prior=None):
    """chi2 and coefficients of one target for all z (zscan.py:626)."""
    wh = to_numpy(weights)
    if wh.sum() == 0:
        return np.full(nz, HUGE_CHI2), np.zeros((nz, nbasis))
    # solve_matrices (zscan.py:1107-1203): PCA, NMF/NNLS, BVLS (bounds from
    # solver_args, default unbounded), else NotImplementedError -> HUGE
    method = solve_code_of(solve_matrices_algorithm)
    bounds = None
    if method == _lib.RR_SOLVE_BVLS and solver_args is not None and 'bounds' in solver_args:
        bounds = solver_args['bounds']
    layout = _plain_layout(spectra, tdata)
    sub = {k: tdata[k] for k in layout.keys}
    basis = DeviceBasis.from_tdata(sub, layout)
    pt = PlainTarget(spectra, layout, weights, flux, wflux)
    zchi2, zcoeff = run_plain(pt, basis, prior=prior, method=method, bounds=bounds)
    torch.cuda.current_stream().synchronize()
    pt._status.check("rr_zchi2_batch_plain")
    if use_gpu:
        return zchi2.cpu().numpy(), zcoeff
    return zchi2.cpu().numpy(), zcoeff.cpu().numpy()


def calc_zchi2_one(spectra, weights, flux, wflux, tdata, solve_matrices_algorithm):
    """chi2 and coefficients at one redshift (zscan.py:213)."""
    t3 = {k: (v[None] if isinstance(v, torch.Tensor) else np.asarray(v)[None])
          for k, v in tdata.items()}
    nbasis = next(iter(t3.values())).shape[-1]
    zc, co = calc_zchi2_batch(spectra, t3, weights, flux, wflux, 1, nbasis,
                              solve_matrices_algorithm)
    return float(zc[0]), np.asarray(to_numpy(co))[0]


def per_camera_coeff_with_least_square_batch(target, tdata, weights, flux, wflux, nleg, narch,
                                             method=None, n_nbh=None, prior=None, use_gpu=False,
                                             bands=None):
    """Archetype fit with a separate set of Legendre terms per camera
    (zscan.py:245-348).

    ``tdata[hs]`` is (narch, npix, n_nbh + nleg): n_nbh archetype columns
    followed by the camera's Legendre polynomials.  Each camera's Legendre
    block moves to its own columns of an (narch, npix, n_nbh + nleg * ncam)
    basis -- built on the device -- and all narch fits run as one batch of
    the solve chain (``calc_zchi2_batch`` with nz = narch), BVLS keeping
    the archetype coefficients >= 0.  Coefficients come back as
    [archetype terms, then each camera's Legendre terms in ``bands``
    order].  With n_nbh > 1 redrock keeps only the first row's archetype
    terms, so that case needs narch == 1, as redrock's caller has it.
    """
    spectra = target.spectra
    ncam = len(bands)
    nbasis = n_nbh + nleg * ncam
    method = method.upper()
    solver_args = {}
    if method == 'BVLS':
        bounds = np.zeros((2, nbasis))
        bounds[0][n_nbh:] = -np.inf
        bounds[1] = np.inf
        solver_args['bounds'] = bounds
    wide = {}
    for i, hs in enumerate(tdata):
        a = to_device(tdata[hs])
        w = torch.zeros((a.shape[0], a.shape[1], nbasis), dtype=torch.float64, device=a.device)
        w[:, :, :n_nbh] = a[:, :, :n_nbh]
        w[:, :, n_nbh + i * nleg:n_nbh + (i + 1) * nleg] = a[:, :, n_nbh:]
        wide[hs] = w
    zzchi2, zzcoeff = calc_zchi2_batch(spectra, wide, weights, flux, wflux, narch, nbasis,
                                       solve_matrices_algorithm=method, solver_args=solver_args,
                                       prior=prior)
    # redrock's column bookkeeping: an 'alpha' entry, then one entry per band
    # in ``bands`` order (dict insertion order), filled camera by camera
    parts = {'alpha': [zzcoeff[:, k] for k in range(n_nbh)]}
    if nleg > 0:
        for b in bands:
            parts[b] = []
    if n_nbh > 1:
        parts['alpha'] = np.array([parts['alpha'][k][0] for k in range(n_nbh)])[None, :]
    else:
        parts['alpha'] = parts['alpha'][0][:, None]
    if nleg >= 1:
        blocks = np.split(zzcoeff[:, n_nbh:], ncam, axis=1)
        by_band = {band: blocks[i] for i, band in enumerate(bands)}
        for band in sorted(bands):
            parts[band] = by_band[band]
    return zzchi2, np.concatenate(list(parts.values()), axis=1)


def calc_zchi2_plain(target_ids, target_data, dtemplate):
    """calc_zchi2 through the plain per-target kernel chain (the structure of
    redrock's own GPU branch: one chain of launches and one host read-back
    per target).  Used as the comparison path for the fused scan."""
    ntargets = len(target_ids)
    nz = len(dtemplate.local.redshifts)
    nbasis = dtemplate.template.nbasis
    zchi2 = np.zeros((ntargets, nz))
    zcoeff = np.zeros((ntargets, nz, nbasis))
    pen = np.zeros((ntargets, nz))
    layout = _layout_for(dtemplate, target_data)
    basis = _device_basis(dtemplate, layout)
    oii = oii_sums(dtemplate.template)
    for j, t in enumerate(target_data):
        w, f, wf = spectral_data(t.spectra)
        if np.sum(w) == 0:
            zchi2[j, :] = HUGE_CHI2
            continue
        pt = PlainTarget(t.spectra, layout, w, f, wf)
        zc, co = run_plain(pt, basis, method=basis.method)
        zchi2[j] = zc.cpu().numpy()
        zcoeff[j] = co.cpu().numpy()
        if oii is not None:
            pen[j] = calc_negOII_penalty(dtemplate.template.OIItemplate, co).cpu().numpy()
    return zchi2, zcoeff, pen
