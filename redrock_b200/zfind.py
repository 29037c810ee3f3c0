"""Redshift finding driver on the GPU engine (redrock zfind.py:220-711).

``zfind(targets, templates, nminima=3, ...)`` runs, for the local targets:

  1. the coarse scan of every template in one fused launch
     (``calc_zchi2_targets``),
  2. the fine-grid refinement of every target's minima, one batched pair-scan
     launch group per template (``fitz_targets``),
  3. redrock's finalisation: NODATA / LITTLE_COVERAGE bits, sort by badfit
     bits then chi2, keep ``nminima`` per spectral type, delta-chi2 and
     SMALL_DELTA_CHI2 (``calc_deltachi2``, zfind.py:103-155).

With ``archetypes`` (dict spectype -> Archetype) each refined minimum of a
template with an archetype set is refitted with the archetypes
(``fitz_targets(archetype=...)``), and the finalisation adds redrock's
archetype columns (pca_coeff / pca_spectype / pca_subtype, legcoeff) and the
NEGATIVE_MODEL bit (zfind.py:470-580).

It returns ``(allresults, allzfit)`` like redrock, except that ``allzfit`` is
a dict of numpy columns (``astropy.table.Table(allzfit)`` gives redrock's
table) with redrock's column names and order of rows.  ``priors`` is a
``redrock_b200.priors.Priors`` (or redrock's) object, or a prior file name.
``chi2_scan`` names a details file (``redrock_b200.results.write_zscan`` or
redrock's) whose coarse scans replace the scan.

``graph=True`` runs the device part for the whole local batch -- target
packing, the fused scan, the K lowest minima of every (target, template) and
the chi2 of their fine redshift grids (``DeviceFitzPlan``) -- as one
captured CUDA graph, so no host round trip sits between the coarse scan and
the fine grids; the host then replays redrock's candidate logic on those
values exactly as the eager path does (rows with tied minima, and targets
that need more than K candidates, continue on the host), so the outputs are
the eager path's bit for bit.  ``refine="newton"`` replaces the parabola
through the three fine-grid points by batched Newton steps on chi2(z).

Several processes (one per GPU): give the targets an mpi4py-style
communicator (``rank``, ``size``, ``bcast``, ``allgather``, ``gather``,
``barrier``; ``redrock_b200.shard.TorchComm`` wraps a torch.distributed
group).  Each rank scans and refines its own targets against every redshift
of every template (redrock's GPU mode, templates.py:558-563); the per-target
results are then gathered on rank 0 (zfind.py:416-456), which finalises and
returns them, while the other ranks return ``(None, None)``.
"""

from __future__ import annotations

import numpy as np

from . import fitz as _fitz
from . import _lib
from .templates import parse_fulltype, solve_code
from .engine import GridLayout, RowPack
from .zscan import calc_zchi2_targets

MAX_VELO_DIFF = 1000.0
MAX_VELO_DIFF_STAR = 100.0
MIN_DELTACHI2 = 9.0                 # constants.py:10
SMALL_DELTA_CHI2 = 2 ** 2           # zwarning.py:17
LITTLE_COVERAGE = 2 ** 1
NODATA = 2 ** 9
NEGATIVE_MODEL = 2 ** 3
MANY_OUTLIERS = 2 ** 4
Z_FITLIMIT = 2 ** 5
NEGATIVE_EMISSION = 2 ** 6
BAD_MINFIT = 2 ** 10
BADFIT_MASK = NEGATIVE_MODEL | MANY_OUTLIERS | Z_FITLIMIT | NEGATIVE_EMISSION | BAD_MINFIT


def calc_deltachi2(chi2, z, zwarn, dvlimit=MAX_VELO_DIFF):
    """chi2 difference to the next good fit farther than dvlimit; and which
    fits have another good fit within MIN_DELTACHI2 (zfind.py:103-155)."""
    nz = len(chi2)
    deltachi2 = np.zeros(nz)
    okfit = (zwarn & BADFIT_MASK) == 0
    if np.isscalar(dvlimit):
        dvlimit = np.full(nz, dvlimit)
    return _deltachi2_f64(np.asarray(chi2, dtype=np.float64), np.asarray(z, dtype=np.float64),
                          okfit, np.asarray(dvlimit, dtype=np.float64))


def _deltachi2_f64(chi2, z, okfit, dvlimit):
    """calc_deltachi2 on float64 inputs with Python floats: the same IEEE
    operations in the same order per pair (a target has a handful of
    fits, where numpy's per-call cost dominates)."""
    c, zz, ok, dl = chi2.tolist(), z.tolist(), okfit.tolist(), dvlimit.tolist()
    nz = len(c)
    deltachi2 = np.zeros(nz)
    for i in range(nz - 1):
        best = None
        for j in range(i + 1, nz):
            if ok[j] and abs(_fitz.C_KMS * (zz[j] - zz[i]) / (1.0 + zz[i])) > min(dl[i], dl[j]):
                d = c[j] - c[i]
                # a NaN difference sticks, as in numpy's min
                if best is None or d < best or d != d:
                    best = d
        if best is not None:
            deltachi2[i] = best
    setzwarn = np.zeros(nz, dtype=bool)
    for i in range(nz):
        for j in range(nz):
            if j != i and ok[j] and abs(c[j] - c[i]) < MIN_DELTACHI2 and \
                    abs(_fitz.C_KMS * (zz[j] - zz[i]) / (1.0 + zz[i])) >= min(dl[i], dl[j]):
                setzwarn[i] = True
                break
    return deltachi2, setzwarn


def sort_dict_by_cols(d, colnames, sort_first_column_first=True):
    """Stable multi-key sort of a dict of arrays (zfind.py:53-80)."""
    vals = tuple(d[c] for c in colnames)
    if sort_first_column_first:
        vals = vals[::-1]
    idx = np.lexsort(vals, axis=0).flatten()
    for k in d.keys():
        d[k] = d[k][idx]


def sort_zfit_dict(zfit):
    """Sort by badfit bits, then chi2 (zfind.py:206-218)."""
    zfit['__badfit__'] = (zfit['zwarn'] & BADFIT_MASK) != 0
    sort_dict_by_cols(zfit, ('__badfit__', 'chi2'), sort_first_column_first=True)
    zfit.pop('__badfit__')


# archetype mode: result columns that fall back to another column of a
# template fitted without archetypes, and columns filled with zeros
# (utils.py:273-279)
PCA_MAP = {"pca_coeff": "coeff", "pca_subtype": "subtype", "pca_spectype": "spectype"}
ZERO_LIKE_KEYS = {"archcoeff", "legcoeff"}


def _pad_cols(val, ref):
    return np.pad(val, ((0, 0), (0, max(0, ref.shape[1] - val.shape[1]))),
                  constant_values=0)[:, :ref.shape[1]]


def _finalise_target(tid, fits, nminima, arch=None):
    """One target's rows of the zfit table (zfind.py:466-616).  ``arch``:
    None, or dict(spectypes=archetype spectypes, all_spectypes=template
    spectypes, n_nearest=...)."""
    tzfit = []
    for fulltype, tmp in fits:
        tmp = dict(tmp)
        if arch is not None and 'fulltype' in tmp:
            spectype, subtype = [], []
            for el in tmp['fulltype']:
                a, b = parse_fulltype(el[0])
                spectype.append(a)
                subtype.append(b)
            del tmp['fulltype']
        else:
            spectype, subtype = parse_fulltype(fulltype)
        nmin = len(tmp['chi2'])
        if nmin == 0:
            print(f'WARNING: no {fulltype} chi2 vs. z minima for targetid {tid}')
            continue
        if np.isscalar(spectype):
            tmp['spectype'] = np.full((nmin, 1), spectype)
            tmp['subtype'] = np.full((nmin, 1), subtype)
        else:
            tmp['spectype'] = np.array([spectype]).reshape((nmin, 1))
            tmp['subtype'] = np.array([subtype]).reshape((nmin, 1))
        tmp['ncoeff'] = np.array([tmp['coeff'].shape[1]] * nmin).reshape((nmin, 1))
        star = (spectype.upper() == 'STAR') if np.isscalar(spectype) else \
            (spectype[0].upper() == 'STAR')
        tmp['max_velo_diff'] = np.full((nmin, 1), MAX_VELO_DIFF_STAR if star else MAX_VELO_DIFF)
        tzfit.append(tmp)
    maxncoeff = max(t['coeff'].shape[1] for t in tzfit)
    for t in tzfit:
        if t['coeff'].shape[1] < maxncoeff:
            n = maxncoeff - t['coeff'].shape[1]
            t['coeff'] = np.append(t['coeff'], np.zeros((t['coeff'].shape[0], n)), axis=1)
    out = {}
    for k in tzfit[0].keys():
        ref = tzfit[0][k]
        vals = []
        val = None
        for row in tzfit:
            if k in row:
                val = row[k]
                if arch is not None and k in PCA_MAP:
                    val = _pad_cols(val, ref)
            elif arch is not None and k in PCA_MAP and PCA_MAP[k] in row:
                val = _pad_cols(row[PCA_MAP[k]], ref)
            elif k in ZERO_LIKE_KEYS:
                val = np.zeros_like(ref)
            # otherwise the previous row's value repeats, as in redrock's loop
            vals.append(val)
        # np.vstack of 2-D arrays is their concatenation (without vstack's
        # per-call promotion overhead)
        if all(type(v) is np.ndarray and v.ndim == 2 for v in vals):
            out[k] = np.concatenate(vals, axis=0)
        else:
            out[k] = np.vstack(vals)
        if k != 'coeff' and out[k].shape[1] == 1:
            out[k] = out[k].flatten()
    n = len(out['chi2'])
    out['targetid'] = np.array([tid] * n)
    if arch is not None:
        nn = arch['n_nearest']
        if len(arch['spectypes']) == len(arch['all_spectypes']):
            if nn is None:
                if out['coeff'].ndim == 1:
                    out['coeff'] = out['coeff'].reshape(-1, 1)
                ibad = out['coeff'][:, 0] <= 0.
            else:
                ibad = np.any(out['coeff'][:, :nn] < 0, axis=1)
        else:
            ibad = np.isin(out['spectype'], np.array(arch['spectypes']))
            for k in np.where(ibad)[0]:
                if nn is None:
                    if out['coeff'][:, 0][k] >= 0.:
                        ibad[k] = False
                elif np.all(out['coeff'][:, :nn][k] >= 0):
                    ibad[k] = False
        out['zwarn'][ibad] |= NEGATIVE_MODEL
    out['zwarn'][out['npixels'] == 0] |= NODATA
    out['zwarn'][out['npixels'] < 10 * out['ncoeff']] |= LITTLE_COVERAGE
    sort_zfit_dict(out)
    keep = []
    for spectype in np.unique(out['spectype']):
        keep.extend(np.where(out['spectype'] == spectype)[0][0:nminima])
    if len(keep) < n:
        for k in out.keys():
            out[k] = out[k][keep]
        sort_zfit_dict(out)
    n = len(out['chi2'])
    out['znum'] = np.arange(n)
    deltachi2, setzwarn = calc_deltachi2(out['chi2'], out['z'], out['zwarn'],
                                         dvlimit=out['max_velo_diff'])
    out['deltachi2'] = deltachi2
    out['zwarn'][setzwarn] |= SMALL_DELTA_CHI2
    del out['max_velo_diff']
    return out


def _deltachi2_batch(chi2, z, okfit, dvlimit, first, n):
    """_deltachi2_f64 of many targets at once: target i owns rows
    first[i] .. first[i] + n[i] - 1.  The rows are laid out as a padded
    [target][row][row] block and every pair gets the same IEEE operations
    as the per-target loop: deltachi2[i] is the minimum of c_j - c_i over
    the later good fits farther than the velocity limit (NaN if one of
    them is NaN, 0 if there is none); setzwarn[i] flags another good fit
    within MIN_DELTACHI2 and at least the velocity limit away."""
    nt, m = len(n), int(n.max()) if len(n) else 0
    rows = first[:, None] + np.arange(m)[None, :]
    valid = np.arange(m)[None, :] < n[:, None]
    rows = np.where(valid, rows, 0)
    c, zz, ok, dl = chi2[rows], z[rows], okfit[rows] & valid, dvlimit[rows]
    dv = np.abs(_fitz.C_KMS * (zz[:, None, :] - zz[:, :, None]) / (1.0 + zz[:, :, None]))
    lim = np.minimum(dl[:, :, None], dl[:, None, :])
    d = c[:, None, :] - c[:, :, None]           # [t][i][j] = c_j - c_i
    later = np.arange(m)[None, :] > np.arange(m)[:, None]
    far = ok[:, None, :] & later[None] & (dv > lim)
    dmin = np.where(far, d, np.inf).min(axis=2)
    has_nan = (far & np.isnan(d)).any(axis=2)
    dmin = np.where(has_nan, np.nan, dmin)
    dmin = np.where(far.any(axis=2), dmin, 0.0)
    other = ~np.eye(m, dtype=bool)[None]
    near = (ok[:, None, :] & other & (np.abs(d) < MIN_DELTACHI2) & (dv >= lim)).any(axis=2)
    deltachi2 = dmin[valid]
    setzwarn = near[valid]
    return deltachi2, setzwarn


def _finalise_batch(tids, fits_list, nminima):
    """The zfit table of many targets at once -- the concatenation of
    _finalise_target(tid, fits, nminima) over the targets (no archetypes),
    as column arrays -- or None when the batch needs the per-target path
    (a target without minima for some template, or templates in different
    orders or with differently shaped columns).

    The same steps as _finalise_target, over all rows: the derived columns
    per template, ZWARN's NODATA / LITTLE_COVERAGE bits, the stable
    (badfit, chi2) order within each target, the first nminima fits per
    spectype kept (a target that loses fits is re-sorted from the
    spectype-grouped order, as the per-target code does), znum, and
    calc_deltachi2 per target."""
    if not tids:
        return None
    fts = [ft for ft, _ in fits_list[0]]
    for fits in fits_list:
        if [ft for ft, _ in fits] != fts:
            return None
        for _, z in fits:
            if len(z['chi2']) == 0:
                return None
    keys = list(fits_list[0][0][1].keys())
    if any(list(z.keys()) != keys for fits in fits_list for _, z in fits):
        return None
    nt, ntm = len(tids), len(fts)
    counts = np.array([[len(z['chi2']) for _, z in fits] for fits in fits_list], dtype=np.int64)
    ncoeffs = [fits_list[0][k][1]['coeff'].shape[1] for k in range(ntm)]
    if any(z['coeff'].ndim != 2 or z['coeff'].shape[1] != ncoeffs[k]
           for fits in fits_list for k, (_, z) in enumerate(fits)):
        return None
    maxncoeff = max(ncoeffs)
    out = {}
    # rows in target-major order: target, then template, then minimum
    for k in keys:
        vals = [z[k] for fits in fits_list for _, z in fits]
        if k == 'coeff':
            vals = [v if v.shape[1] == maxncoeff else
                    np.append(v, np.zeros((v.shape[0], maxncoeff - v.shape[1])), axis=1)
                    for v in vals]
        if not all(type(v) is np.ndarray and v.ndim == 2 for v in vals):
            return None
        col = np.concatenate(vals, axis=0)
        out[k] = col.flatten() if (k != 'coeff' and col.shape[1] == 1) else col
    n_tm = counts.ravel()  # rows per (target, template), target-major
    spec_sub = [parse_fulltype(ft) for ft in fts]
    tm_idx = np.tile(np.arange(ntm), nt)
    spectype = np.repeat(np.array([st for st, _ in spec_sub])[tm_idx], n_tm)
    subtype = np.repeat(np.array([sb for _, sb in spec_sub])[tm_idx], n_tm)
    ncoeff = np.repeat(np.array(ncoeffs, dtype=np.int64)[tm_idx], n_tm)
    mvd = np.repeat(np.array([MAX_VELO_DIFF_STAR if st.upper() == 'STAR' else MAX_VELO_DIFF
                              for st, _ in spec_sub])[tm_idx], n_tm)
    out['spectype'], out['subtype'], out['ncoeff'] = spectype, subtype, ncoeff
    n_t = counts.sum(axis=1)
    tix = np.repeat(np.arange(nt), n_t)
    out['targetid'] = np.repeat(np.asarray(tids), n_t)
    zwarn = out['zwarn']
    zwarn[out['npixels'] == 0] |= NODATA
    zwarn[out['npixels'] < 10 * out['ncoeff']] |= LITTLE_COVERAGE
    badfit = (zwarn & BADFIT_MASK) != 0
    chi2 = out['chi2']
    # stable (badfit, chi2) order within each target
    order = np.lexsort((chi2, badfit, tix))
    # the first nminima of each (target, spectype) in that order
    scode = np.unique(spectype, return_inverse=True)[1].ravel()
    g = tix[order] * (scode.max() + 1) + scode[order]
    gs = np.argsort(g, kind='stable')
    gsorted = g[gs]
    start = np.r_[0, np.nonzero(np.diff(gsorted))[0] + 1]
    rank_sorted = np.arange(len(g)) - np.repeat(start, np.diff(np.r_[start, len(g)]))
    rank = np.empty_like(rank_sorted)
    rank[gs] = rank_sorted
    keep = rank < nminima
    kept = order[keep]
    # targets that lost fits: ties in (badfit, chi2) follow the spectype
    # grouping their kept rows were put in before the second sort
    lost = np.zeros(nt, dtype=bool)
    lost[tix[order[~keep]]] = True
    pos = np.empty(len(order), dtype=np.int64)
    pos[order] = np.arange(len(order))
    sec = np.where(lost[tix[kept]], scode[kept], 0)
    final = kept[np.lexsort((pos[kept], sec, chi2[kept], badfit[kept], tix[kept]))]
    res = {k: v[final] for k, v in out.items()}
    res['max_velo_diff'] = mvd[final]
    ft_t = tix[final]
    n_keep = np.bincount(ft_t, minlength=nt)
    first = np.r_[0, np.cumsum(n_keep)[:-1]]
    res['znum'] = np.arange(len(final)) - np.repeat(first, n_keep)
    okfit = (res['zwarn'] & BADFIT_MASK) == 0
    deltachi2, setzwarn = _deltachi2_batch(np.asarray(res['chi2'], dtype=np.float64),
                                           np.asarray(res['z'], dtype=np.float64), okfit,
                                           np.asarray(res['max_velo_diff'], dtype=np.float64),
                                           first, n_keep)
    res['deltachi2'] = deltachi2
    res['zwarn'][setzwarn] |= SMALL_DELTA_CHI2
    del res['max_velo_diff']
    # the per-target path's column order: the fit columns, the derived
    # ones, then targetid, znum, deltachi2 (zfind puts targetid first)
    cols = keys + ['spectype', 'subtype', 'ncoeff', 'targetid', 'znum', 'deltachi2']
    return {k: res[k] for k in cols}


# candidates per target and template evaluated on the device in the graph
# path (rr_fitz_candidates): nminima plus this many spares for candidates
# that fall within max_velo_diff of a better one.  Rows that need more are
# continued by further pair launches from the host, as in the eager path;
# for 500 DESI-like targets x 7 templates no spare measured fastest (1.03 s
# per call against 1.10 s with one and 1.18 s with two)
DEVICE_CANDIDATES_EXTRA = 0


_warm_devices = set()


class _PackShape:
    """What the tile autotuner keys a choice on (grid layout, number of
    target blocks), without packing the targets."""

    def __init__(self, layout, nblock):
        self.layout = layout
        self.nblock = nblock


class DeviceFitzPlan:
    """The device part of zfind for one target batch -- target packing, the
    fused coarse scan of every template, the K lowest chi2 minima of every
    (target, template) and the chi2 of their fine redshift grids -- as
    launches with no host round trip, optionally captured as CUDA graphs
    (one for the scan, one per template) and replayed.  ``launch()`` starts
    it; ``coarse()`` returns the coarse-scan results in calc_zchi2_targets'
    form once the scan is done, ``fine(k)`` template k's
    ``fitz.PrecomputedFine`` once its fine grids are done, so the host can
    refine one template while the device still works on the next.

    Lazy one-time set-up (kernel attributes, constant tables) happens in an
    eager warm-up on the first target block before the first capture on a
    device; the tile autotuner's choice is cached per batch shape."""

    def __init__(self, local, templates, layout, nminima=3, nfine=15, graph=True):
        import torch
        from . import autotune
        from .device import StatusWord, to_device
        from .engine import TargetBatch, TargetPack, TemplateSource
        from .zscan import _bases_for
        self.local = local
        self.templates = list(templates)
        self.layout = layout
        self.K = min(8, nminima + DEVICE_CANDIDATES_EXTRA)
        self.nfine = nfine
        self.status = StatusWord()
        self.bases = _bases_for(self.templates, layout)
        self.srcs = [TemplateSource.from_template(t.template) for t in self.templates]
        self.zdev = [to_device(np.asarray(t.template.redshifts, dtype=np.float64))
                     for t in self.templates]
        self.dbatch = TargetBatch(local, layout).to_device()
        self.rowpack = RowPack(self.dbatch)
        key = _PackShape(layout, self.dbatch.batch.nblock)
        best = autotune.choice(key, self.bases)
        if best is None:
            pack0 = TargetPack(self.dbatch, status=self.status)
            best = autotune.tune(pack0, self.bases)
            del pack0
        self.tiles = autotune.tiles_of(best)
        dev = torch.cuda.current_device()
        if dev not in _warm_devices:
            # once per process and device, before any capture: every
            # kernel's lazy set-up (attributes, constant tables), on the
            # first 32 targets
            small = local[:32]
            wb = TargetBatch(small, layout).to_device()
            wres = self._scan(wb)
            wrows = RowPack(wb)
            for k in range(len(self.templates)):
                self._fine(k, wres[k], wrows)
            torch.cuda.synchronize()
            self.status.check("zfind warm-up")
            _warm_devices.add(dev)
        # graph mode: one graph for packing + the fused scan, one per
        # template for its candidates and fine-grid scans, replayed back to
        # back with an event after each, so the host can read one
        # template's results while the next graphs run
        self.graphs = None
        if graph:
            from .device import capture_graph
            g_scan, self.res = capture_graph(lambda: self._scan(self.dbatch))
            self.graphs = [g_scan]
            self.fouts = []
            for k in range(len(self.templates)):
                g, out = capture_graph(lambda k=k: self._fine(k, self.res[k], self.rowpack))
                self.graphs.append(g)
                self.fouts.append(out)

    def _scan(self, dbatch):
        from .engine import TargetPack, run_fused
        pack = TargetPack(dbatch, status=self.status)
        res, _ = run_fused(pack, self.bases, status=self.status, tiles=self.tiles)
        return res

    def _fine(self, k, r, rowpack):
        from .engine import FitzCandidates, run_pairs_device
        b = self.bases[k]
        fc = FitzCandidates(r.zchi2, r.penalty if b.oii is not None else None, self.zdev[k],
                            self.K, self.nfine)
        c2, _, pen = run_pairs_device(rowpack, self.srcs[k], fc.pair_t, fc.pair_z, self.status)
        return fc, c2, pen

    def launch(self):
        """Start the plan's device work (the graph replays, or the eager
        launches) without waiting for it; an event follows the scan and
        each template's fine-grid scans."""
        import torch
        if self.graphs is not None:
            self.graphs[0].replay()
            res = self.res
        else:
            res = self._scan(self.dbatch)
        ev_scan = torch.cuda.Event()
        ev_scan.record()
        outs = []
        for k in range(len(self.templates)):
            if self.graphs is not None:
                self.graphs[k + 1].replay()
                fc, c2, pen = self.fouts[k]
            else:
                fc, c2, pen = self._fine(k, res[k], self.rowpack)
            ev = torch.cuda.Event()
            ev.record()
            outs.append((res[k], fc, c2, pen, ev))
        self._cur = (ev_scan, outs)
        self._read = _read_stream()

    def _to_host(self, ev, tensors):
        """Host copies of device tensors once `ev` has completed, made on a
        side stream, so that they do not wait for the work queued after
        `ev` on the launching stream; the status word is read with them."""
        import torch
        side = self._read
        side.wait_event(ev)
        with torch.cuda.stream(side):
            out = [t.cpu().numpy() for t in tensors]
            code = int(self.status.t.item())
        if code:
            from . import _lib as L
            L.check(code, "zfind device plan")
        return out

    def coarse(self):
        """calc_zchi2_targets' results of the batch (after launch()): waits
        for the fused scan only."""
        ev_scan, outs = self._cur
        results = {t.id: {} for t in self.local}
        for t, (r, fc, c2, pen, ev) in zip(self.templates, outs):
            ft = t.template.full_type
            zc, co, pe = self._to_host(ev_scan, (r.zchi2, r.zcoeff, r.penalty))
            for i, tg in enumerate(self.local):
                results[tg.id][ft] = dict(redshifts=t.template.redshifts, zchi2=zc[i],
                                          penalty=pe[i], zcoeff=co[i])
        return results

    def fine(self, k):
        """fitz.PrecomputedFine of template k (after launch()): waits for
        that template's candidates and fine-grid scans only."""
        ev_scan, outs = self._cur
        r, fc, c2, pen, ev = outs[k]
        cand, count, tie, pz, c2h, peh = self._to_host(
            ev, (fc.cand, fc.count, fc.tie, fc.pair_z, c2, pen))
        shape = (len(self.local), self.K, self.nfine)
        c2h = c2h.reshape(shape)
        if self.bases[k].oii is not None:
            c2h = c2h + peh.reshape(shape)
        return _fitz.PrecomputedFine(cand, count, tie, pz.reshape(shape), c2h)


class _LazyFine:
    """fitz.PrecomputedFine per template full_type, read back from the plan
    when first asked for (so the host refines one template while the
    device still scans the fine grids of the next ones)."""

    def __init__(self, plan):
        self.plan = plan
        self.index = {t.template.full_type: k for k, t in enumerate(plan.templates)}
        self.done = {}

    def get(self, ft):
        if ft not in self.done:
            self.done[ft] = self.plan.fine(self.index[ft])
        return self.done[ft]


_read_streams = {}


def _read_stream():
    """One stream per device for the plan's read-backs."""
    import torch
    d = torch.cuda.current_device()
    if d not in _read_streams:
        _read_streams[d] = torch.cuda.Stream()
    return _read_streams[d]



def _refine_all(templates, sort, local, results, archetypes, nminima, use_gpu, deg_legendre,
                zminfit_npoints, per_camera, n_nearest, prior_sigma, layout, rowpack, refine,
                pres):
    """fitz of every template over the local targets (zfind.py:330-363),
    in redrock's template order; each result goes to results[id][ft]['zfit']."""
    for t in np.array(list(templates), dtype=object)[sort] if local else []:
        ft = t.template.full_type
        archetype = archetypes.get(t.template._rrtype) if archetypes else None
        chi2 = [results[tg.id][ft]['zchi2'] + results[tg.id][ft]['penalty'] for tg in local]
        fits = _fitz.fitz_targets(chi2, t.template.redshifts, local, t.template,
                                  nminima=nminima, archetype=archetype, use_gpu=use_gpu,
                                  deg_legendre=deg_legendre, zminfit_npoints=zminfit_npoints,
                                  per_camera=per_camera, n_nearest=n_nearest,
                                  prior_sigma=prior_sigma, layout=layout, rowpack=rowpack,
                                  refine=refine, pre=None if pres is None else pres.get(ft))
        for tg, zf in zip(local, fits):
            results[tg.id][ft]['zfit'] = zf


def zfind(targets, templates, mp_procs=1, nminima=3, archetypes=None, priors=None,
          chi2_scan=None, use_gpu=True, zminfit_npoints=15, per_camera=None, deg_legendre=None,
          n_nearest=None, prior_sigma=None, ncamera=None, refine="parabola", graph=False):
    if priors is not None and not hasattr(priors, 'eval'):
        from .priors import Priors
        priors = Priors(priors)
    comm = targets.comm
    local = list(targets.local())
    # wavegrids() is collective when the targets have a communicator: every
    # rank calls it, with or without local targets
    dwave = targets.wavegrids()
    layout = GridLayout.from_dwave(dwave) if local else None
    pres = None
    if graph and chi2_scan is None and priors is None and local \
            and not archetypes \
            and all(solve_code(t.template) == _lib.RR_SOLVE_PCA for t in templates):
        # scan, candidates and fine grids on the device in one graph
        nfine = 15 if zminfit_npoints is None else zminfit_npoints
        # the plan (device buffers and the captured graph) is kept for the
        # same target and template objects, so that a repeated call replays
        # the graph; like the packed-target cache it is keyed by identity
        from .zscan import _plan_cache
        key = ("plan", layout.signature, nminima, nfine)
        plan = _plan_cache.get(key, list(local) + list(templates),
                               lambda: DeviceFitzPlan(local, templates, layout, nminima=nminima,
                                                      nfine=nfine))
        plan.launch()
        results = plan.coarse()
        pres = _LazyFine(plan)
    elif chi2_scan is None:
        results = calc_zchi2_targets(targets, templates, mp_procs=mp_procs)
    else:
        # the coarse scans of a details file (zfind.py:298-301)
        from .results import read_zscan_redrock
        results = read_zscan_redrock(chi2_scan)
    if priors is not None:
        # redshift prior on the coarse chi2 of every template (zfind.py:318-322)
        for tg in results.keys():
            for ft in results[tg].keys():
                results[tg][ft]['zchi2'] += priors.eval(tg, results[tg][ft]['redshifts'])
    # the targets' packed rows for the fine-grid pair scans do not depend on
    # the template: pack them once for every template's refinement (the
    # device plan has them already)
    if pres is not None:
        rowpack, layout = pres.plan.rowpack, pres.plan.layout
    else:
        rowpack = RowPack.from_targets(local, layout) if local else None
    sort = np.array([t.template.full_type for t in templates]).argsort()
    arch = None
    if archetypes:
        all_spectypes = []
        for t in templates:
            if t.template.template_type not in all_spectypes:
                all_spectypes.append(t.template.template_type)
        arch = dict(spectypes=list(archetypes.keys()), all_spectypes=all_spectypes,
                    n_nearest=n_nearest)
    # with the device plan, the host-driven pair launches of the refinement
    # (further candidates, single-z fits) go to the plan's read-back stream:
    # they need only the packed rows and template arrays, so they need not
    # queue behind the graphs of the templates not yet refined
    import contextlib
    import torch
    on_side = torch.cuda.stream(pres.plan._read) if pres is not None \
        else contextlib.nullcontext()
    with on_side:
        _refine_all(templates, sort, local, results, archetypes, nminima, use_gpu, deg_legendre,
                    zminfit_npoints, per_camera, n_nearest, prior_sigma, layout, rowpack,
                    refine, pres)
    if pres is not None:
        torch.cuda.current_stream().wait_stream(pres.plan._read)
    for tg in local:
        results[tg.id]['meta'] = tg.meta
    if comm is not None and comm.size > 1:
        # every rank's results on rank 0, rank order kept (zfind.py:416-456)
        parts = comm.gather(results, root=0)
        comm.barrier()
        if comm.rank != 0:
            return None, None
        allresults = {}
        for part in parts:
            allresults.update(part)
    else:
        allresults = results
    tids = list(targets.all_target_ids)
    fits_list = []
    for tid in tids:
        fits_list.append([(ft, allresults[tid][ft]['zfit']) for ft in allresults[tid]
                          if ft != 'meta'])
        for ft in allresults[tid]:
            if ft != 'meta':
                del allresults[tid][ft]['zfit']
    batch = _finalise_batch(tids, fits_list, nminima) if arch is None else None
    if batch is not None:
        allzfit = {'targetid': batch['targetid']}
        allzfit.update((k, v) for k, v in batch.items() if k != 'targetid')
    else:
        rows = [_finalise_target(tid, fits, nminima, arch) for tid, fits in zip(tids, fits_list)]
        # stack the per-target tables (astropy.table.vstack equivalent)
        cols = ['targetid'] + [k for k in rows[0] if k != 'targetid']
        allzfit = {}
        for k in cols:
            allzfit[k] = np.concatenate([r[k] for r in rows], axis=0)
    for k in list(allzfit):
        if 'pca' in k.lower():
            allzfit[k] = allzfit.pop(k)
    metakeys = sorted(k for k in allresults[allzfit['targetid'][0]]['meta'].keys()
                      if not k.endswith('_datatype'))
    for mk in metakeys:
        dt = allresults[allzfit['targetid'][0]]['meta'].get(mk + '_datatype')
        allzfit[mk] = np.array([allresults[x]['meta'][mk] for x in allzfit['targetid']], dtype=dt)
    for tid in targets.all_target_ids:
        del allresults[tid]['meta']
    if allzfit['subtype'].dtype != '<U20':
        ml = max(20, max(len(s) for s in allzfit['subtype']))
        allzfit['subtype'] = allzfit['subtype'].astype(f'<U{ml}')
    if allzfit['spectype'].dtype != '<U6':
        allzfit['spectype'] = allzfit['spectype'].astype('<U6')
    maxcoeff = np.max([t.template.nbasis for t in templates])
    if archetypes and per_camera:
        maxcoeff = max(maxcoeff, ncamera * deg_legendre + (1 if n_nearest is None else n_nearest))
    co = allzfit['coeff']
    ntarg, ncoeff = (co.shape[0], 1) if co.ndim == 1 else co.shape
    if ncoeff != maxcoeff:
        c = np.zeros((ntarg, maxcoeff), dtype=co.dtype)
        c[:, 0:ncoeff] = co if co.ndim == 2 else co[:, None]
        allzfit['coeff'] = c
    if len(np.unique(allzfit['ncoeff'])) == 1:
        m = int(np.unique(allzfit['ncoeff'])[0])
        allzfit['coeff'] = allzfit['coeff'][:, 0:m]
    return allresults, allzfit
