"""Fine-grid refinement of the coarse chi2 minima on the GPU (redrock fitz).

Same contract as redrock 0.22 ``fitz.fitz`` (fitz.py:133-395) for PCA
templates: for each coarse minimum (best first) that is more than
max_velo_diff away from the results so far, scan a ``zminfit_npoints`` grid
between its neighbours, fit a parabola to the three points around the best
one, fit the template once more at the parabola minimum, set ZWARN bits, and
return the results sorted by chi2.

All chi2 evaluations run in the pair-scan kernel (``rr_zscan_pairs``): one
launch per template evaluates the fine grids of every target's candidate
minima (each target at its own redshifts), and one more launch does the
single-z fits at the parabola minima.  Templates with a bounded solve (NMF /
NNLS / BVLS) use the same launches with the kernel's bounded solvers and
the direct-residual chi2 of calc_zchi2_batch.  The sequential candidate logic is
replayed on the host with the precomputed fine grids (candidates beyond the
first batch are fetched in further launches only for targets that need
them), so the decisions are redrock's.

``fitz_targets`` is the batched entry point (many targets, one template);
``fitz`` keeps redrock's single-target signature.  With an archetype set,
each refined minimum is then fitted with every archetype
(``archetype.get_best_archetype``: one batched bounded solve on the device)
and the result carries the archetype's chi2, coefficients, Legendre
coefficients and name next to the template's own coefficients
(fitz.py:331-357).
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import GridLayout, RowPack, TemplateSource, pair_ranges_ok, run_pairs

C_KMS = 299792.458          # scipy.constants.speed_of_light / 1000
MAX_VELO_DIFF = 1000.0      # constants.py:7
MAX_VELO_DIFF_STAR = 100.0  # constants.py:8
Z_FITLIMIT = 2 ** 5         # zwarning.py:20
BAD_MINFIT = 2 ** 10        # zwarning.py:25


def prior_on_coeffs(n_nbh, deg_legendre, sigma, ncamera):
    """Diagonal prior 1/sigma^2 on the Legendre coefficients, none on the
    n_nbh archetype coefficients (fitz.py:113-130)."""
    nbasis = n_nbh + deg_legendre * ncamera
    prior = np.zeros((nbasis, nbasis), dtype='float64')
    np.fill_diagonal(prior, 1 / (sigma ** 2))
    for i in range(n_nbh):
        prior[i][i] = 0.
    return prior


def _stack_rows(vals):
    """np.vstack of one result column over many minima, when every value
    has the same type (and, for strings, length; for arrays, shape):
    scalars -> (n, 1), 1-D arrays -> (n, len), 2-D arrays concatenated.
    None for a mixed column."""
    if not vals:
        return None
    v0 = vals[0]
    t0 = type(v0)
    if isinstance(v0, _SCALARS):
        if isinstance(v0, (str, np.str_)):
            n0 = len(v0)
            if not all(type(v) is t0 and len(v) == n0 for v in vals):
                return None
        elif not all(type(v) is t0 for v in vals):
            return None
        return np.array(vals).reshape(len(vals), 1)
    if isinstance(v0, np.ndarray) and v0.ndim in (1, 2):
        sh, dt = v0.shape, v0.dtype
        if not all(type(v) is np.ndarray and v.shape == sh and v.dtype == dt for v in vals):
            return None
        return np.stack(vals) if v0.ndim == 1 else np.concatenate(vals, axis=0)
    return None


def _vstack(vals):
    """np.vstack of the values, with a faster path for all-scalar lists
    (the same (n, 1) array and dtype)."""
    if all(isinstance(v, _SCALARS) for v in vals):
        return np.array(vals).reshape(len(vals), 1)
    return np.vstack(vals)


_SCALARS = (float, int, str, np.floating, np.integer, np.str_)


def _near_any(z, zprev, maxv):
    """np.any(np.abs(get_dv(z, np.array(zprev))) < maxv), elementwise in
    the same operation order, without building arrays."""
    for zr in zprev:
        if abs(C_KMS * (z - zr) / (1.0 + zr)) < maxv:
            return True
    return False


def get_dv(z, zref):
    """Velocity difference in km/s (fitz.py:28-43)."""
    return C_KMS * (z - zref) / (1.0 + zref)


def find_minima(x):
    """Indices of local minima including edges, sorted by value (fitz.py:46-67):
    x[i] <= both neighbours (<=: plateaus count), the first and last point
    compared with their one neighbour, ordered by np.argsort of the values."""
    x = np.asarray(x)
    is_min = np.ones(len(x), dtype=bool)
    if len(x) > 1:
        is_min[1:] = x[1:] <= x[:-1]
        is_min[:-1] &= x[:-1] <= x[1:]
    ii = np.flatnonzero(is_min)
    return ii[np.argsort(x[ii])]


def minfit(x, y):
    """y = y0 + ((x - x0)/xerr)^2 through 3 points (fitz.py:70-110)."""
    if len(x) < 3:
        return (-1, -1, -1, BAD_MINFIT)
    try:
        a, b, c = np.polyfit(x, y, 2)
    except np.linalg.LinAlgError:
        return (-1, -1, -1, BAD_MINFIT)
    if a == 0.0:
        return (-1, -1, -1, BAD_MINFIT)
    x0 = -b / (2 * a)
    y0 = -(b ** 2) / (4 * a) + c
    zwarn = 0
    if (x0 <= np.min(x)) or (np.max(x) <= x0):
        zwarn |= BAD_MINFIT
    if (y0 <= 0.):
        zwarn |= BAD_MINFIT
    if a > 0.0:
        xerr = 1 / np.sqrt(a)
    else:
        xerr = 1 / np.sqrt(-a)
        zwarn |= BAD_MINFIT
    return (x0, xerr, y0, zwarn)


def minfit_batch(x, y):
    """minfit for K triples at once: x, y (K, 3) -> x0, xerr, y0 (K,) and
    zwarn (K,) int.

    The parabola through three points is the Newton form
    y0 + d1 (x - x0) + a (x - x0)(x - x1), a = the second divided
    difference; its vertex differs from np.polyfit's least-squares fit by
    rounding only (~1e-10 in z on redrock's fine grids, below the ~1e-9 the
    FP64 chi2 noise itself moves it).  Triples where that form is not well
    determined -- non-finite values, repeated x, or a second difference
    within 1e-9 of the values' scale (flat or constant chi2, e.g.
    HUGE_CHI2) -- go through minfit, so degenerate cases return exactly
    what redrock's polyfit returns."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    k = len(x)
    x0 = np.empty(k)
    xerr = np.empty(k)
    y0 = np.empty(k)
    zwarn = np.zeros(k, dtype=np.int64)
    if k == 0:
        return x0, xerr, y0, zwarn
    with np.errstate(all='ignore'):
        h0 = x[:, 1] - x[:, 0]
        h1 = x[:, 2] - x[:, 1]
        d1 = (y[:, 1] - y[:, 0]) / h0
        d2 = (y[:, 2] - y[:, 1]) / h1
        a = (d2 - d1) / (x[:, 2] - x[:, 0])
        dd = y[:, 0] - 2.0 * y[:, 1] + y[:, 2]
        scale = np.max(np.abs(y), axis=1)
        good = (np.all(np.isfinite(x), axis=1) & np.all(np.isfinite(y), axis=1)
                & (h0 > 0) & (h1 > 0) & (np.abs(dd) > 1e-9 * scale) & (a != 0.0))
        xv = 0.5 * (x[:, 0] + x[:, 1]) - d1 / (2.0 * a)
        yv = y[:, 0] + d1 * (xv - x[:, 0]) + a * (xv - x[:, 0]) * (xv - x[:, 1])
        sig = 1.0 / np.sqrt(np.abs(a))
    x0[:] = xv
    y0[:] = yv
    xerr[:] = sig
    zwarn[(xv <= np.min(x, axis=1)) | (np.max(x, axis=1) <= xv)] |= BAD_MINFIT
    zwarn[yv <= 0.0] |= BAD_MINFIT
    zwarn[~(a > 0.0)] |= BAD_MINFIT
    for i in np.nonzero(~good)[0]:
        x0[i], xerr[i], y0[i], zwarn[i] = minfit(x[i], y[i])
    return x0, xerr, y0, zwarn


class _NewtonCtx:
    """The pair context refine_newton expects, built from a _Refiner."""

    def __init__(self, ref):
        self.layout = ref.layout
        self.rows = ref.rows
        self.src = ref.src


class _Refiner:
    """Device state shared by the pair launches of one fitz_targets call."""

    def __init__(self, targets, template, layout=None, rowpack=None):
        if layout is None:
            dwave = {}
            for t in targets:
                for s in t.spectra:
                    dwave.setdefault(s.wavehash, s.wave)
            layout = GridLayout.from_dwave(dwave)
        self.layout = layout
        self.rows = rowpack or RowPack.from_targets(targets, layout)
        self.src = TemplateSource.from_template(template)
        self.oii = getattr(template, "OIItemplate", None)

    def scan(self, tidx, z):
        """chi2 (+ [OII] penalty for the fine grids) and coefficients at the
        given (target, z) pairs; pairs outside the template range -> None."""
        z = np.asarray(z, dtype=np.float64)
        tidx = np.asarray(tidx, dtype=np.int32)
        ok = pair_ranges_ok(self.src, self.layout, z)
        chi2 = np.full(len(z), np.nan)
        pen = np.zeros(len(z))
        coeff = np.full((len(z), self.src.nbasis), np.nan)
        sel = np.nonzero(ok)[0]
        if len(sel):
            c2, co, pe = run_pairs(self.rows, self.src, tidx[sel], z[sel])
            chi2[sel] = c2.cpu().numpy()
            coeff[sel] = co.cpu().numpy()
            pen[sel] = pe.cpu().numpy()
        return chi2, coeff, pen, ok


class PrecomputedFine:
    """Host copies of device-evaluated fitz candidates for one template
    (rr_fitz_candidates + one rr_zscan_pairs launch over their fine grids):
    cand [T][K], count [T], tie [T], zz [T][K][nfine] and c2 [T][K][nfine]
    (chi2, plus the [OII] penalty when the template has one)."""

    def __init__(self, cand, count, tie, zz, c2):
        self.cand = np.asarray(cand)
        self.count = np.asarray(count)
        self.tie = np.asarray(tie).astype(bool)
        self.K = self.cand.shape[1]
        self.zz = np.asarray(zz)
        self.c2 = np.asarray(c2)


def fitz_targets(zchi2_list, redshifts, targets, template, nminima=3, archetype=None,
                 use_gpu=True, deg_legendre=None, zminfit_npoints=15, per_camera=False,
                 n_nearest=None, prior_sigma=None, layout=None, rowpack=None, batch_extra=0,
                 refine="parabola", pre=None):
    """redrock's fitz for many targets of one template; returns a list of
    per-target result dicts (the same dict-of-arrays fitz returns).

    ``pre`` (optional): candidates and fine grids already evaluated on the
    device for every target (``PrecomputedFine``: the K lowest minima of
    each row from rr_fitz_candidates and the chi2 of their fine grids from
    one pair launch).  Rows it covers skip the host find_minima and the
    first launch; a row flagged as tied, or one that needs more than K
    candidates, continues on the host exactly as without ``pre``.

    The first launch evaluates each target's first nminima + batch_extra
    candidate minima; targets whose candidates fall within max_velo_diff of
    one another get further launches for the next ones (0 extra measured
    fastest: most targets need no more than nminima).

    refine="parabola" is redrock's minfit through the three fine-grid points
    around the best one.  refine="newton" instead runs safeguarded Newton
    steps on chi2(z) (the adjoint kernel's dchi2/dz and envelope curvature)
    inside that three-point cell, with zerr = sqrt(2 / d2chi2/dz2); the
    decisions that follow (ZWARN bits, velocity separation) are the same."""
    from . import _lib
    from .templates import solve_code
    redshifts = np.asarray(redshifts)
    nz = 15 if zminfit_npoints is None else zminfit_npoints
    maxv = MAX_VELO_DIFF_STAR if template.template_type == 'STAR' else MAX_VELO_DIFF
    if refine == "newton" and solve_code(template) != _lib.RR_SOLVE_PCA:
        raise NotImplementedError("Newton refinement needs a PCA template (the adjoint of a "
                                  "bounded solve is not implemented)")
    ref = _Refiner(targets, template, layout, rowpack)
    has_oii = ref.oii is not None

    ntg = len(targets)
    use_pre = [pre is not None and not pre.tie[j] for j in range(ntg)]
    # device candidate lists are the first K entries of find_minima's order
    # (rows without ties); partial rows get the full host list when the
    # replay needs more of them
    cands = [pre.cand[j, :pre.count[j]] if use_pre[j] else find_minima(np.asarray(z))
             for j, z in enumerate(zchi2_list)]
    partial = [use_pre[j] and pre.count[j] == pre.K for j in range(ntg)]
    pos = [int(pre.count[j]) if use_pre[j] else 0 for j in range(ntg)]
    fine = [dict() for _ in range(ntg)]   # imin -> (zz, zzchi2)
    results = [list() for _ in range(ntg)]
    state = [dict(ci=0) for _ in range(ntg)]   # replay cursor per target
    done = [False] * ntg
    want = nminima + batch_extra

    def refine_fits(tj, zz3, c23, zzall, c2all):
        """Per candidate (z, zerr, zwarn, chi2, zmin) after the refinement
        and redrock's checks on it (fitz.py:263-280): a minimum outside the
        fine grid is BAD_MINFIT and replaced by the grid's first lowest
        point; Z_FITLIMIT when it or the refined minimum is outside
        redshifts[1:-1]."""
        if refine == "newton":
            fx0, ferr, fy0, fzw = newton_batch(tj, zz3)
        else:
            fx0, ferr, fy0, fzw = minfit_batch(zz3, c23)
        fzw = np.asarray(fzw, dtype=np.int64)
        rows = np.arange(len(fx0))
        kmin = np.argmin(c2all, axis=1)
        off = (fx0 < zzall[:, 0]) | (fx0 > zzall[:, -1])
        zbest = np.where(off, zzall[rows, kmin], fx0)
        chi2b = np.where(off, c2all[rows, kmin], fy0)
        zw = fzw | np.where(off, BAD_MINFIT, 0)
        lim = (zbest < redshifts[1]) | (zbest > redshifts[-2]) | \
            (fx0 < redshifts[1]) | (fx0 > redshifts[-2])
        zw = zw | np.where(lim, Z_FITLIMIT, 0)
        return list(zip(zbest.tolist(), ferr.tolist(), zw.tolist(), chi2b.tolist(),
                        fx0.tolist()))

    def fetch(tlist, count):
        tid, key = [], []
        for j in tlist:
            if partial[j] and pos[j] >= len(cands[j]):
                cands[j] = find_minima(np.asarray(zchi2_list[j]))
                partial[j] = False
            c = cands[j]
            for imin in c[pos[j]:pos[j] + count]:
                tid += [j] * nz
                key.append((j, int(imin)))
            pos[j] = min(len(c), pos[j] + count)
        if not key:
            return
        imins = np.array([k[1] for k in key])
        lo = redshifts[np.maximum(0, imins - 1)]
        hi = redshifts[np.minimum(imins + 1, len(redshifts) - 1)]
        if nz > 1 and np.all(hi != lo):
            # np.linspace over all candidates at once: the same
            # start + i * ((stop - start) / (nz - 1)) per row, last = stop
            zzall = np.linspace(lo, hi, nz, axis=1)
        else:
            zzall = np.stack([np.linspace(a, b, nz) for a, b in zip(lo, hi)])
        chi2, _, pen, ok = ref.scan(tid, zzall.reshape(-1))
        if not np.all(ok):
            raise ValueError('edges must be within input x range')
        c2all = chi2.reshape(len(key), nz).copy()
        if has_oii:
            c2all += pen.reshape(len(key), nz)
        fits = [None] * len(key)
        if nz >= 3:
            # every candidate's refinement in one pass (the replay below only
            # picks the ones it reaches): the parabola through the three
            # fine-grid points around the best one, or Newton steps inside
            # that cell for all candidates in one batch of pair launches
            ib = np.clip(np.argmin(c2all, axis=1), 1, nz - 2)
            cols = ib[:, None] + np.arange(-1, 2)[None, :]
            rows = np.arange(len(key))[:, None]
            fits = refine_fits([k[0] for k in key], zzall[rows, cols], c2all[rows, cols],
                               zzall, c2all)
        for n_, (j, imin) in enumerate(key):
            fine[j][imin] = (zzall[n_], c2all[n_], fits[n_])

    newton_ctx = {}

    def newton_batch(tj, z3):
        # safeguarded Newton in [z3[:, 0], z3[:, 2]] from z3[:, 1], all
        # candidates together: one pair-gradient launch per Newton iteration
        from .adjoint import refine_newton
        ctx = newton_ctx.get("ctx")
        if ctx is None:
            ctx = newton_ctx["ctx"] = _NewtonCtx(ref)
        # the objective of the fine grid: chi2 plus the [OII] penalty
        z, c2, co, g, h, _ = refine_newton(ctx, np.asarray(tj, dtype=np.int32), z3[:, 1],
                                           z3[:, 0], z3[:, 2], penalty=has_oii)
        zwarn = np.zeros(len(z), dtype=np.int64)
        pos_h = h > 0
        sigma = np.where(pos_h, np.sqrt(2.0 / np.where(pos_h, h, 1.0)), -1.0)
        zwarn[~pos_h] |= BAD_MINFIT
        zwarn[~((z3[:, 0] < z) & (z < z3[:, 2]))] |= BAD_MINFIT
        return z, sigma, c2, zwarn

    if pre is not None and any(use_pre):
        # the device-evaluated candidates: their fine grids and one batch of
        # refinements, as fetch() would have made them
        key = [(j, int(pre.cand[j, k])) for j in range(ntg) if use_pre[j]
               for k in range(int(pre.count[j]))]
        jj = np.array([k[0] for k in key])
        kk = np.concatenate([np.arange(int(pre.count[j])) for j in range(ntg) if use_pre[j]])
        zzp = pre.zz[jj, kk]
        c2p = pre.c2[jj, kk]
        fits = [None] * len(key)
        if nz >= 3:
            ib = np.clip(np.argmin(c2p, axis=1), 1, nz - 2)
            cols = ib[:, None] + np.arange(-1, 2)[None, :]
            rows = np.arange(len(key))[:, None]
            fits = refine_fits(jj.tolist(), zzp[rows, cols], c2p[rows, cols], zzp, c2p)
        for n_, (j, imin) in enumerate(key):
            fine[j][imin] = (zzp[n_], c2p[n_], fits[n_])

    pending_final = []   # (target, result dict, zmin)
    active = list(range(ntg))
    fetch([j for j in active if not use_pre[j]], want)
    while active:
        need_more = []
        for j in active:
            c = cands[j]
            st = state[j]
            while st['ci'] < len(c) and len(results[j]) < nminima:
                imin = c[st['ci']]
                if imin not in fine[j]:
                    break        # not fetched yet
                st['ci'] += 1
                zprev = [tmp['z'] for tmp in results[j]]
                if _near_any(redshifts[imin], zprev, maxv):
                    continue
                zz, zzchi2, fit = fine[j][imin]
                if fit is not None:
                    zbest, zerr, zwarn, chi2min, zmin = fit
                else:
                    i = min(max(np.argmin(zzchi2), 1), len(zz) - 2)
                    zmin, sigma, chi2min, zwarn = minfit(zz[i - 1:i + 2], zzchi2[i - 1:i + 2])
                    zbest = zmin
                    zerr = sigma
                    if zbest < zz[0] or zbest > zz[-1]:
                        zwarn |= BAD_MINFIT
                        k = np.where(zzchi2 == np.min(zzchi2))[0][0]
                        zbest = zz[k]
                        chi2min = zzchi2[k]
                    if zbest < redshifts[1] or zbest > redshifts[-2]:
                        zwarn |= Z_FITLIMIT
                    if zmin < redshifts[1] or zmin > redshifts[-2]:
                        zwarn |= Z_FITLIMIT
                if _near_any(zbest, zprev, maxv):
                    continue
                r = dict(z=zbest, zerr=zerr, zwarn=zwarn, chi2=chi2min, zz=zz, zzchi2=zzchi2,
                         coeff=None, fitmethod=template.method)
                results[j].append(r)
                pending_final.append((j, r, zmin))
            if len(results[j]) < nminima and (st['ci'] < len(c) or partial[j]):
                need_more.append(j)
        if need_more:
            fetch(need_more, want)
        active = need_more

    # single-z fits at the parabola minima (fitz.py:263-293); a minimum
    # outside the template's valid range gets zero coefficients and
    # Z_FITLIMIT | BAD_MINFIT when it is also outside the scanned range
    if pending_final:
        tj = [p[0] for p in pending_final]
        zm = np.array([p[2] for p in pending_final], dtype=np.float64)
        _, coeff, _, ok = ref.scan(tj, zm)
        for (j, r, zmin), co, good in zip(pending_final, coeff, ok):
            if good:
                r['coeff'] = co[None, :]
            elif zmin < redshifts[0] or redshifts[-1] < zmin:
                r['coeff'] = np.zeros(template.nbasis)
                r['zwarn'] |= Z_FITLIMIT
                r['zwarn'] |= BAD_MINFIT
            else:
                raise ValueError('edges must be within input x range')
        if archetype is not None:
            _archetype_fits([(targets[j], r, zmin, good) for (j, r, zmin), good
                             in zip(pending_final, ok)], template, archetype, use_gpu,
                            deg_legendre, per_camera, n_nearest, prior_sigma)

    out = []
    rows, spans = [], []   # every target's sorted minima; (index, first, end)
    for j, t in enumerate(targets):
        res = results[j]
        ii = np.argsort([tmp['chi2'] for tmp in res])
        res = [res[i] for i in ii]
        if len(res) == 0:
            xfloat = np.zeros((0, 1), dtype=float)
            xint = np.zeros((0, 1), dtype=int)
            xstr = np.zeros((0, 1), dtype=str)
            out.append(dict(z=xfloat, zerr=xfloat, zwarn=xint, chi2=xfloat, zz=xfloat,
                            zzchi2=xfloat, coeff=xfloat, fitmethod=xstr, npixels=xint))
            continue
        npix = 0
        for s in t.spectra:
            npix += (np.asarray(s.ivar) > 0.).sum()
        for r in res:
            r['npixels'] = npix
        spans.append((len(out), len(rows), len(rows) + len(res)))
        rows.extend(res)
        out.append(None)
    # each column stacked once over all targets' minima, then sliced per
    # target: the same arrays as a per-target np.vstack wherever the column
    # has one type and shape throughout (else per target, as before)
    keys = list(rows[0].keys()) if rows else []
    if not all(list(r.keys()) == keys for r in rows):
        keys = []
    cols = {k: _stack_rows([r[k] for r in rows]) for k in keys}
    for j, a, b in spans:
        tmp = {}
        for k in rows[a].keys():
            col = cols.get(k)
            tmp[k] = col[a:b] if col is not None else _vstack([r[k] for r in rows[a:b]])
        out[j] = tmp
    return out


def _archetype_fits(pending, template, archetype, use_gpu, deg_legendre, per_camera, n_nearest,
                    prior_sigma):
    """Replace each refined minimum's fit by the best archetype fit at its
    redshift (fitz.py:263-293, 331-357), all minima of the batch in one
    ``best_archetypes`` call when the archetype set has it (redrock's own
    Archetype is called per minimum).  The IGM transmission at the
    parabola minimum comes along as redrock computes it (none when the
    template could not be evaluated there).  redrock leaves ``ncamera``
    undefined when prior_sigma is None (a NameError); here it is the number
    of grids with per_camera, else 1, in every case."""
    from .archetypes import split_archetype_coeff
    from .igm import transmission_Lyman
    from .templates import parse_fulltype
    from .zscan import spectral_data
    items, extra = [], []
    prior = None
    # transmission_Lyman(zmin, wave) of every good minimum, one call per grid
    # (None where redrock's always_return_array=False gives None)
    tgrid = {}
    if template.igm_model not in ('None', None):
        for target, r, zmin, good in pending:
            for s in target.spectra:
                tgrid.setdefault(s.wavehash, s.wave)
    zgood = np.array([zmin for _, _, zmin, good in pending if good], dtype=np.float64)
    tvals = {}
    if len(zgood):
        for hs, wv in tgrid.items():
            tvals[hs] = np.asarray(transmission_Lyman(zgood, wv, use_gpu=False,
                                                      model=template.igm_model)).reshape(len(zgood), -1)
    igood = 0
    for target, r, zmin, good in pending:
        dwave = {s.wavehash: s.wave for s in target.spectra}
        if target.nleg != deg_legendre or getattr(target, "_legendre", None) is None:
            target.legendre(deg_legendre)
        trans = {hs: None for hs in dwave}
        if good:
            for k in dwave:
                lyman = np.min(dwave[k]) / (1. + zmin) <= 1215.67
                if k in tvals and lyman:
                    trans[k] = tvals[k][igood][None, :]
            igood += 1
            pca_coeff = np.asarray(r['coeff'])[0, :]
        else:
            pca_coeff = np.copy(r['coeff'])
        ncamera = len(dwave) if per_camera else 1
        prior = None
        if prior_sigma is not None:
            prior = prior_on_coeffs(1 if n_nearest is None else n_nearest, deg_legendre,
                                    prior_sigma, ncamera)
        items.append((target, r['z'], trans))
        extra.append((r, pca_coeff, ncamera, prior))
    if not items:
        return
    if hasattr(archetype, "best_archetypes") and len({e[3] is None for e in extra}) == 1 \
            and len({e[2] for e in extra}) == 1:
        for _, _, trans in items:
            for hs in trans:
                if trans[hs] is not None:
                    trans[hs] = trans[hs][0, :]
        fits = archetype.best_archetypes(items, per_camera, n_nearest, prior=extra[0][3])
    else:
        fits = []
        for (target, z, trans), (_, _, _, pri) in zip(items, extra):
            w, f, wf = spectral_data(target.spectra)
            dwave = {s.wavehash: s.wave for s in target.spectra}
            fits.append(archetype.get_best_archetype(target, w, f, wf, dwave, z, per_camera,
                                                     n_nearest, trans=trans, use_gpu=use_gpu,
                                                     prior=pri))
    for (chi2min, coeff, fulltype), (r, pca_coeff, ncamera, _) in zip(fits, extra):
        subtype = parse_fulltype(fulltype)[1]
        archcoeff, legcoeff = split_archetype_coeff(subtype, coeff, ncamera, deg_legendre)
        if per_camera:
            legcoeff = [np.vstack(legcoeff)]
        prev = dict(r)
        r.clear()   # redrock's key order for archetype results
        r.update(z=prev['z'], zerr=prev['zerr'], zwarn=prev['zwarn'], chi2=chi2min,
                 zz=prev['zz'], zzchi2=prev['zzchi2'], coeff=archcoeff, legcoeff=legcoeff,
                 fulltype=fulltype, fitmethod=archetype.method, pca_coeff=pca_coeff,
                 pca_spectype=template._rrtype, pca_subtype=template.sub_type)


def fitz(zchi2, redshifts, target, template, nminima=3, archetype=None, use_gpu=False,
         deg_legendre=None, zminfit_npoints=15, per_camera=False, n_nearest=None,
         prior_sigma=None):
    """redrock's single-target fitz signature (fitz.py:133)."""
    return fitz_targets([zchi2], redshifts, [target], template, nminima=nminima,
                        archetype=archetype, use_gpu=use_gpu, deg_legendre=deg_legendre,
                        zminfit_npoints=zminfit_npoints, per_camera=per_camera,
                        n_nearest=n_nearest, prior_sigma=prior_sigma)[0]
