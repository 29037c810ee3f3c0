"""redrock's details file (redrock 0.22 results.py): the coarse chi2 scans
and the best fits of every target, in HDF5, without h5py.

    /targetids[nt]
    /zbest                       table of the best fit per target (znum 0)
    /zscan/{fulltype}/redshifts[nz]
    /zscan/{fulltype}/zchi2[nt, nz], penalty[nt, nz]      float32
    /zscan/{fulltype}/zcoeff[nt, nz, nc]                  float32
    /zfit/{targetid}/zfit        table of that target's fits

``write_zscan`` / ``read_zscan`` / ``read_zfit`` / ``read_zscan_redrock``
keep redrock's signatures and conversions (results.py:18-241); tables are
numpy structured arrays on disk and dicts of numpy columns in memory (the
form ``redrock_b200.zfind`` returns), since astropy is not required.
``read_zscan_redrock`` is what ``zfind(chi2_scan=...)`` reads to skip the
scan.  The HDF5 layer is ``redrock_b200.hdf5``.
"""

from __future__ import annotations

import os

import numpy as np

from . import hdf5
from .templates import make_fulltype, parse_fulltype

_STR_COLS = ('spectype', 'subtype', 'fitmethod', 'pca_spectype', 'pca_subtype')


def _columns(zfit):
    """dict of columns of a table given as a dict or a structured array."""
    if isinstance(zfit, dict):
        return {k: np.asarray(v) for k, v in zfit.items()}
    a = np.asarray(zfit)
    return {k: a[k] for k in a.dtype.names}


def _structured(cols, rows=None):
    names = list(cols)
    arrs = [np.asarray(cols[k]) if rows is None else np.asarray(cols[k])[rows] for k in names]
    n = len(arrs[0])
    dt = np.dtype([(k, a.dtype, a.shape[1:]) for k, a in zip(names, arrs)])
    out = np.zeros(n, dtype=dt)
    for k, a in zip(names, arrs):
        out[k] = a
    return out


def write_zscan(filename, zscan, zfit, clobber=False):
    """Write zfind's results (results.py:18-97): ``zscan`` the nested dict
    zscan[targetid][fulltype] of redshifts / zchi2 / penalty / zcoeff,
    ``zfit`` the table of fits."""
    filename = os.path.expandvars(filename)
    if clobber and os.path.exists(filename):
        os.remove(filename)
    outdir = os.path.dirname(os.path.abspath(filename))
    if not os.path.exists(outdir):
        os.makedirs(outdir)
    zfit = dict(_columns(zfit))
    for c in _STR_COLS:
        if c in zfit and zfit[c].dtype.kind == 'U':
            zfit[c] = np.char.encode(zfit[c], 'ascii')
    for c in ['zerr', 'chi2', 'zz', 'zzchi2', 'coeff', 'deltachi2']:
        zfit[c] = zfit[c].astype(np.float32)
    zfit['zwarn'] = zfit['zwarn'].astype(np.int32)
    zfit['npixels'] = zfit['npixels'].astype(np.int32)
    zfit['znum'] = zfit['znum'].astype(np.int8)
    zfit['ncoeff'] = zfit['ncoeff'].astype(np.int8)
    best = np.nonzero(zfit['znum'] == 0)[0]
    zbest = {k: v[best] for k, v in zfit.items() if k != 'znum'}
    targetids = np.asarray(zbest['targetid'])
    spectypes = list(zscan[targetids[0]].keys())
    tree = {'targetids': targetids, 'zbest': _structured(zbest), 'zscan': {}, 'zfit': {}}
    for ft in spectypes:
        zchi2 = np.vstack([zscan[t][ft]['zchi2'].astype(np.float32) for t in targetids])
        penalty = np.vstack([zscan[t][ft]['penalty'].astype(np.float32) for t in targetids])
        zcoeff = np.vstack([zscan[t][ft]['zcoeff'].astype(np.float32)[None] for t in targetids])
        tree['zscan'][ft] = {'zchi2': zchi2, 'penalty': penalty, 'zcoeff': zcoeff,
                             'redshifts': np.asarray(zscan[targetids[0]][ft]['redshifts'])}
    for tid in targetids:
        ii = np.nonzero(zfit['targetid'] == tid)[0]
        tree['zfit'][str(tid)] = {'zfit': _structured(zfit, ii)}
    hdf5.write_file(filename, tree)


def read_zfit(filename, select_targetids=None, upper=False):
    """The stacked zfit tables (results.py:180-209), as a dict of columns
    with spectype / subtype decoded to str."""
    if np.isscalar(select_targetids):
        select_targetids = [select_targetids]
    with hdf5.File(os.path.expandvars(filename)) as fx:
        if select_targetids is None:
            select_targetids = fx['targetids'][:]
        zfit = np.hstack([fx[f'zfit/{tid}/zfit'] for tid in select_targetids])
    cols = _columns(zfit)
    for c in ('spectype', 'subtype'):
        cols[c] = cols[c].astype((str, cols[c].dtype.itemsize))
    if upper:
        cols = {k.upper(): v for k, v in cols.items()}
    return cols


def read_zscan(filename, select_targetids=None, upper=False, nozfit=False):
    """zscan[targetid][fulltype] (redshifts, zchi2, penalty, zcoeff and the
    target's zfit rows of that type), and the zfit table (results.py:100-178)."""
    if np.isscalar(select_targetids):
        select_targetids = [select_targetids]
    with hdf5.File(os.path.expandvars(filename)) as fx:
        targetids = fx['targetids']
        fulltypes = fx['zscan'].keys()
        if select_targetids is not None:
            indx = np.where(np.isin(targetids, select_targetids))[0]
        else:
            indx = np.arange(len(targetids))
        zscan = {t: {ft: {} for ft in fulltypes} for t in targetids[indx]}
        for ft in fulltypes:
            zchi2 = fx[f'/zscan/{ft}/zchi2']
            penalty = fx[f'/zscan/{ft}/penalty']
            zcoeff = fx[f'/zscan/{ft}/zcoeff']
            redshifts = fx[f'/zscan/{ft}/redshifts']
            for i, t in zip(indx, targetids[indx]):
                zscan[t][ft].update(redshifts=redshifts, zchi2=zchi2[i], penalty=penalty[i],
                                    zcoeff=zcoeff[i])
    if nozfit:
        return zscan
    zfit = read_zfit(filename, select_targetids=select_targetids, upper=upper)
    tc, sc, uc = ('TARGETID', 'SPECTYPE', 'SUBTYPE') if upper else \
        ('targetid', 'spectype', 'subtype')
    keys = list(zip(zfit[tc], zfit[sc], zfit[uc]))
    for key in sorted(set(keys)):
        rows = np.array([k == key for k in keys])
        zscan[key[0]][make_fulltype(key[1], key[2])]['zfit'] = \
            {k: v[rows] for k, v in zfit.items()}
    return zscan, zfit


def read_zscan_redrock(filename):
    """results[targetid][fulltype] = redshifts / zchi2 / penalty / zcoeff,
    the form zfind's scan produces (results.py:212-241)."""
    with hdf5.File(os.path.expandvars(filename)) as fx:
        targetids = fx['targetids']
        spectypes = fx['zscan'].keys()
        tmp = {ft: {k: fx[f'/zscan/{ft}/{k}'] for k in ('redshifts', 'zchi2', 'penalty', 'zcoeff')}
               for ft in spectypes}
    return {tg: {ft: {'redshifts': tmp[ft]['redshifts'], 'zchi2': tmp[ft]['zchi2'][i],
                      'penalty': tmp[ft]['penalty'][i], 'zcoeff': tmp[ft]['zcoeff'][i]}
                 for ft in spectypes} for i, tg in enumerate(targetids)}


__all__ = ['write_zscan', 'read_zscan', 'read_zfit', 'read_zscan_redrock', 'parse_fulltype']
