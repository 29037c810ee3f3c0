"""Import an unmodified redrock for the tests and the fixture generators.

redrock needs astropy and fitsio only for file I/O and for zfind's output
table; neither is installed here, so they are stood in by empty modules and
a dict-based Table that leaves redrock's numbers untouched.
"""

import os
import sys
import types

import numpy as np



def import_redrock(path=None):
    """Import redrock from ``path`` (default $REDROCK_PY) with astropy and
    fitsio stood in; returns the package."""
    path = path or os.environ.get("REDROCK_PY")
    if not path:
        sys.exit("set REDROCK_PY to the directory that holds redrock's 'redrock' package")
    for name in ["astropy", "astropy.io", "astropy.io.fits", "astropy.table", "fitsio"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["astropy.io.fits"].open = None
    sys.modules["astropy.table"].Table = None
    sys.modules["fitsio"].FITS = None
    sys.modules["astropy"].io = sys.modules["astropy.io"]
    sys.modules["astropy"].table = sys.modules["astropy.table"]
    sys.modules["astropy.io"].fits = sys.modules["astropy.io.fits"]
    sys.path.insert(0, path)
    import redrock.zscan
    import redrock.rebin
    import redrock.igm
    import redrock.templates
    import redrock.targets
    import redrock.fitz
    return redrock


class _Column(np.ndarray):
    """Stand-in for astropy.table.Column (array with a name)."""

    def __new__(cls, data, name=None, dtype=None):
        obj = np.asarray(data, dtype=dtype).view(cls)
        obj.name = name
        return obj


class _Table(dict):
    """Minimal stand-in for astropy.table.Table as zfind uses it (dict of
    columns; the redrock numbers are untouched)."""

    def __init__(self, cols=None):
        super().__init__()
        for k, v in (cols or {}).items():
            self[k] = np.asarray(v)

    @property
    def colnames(self):
        return list(self.keys())

    @property
    def columns(self):
        return self

    def move_to_end(self, key, last=True):
        v = self.pop(key)
        if last:
            self[key] = v
        else:
            items = list(self.items())
            self.clear()
            self[key] = v
            for k, x in items:
                self[k] = x

    def add_column(self, col):
        self[col.name] = np.asarray(col)

    def replace_column(self, name, col):
        self[name] = np.asarray(col)


def _vstack(tables):
    out = _Table()
    for k in tables[0].keys():
        out[k] = np.concatenate([np.asarray(t[k]) for t in tables], axis=0)
    return out




def install_table_stubs():
    """astropy.table.Table / vstack / Column as used by redrock's zfind."""
    sys.modules["astropy.table"].Table = _Table
    sys.modules["astropy.table"].vstack = _vstack
    sys.modules["astropy.table"].Column = _Column


def ref_targets(rr, specs):
    """redrock Target objects (its own Spectrum with a scipy DIA R) from
    synthetic target specs."""
    import scipy.sparse
    out = []
    for t in specs:
        spectra = []
        for s in t.spectra:
            npix = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(npix, npix))
            spectra.append(rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R,
                                               band=s.band))
        out.append(rr.targets.Target(t.targetid, spectra))
    return out


def ref_template(rr, ts):
    """redrock Template from a synthetic template spec."""
    return rr.templates.Template(spectype=ts.spectype, subtype=ts.subtype,
                                 redshifts=ts.redshifts, wave=ts.wave, flux=ts.flux,
                                 method=ts.method, igm_model=ts.igm_model)
