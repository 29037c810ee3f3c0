"""Template containers with redrock's interface, bases built on the GPU.

  Template          templates.py:29-272 (constructor-from-arrays form; the
                                         OIItemplate cache :172-174)
  DistTemplate      templates.py:525-663 (rebin + IGM per wavehash :584-597)
  DistTemplatePiece templates.py:478-501

``DistTemplate`` accepts redrock's own ``Template`` objects too.  Its bases
are built once on the device by the fused rebin + IGM kernel and stay
resident; ``local.data`` (redrock's dict of (nz, npix, nbasis) arrays) is
materialised on the host only when something reads it.
"""

from __future__ import annotations

import numpy as np

from . import _lib

valid_template_methods = ('PCA', 'NMF')


def make_fulltype(spectype, subtype):
    spectype = spectype.strip()
    if subtype is not None:
        subtype = subtype.strip()
    return f'{spectype}:::{subtype}' if subtype else spectype


def parse_fulltype(fulltype):
    fulltype = fulltype.strip()
    if ':::' in fulltype:
        return tuple(fulltype.split(':::'))
    return fulltype, ''


class Template:
    def __init__(self, filename=None, spectype=None, redshifts=None, wave=None, flux=None,
                 subtype=None, method='PCA', igm_model='Inoue14', zscan_galaxy=None,
                 zscan_qso=None, zscan_star=None, version=None):
        if filename is not None:
            raise NotImplementedError("template files are read by redrock.templates.Template; "
                                      "pass arrays or a redrock Template")
        self._filename = None
        self._rrtype = spectype
        self._redshifts = redshifts
        self.wave = wave
        self.flux = flux
        self._subtype = subtype
        self._igm_model = igm_model
        self._method = method
        self._version = version
        self._nbasis = self.flux.shape[0]
        self._nwave = self.flux.shape[1]
        self.minwave = self.wave[0]
        self.maxwave = self.wave[-1]
        self.gpuwave = None
        self.gpuflux = None
        if self._method not in valid_template_methods:
            raise ValueError(f'Template method {self._method} unrecognized; '
                             f'should be one of {valid_template_methods}')
        if self._rrtype == 'GALAXY' and self._method == "PCA":
            isOII = (3724 <= self.wave) & (self.wave <= 3733)
            self.OIItemplate = self.flux[:, isOII]

    def __str__(self):
        z = self._redshifts
        return (f'{self._rrtype} {self._subtype} {self._method} IGM={self._igm_model} '
                f'z={round(z[0], 4)}-{round(z[-1], 4)}')

    __repr__ = __str__

    nbasis = property(lambda self: self._nbasis)
    nwave = property(lambda self: self._nwave)
    template_type = property(lambda self: self._rrtype)
    sub_type = property(lambda self: self._subtype)
    full_type = property(lambda self: make_fulltype(self._rrtype, self._subtype))
    version = property(lambda self: self._version)
    filename = property(lambda self: self._filename)
    redshifts = property(lambda self: self._redshifts)
    solve_matrices_algorithm = property(lambda self: self._method)
    method = property(lambda self: self._method)
    igm_model = property(lambda self: self._igm_model)

    def eval(self, coeff, wave, z, R=None):
        from .rebin import trapz_rebin
        coeff = coeff[0:self.nbasis]
        flux = self.flux.T.dot(coeff).T
        model = trapz_rebin(self.wave * (1 + z), flux, wave)
        if R is not None:
            model = R.dot(model)
        return model


def from_synth(tspec):
    return Template(spectype=tspec.spectype, subtype=tspec.subtype, redshifts=tspec.redshifts,
                    wave=tspec.wave, flux=tspec.flux, method=tspec.method,
                    igm_model=tspec.igm_model)


def solve_code(template):
    """rr_solve_method of a template's solve_matrices_algorithm
    (zscan.py:1107-1203): PCA; NMF / NNLS; BVLS; anything else is
    redrock's NotImplementedError (HUGE_CHI2)."""
    return solve_code_of(getattr(template, 'solve_matrices_algorithm', 'PCA'))


def solve_code_of(name):
    m = 'PCA' if name is None else str(name).upper()
    if m == 'PCA':
        return _lib.RR_SOLVE_PCA
    if m in ('NMF', 'NNLS'):
        return _lib.RR_SOLVE_NNLS
    if m == 'BVLS':
        return _lib.RR_SOLVE_BVLS
    return _lib.RR_SOLVE_UNSUPPORTED


def oii_sums(template):
    """Per-basis sums of the [OII] window (calc_negOII_penalty's reduction
    split as sum_j sum_b c_b O[b, j] = sum_b c_b (sum_j O[b, j]))."""
    if not hasattr(template, 'OIItemplate'):
        return None
    return np.asarray(template.OIItemplate, dtype=np.float64).sum(axis=1)


class DistTemplatePiece:
    def __init__(self, index, redshifts, data):
        self.index = index
        self.redshifts = redshifts
        self._data = data

    @property
    def data(self):
        if callable(self._data):
            self._data = self._data()
        return self._data

    @data.setter
    def data(self, v):
        self._data = v


class DistTemplate:
    """Every redshift of the template, rebinned (+ IGM) on the GPU.

    Like redrock's GPU mode (templates.py:558-563) each process holds all
    redshifts, so ``cycle()`` is a no-op.
    """

    def __init__(self, template, dwave, mp_procs=1, comm=None, use_gpu=True, gpu_mode=True):
        from .device import StatusWord
        from .engine import DeviceBasis, GridLayout, TemplateSource
        self._comm = comm
        self._template = template
        self._dwave = dwave
        self._layout = GridLayout.from_dwave(dwave)
        self.source = TemplateSource.from_template(template)
        # built asynchronously: the device status is checked when the basis
        # is first read (the scan, or the host view below)
        status = StatusWord()
        self._status = status
        self.basis = DeviceBasis.build(self.source, self._layout, status=status)
        rank = 0 if comm is None else comm.rank
        # the lazy host view holds the basis, not self: a closure over self
        # would make a reference cycle that keeps the device basis (GBs)
        # alive until the cyclic collector happens to run
        basis = self.basis

        def host_view():
            status.check("rr_build_basis")
            return basis.data_dict(as_numpy=True)
        self._piece = DistTemplatePiece(rank, template.redshifts, host_view)

    def check(self):
        """Raise if building the basis on the device reported an error."""
        self._status.check("rr_build_basis")

    @property
    def comm(self):
        return self._comm

    @property
    def template(self):
        return self._template

    @property
    def local(self):
        return self._piece

    @property
    def layout(self):
        return self._layout

    def cycle(self):
        return True
