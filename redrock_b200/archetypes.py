"""Archetype fits on the GPU (redrock 0.22 archetypes.py).

An archetype set is a few hundred rest-frame spectra of one spectral class.
At a redshift found by the template scan redrock rebins every archetype onto
the target's cameras, multiplies by the IGM transmission, appends Legendre
polynomials (one set for the whole spectrum, or one per camera) and fits
every archetype at once with a bounded least-squares solve (archetype
coefficient >= 0); the best one -- or a combination of the n nearest ones in
chi2 -- becomes the final model (archetypes.py:228-400).

Here the rebin (``rr_trapz_rebin``), the transmission, the basis assembly and
the batched solve (the plain chain with ``RR_SOLVE_BVLS`` / ``RR_SOLVE_NNLS``)
all run on the device; only the per-archetype chi2 and coefficients come
back to the host for the argmin / argsort.

``Archetype`` mirrors redrock's class.  It is built from arrays
(``Archetype(wave=..., flux=..., rrtype=..., subtype=...)`` or
``Archetype.from_synth``) or, when astropy is importable, from a
redrock-format archetype file.  redrock's own ``Archetype`` also runs on the
GPU once ``redrock_b200.install`` has rebound its ``trapz_rebin``,
``transmission_Lyman``, ``calc_zchi2_batch`` and
``per_camera_coeff_with_least_square_batch``.
"""

from __future__ import annotations

import os

import numpy as np
import torch

from .device import to_device, to_numpy
from .igm import transmission_Lyman
from .rebin import trapz_rebin
from .templates import make_fulltype
from .zscan import calc_zchi2_batch, per_camera_coeff_with_least_square_batch


def split_archetype_coeff(subtype, coeff, nbands, nleg):
    """(archetype coefficients, [Legendre coefficients per band]) of a fit
    whose subtype names ';'-separated archetypes (archetypes.py:428-443)."""
    narchetypes = len(subtype.split(';'))
    archcoeff = coeff[0:narchetypes]
    rest = coeff[narchetypes:]
    return archcoeff, [rest[i * nleg:(i + 1) * nleg] for i in range(nbands)]


def _interp(x, xp, fp):
    """Linear interpolation that extrapolates the end segments, like
    scipy's interp1d(kind='linear', fill_value='extrapolate')."""
    x = np.asarray(x, dtype=np.float64)
    y = np.interp(x, xp, fp)
    lo = x < xp[0]
    hi = x > xp[-1]
    y[lo] = fp[0] + (x[lo] - xp[0]) * (fp[1] - fp[0]) / (xp[1] - xp[0])
    y[hi] = fp[-1] + (x[hi] - xp[-1]) * (fp[-1] - fp[-2]) / (xp[-1] - xp[-2])
    return y


def _read_archetype_file(filename):
    try:
        from astropy.io import fits
    except ImportError as e:
        raise ImportError("reading a redrock archetype file needs astropy; build the "
                          "Archetype from arrays instead") from e
    with fits.open(os.path.expandvars(filename), memmap=False) as h:
        hdr = h['ARCHETYPES'].header
        flux = np.asarray(h['ARCHETYPES'].data['ARCHETYPE']).astype('float64')
        sub = [str(s).strip() for s in h['ARCHETYPES'].data['SUBTYPE']]
        wave = np.asarray(hdr['CRVAL1'] + hdr['CDELT1'] * np.arange(flux.shape[1]))
        if hdr['LOGLAM']:
            wave = 10 ** wave
        return wave, flux, hdr['RRTYPE'].strip(), sub, hdr['VERSION']


class Archetype:
    """All archetypes of one spectral class (archetypes.py:26-400)."""

    def __init__(self, filename=None, wave=None, flux=None, rrtype=None, subtype=None,
                 version=None):
        self._filename = filename
        if filename is not None:
            wave, flux, rrtype, subtype, version = _read_archetype_file(filename)
        self.flux = np.asarray(flux, dtype=np.float64)
        self._narch, self._nwave = self.flux.shape
        self._rrtype = rrtype.strip()
        # subtypes get the archetype's row number appended (archetypes.py:46-47)
        self._subtype = np.array([f"{str(s).strip()}_{i}" for i, s in enumerate(subtype)])
        self._full_type = np.array([make_fulltype(self._rrtype, s) for s in self._subtype])
        self._version = version
        self.wave = np.asarray(wave, dtype=np.float64)
        self.minwave = self.wave[0]
        self.maxwave = self.wave[-1]
        self.igm_model = 'Inoue14'
        self.method = 'ARCH'
        self._dflux = None

    @classmethod
    def from_synth(cls, spec):
        return cls(wave=spec.wave, flux=spec.flux, rrtype=spec.rrtype, subtype=spec.subtype,
                   version=spec.version)

    version = property(lambda self: self._version)
    filename = property(lambda self: self._filename)
    template_type = property(lambda self: self._rrtype)
    sub_type = property(lambda self: self._subtype)
    full_type = property(lambda self: self._full_type)

    @property
    def dflux(self):
        """The archetype fluxes on the device, copied once."""
        if self._dflux is None:
            self._dflux = to_device(self.flux)
        return self._dflux

    def rebin_template(self, index, z, dwave, trapz=True):
        """One archetype at redshift z on each grid (archetypes.py:121-127)."""
        if not trapz:
            return {hs: _interp(w / (1. + z), self.wave, self.flux[index])
                    for hs, w in dwave.items()}
        return {hs: trapz_rebin((1. + z) * self.wave, self.flux[index], w)
                for hs, w in dwave.items()}

    def rebin_template_batch(self, z, dwave, trapz=True, dedges=None, indx=None, use_gpu=False):
        """All archetypes (or rows ``indx``) at redshift z:
        dict[wavehash] -> (nbin, narch), a CUDA tensor when use_gpu
        (archetypes.py:129-183).  The observed-frame grid (1+z) * wave is
        formed on the host, as redrock does, so the bin integrals are the
        same floating-point operations."""
        if not trapz:
            sel = self.flux if indx is None else self.flux[indx]
            out = {hs: np.stack([_interp(w / (1. + z), self.wave, f) for f in sel], axis=1)
                   for hs, w in dwave.items()}
            return {hs: to_device(a) for hs, a in out.items()} if use_gpu else out
        flux = self.dflux
        if indx is not None:
            flux = flux[torch.as_tensor(np.asarray(indx), device=flux.device)]
        x = (1. + z) * self.wave
        return {hs: trapz_rebin(x, flux, w, use_gpu=use_gpu) for hs, w in dwave.items()}

    def eval(self, subtype, coeff, wave, z, R=None, legcoeff=None):
        """Model flux of the given archetype(s) and Legendre terms
        (archetypes.py:185-226)."""
        import scipy.special
        from .targets import reduced_wavelength
        model = np.zeros(len(wave))
        for this_subtype, c in zip(subtype.split(';'), coeff):
            index = np.where(self._subtype == this_subtype)[0][0]
            binned = trapz_rebin((1 + z) * self.wave, self.flux[index], wave)
            binned *= transmission_Lyman(z, wave, model=self.igm_model)
            model += c * binned
        if legcoeff is not None:
            deg = len(legcoeff) if legcoeff.ndim == 1 else legcoeff.shape[1]
            leg = np.array([scipy.special.legendre(i)(reduced_wavelength(wave))
                            for i in range(deg)])
            model += leg.T.dot(legcoeff).T
        if R is not None:
            model = R.dot(model)
        return model

    def nearest_neighbour_model(self, target, weights, flux, wflux, dwave, z, n_nearest,
                                zzchi2, trans, per_camera, dedges=None, binned=None,
                                use_gpu=False, prior=None, ncam=None):
        """Fit the n_nearest archetypes of lowest chi2 together
        (archetypes.py:228-294); returns (chi2, coefficients, fulltype with
        the ';'-joined subtypes)."""
        nleg = target.nleg
        legendre = target.legendre(nleg=nleg, use_gpu=True)
        iBest = np.argsort(zzchi2)[0:n_nearest]
        sel = torch.as_tensor(iBest, device=self.dflux.device)
        if binned is not None:
            binned = {hs: to_device(b)[:, sel] for hs, b in binned.items()}
        else:
            binned = self.rebin_template_batch(z, dwave, trapz=True, indx=iBest, use_gpu=True)
            for hs in dwave:
                if trans[hs] is not None:
                    binned[hs] = binned[hs] * to_device(np.asarray(trans[hs]))[:, None]
        tdata = {}
        for hs in dwave:
            a = binned[hs][None]
            if nleg > 0:
                a = torch.cat([a, to_device(legendre[hs]).transpose(0, 1)[None]], dim=2)
            tdata[hs] = a.contiguous()
        nbasis = next(iter(tdata.values())).shape[2]
        if per_camera:
            zzchi2, zzcoeff = per_camera_coeff_with_least_square_batch(
                target, tdata, weights, flux, wflux, nleg, 1, method='bvls', n_nbh=n_nearest,
                prior=prior, bands=target.bands)
        else:
            zzchi2, zzcoeff = calc_zchi2_batch(target.spectra, tdata, weights, flux, wflux, 1,
                                               nbasis)
        fsstype = ';'.join('%s' % self._subtype[k] for k in iBest)
        return zzchi2[0], zzcoeff[0], make_fulltype(self._rrtype, fsstype)

    def get_best_archetype(self, target, weights, flux, wflux, dwave, z, per_camera, n_nearest,
                           trans=None, solve_method='bvls', prior=None, use_gpu=False):
        """Best archetype (or nearest-archetype combination) at redshift z
        (archetypes.py:295-400): every archetype is fitted with the target's
        Legendre terms in one batched bounded solve.  ``trans`` (the IGM
        transmission per grid at z, as (1, npix) arrays or None) is reduced
        to 1-D in place, as redrock does.  Returns (chi2, coefficients,
        fulltype)."""
        nleg = target.nleg
        legendre = target.legendre(nleg=nleg, use_gpu=True)
        if trans is None:
            trans = {hs: transmission_Lyman(z, w, use_gpu=False, model=self.igm_model)
                     for hs, w in dwave.items()}
        else:
            for hs in trans:
                if trans[hs] is not None:
                    trans[hs] = trans[hs][0, :]
        binned = self.rebin_template_batch(z, dwave, trapz=True, use_gpu=True)
        nnearest_prior = None
        if n_nearest is not None:
            nnearest_prior = prior.copy()
            prior = prior[n_nearest - 1:, ][:, n_nearest - 1:]
        tdata = {}
        for hs in dwave:
            if trans[hs] is not None:
                binned[hs] = binned[hs] * to_device(np.asarray(trans[hs]))[:, None]
            a = binned[hs].transpose(0, 1)[:, :, None]
            if nleg > 0:
                leg = to_device(legendre[hs]).transpose(0, 1)[None].expand(self._narch, -1, -1)
                a = torch.cat([a, leg], dim=2)
            tdata[hs] = a.contiguous()
        nbasis = next(iter(tdata.values())).shape[2]
        if per_camera:
            zzchi2, zzcoeff = per_camera_coeff_with_least_square_batch(
                target, tdata, weights, flux, wflux, nleg, self._narch, method=solve_method,
                n_nbh=1, prior=prior, bands=target.bands)
        else:
            bounds = np.zeros((2, nbasis))
            bounds[0][1:] = -np.inf
            bounds[1] = np.inf
            zzchi2, zzcoeff = calc_zchi2_batch(target.spectra, tdata, weights, flux, wflux,
                                               self._narch, nbasis,
                                               solve_matrices_algorithm=solve_method.upper(),
                                               solver_args={'bounds': bounds})
            zzcoeff = to_numpy(zzcoeff)
        if n_nearest is not None:
            ncam = len(dwave) if per_camera else 1
            return self.nearest_neighbour_model(target, weights, flux, wflux, dwave, z,
                                                n_nearest, zzchi2, trans, per_camera,
                                                binned=binned, prior=nnearest_prior, ncam=ncam)
        iBest = np.argmin(zzchi2)
        return zzchi2[iBest], zzcoeff[iBest], self._full_type[iBest]


class All_archetypes:
    """Archetype sets keyed by spectral class (archetypes.py:403-426)."""

    def __init__(self, lstfilename=None, archetypes_dir=None, verbose=False, archetypes=None):
        self.archetypes = {}
        if archetypes is not None:
            for a in archetypes:
                self.archetypes[a._rrtype] = a
            return
        if lstfilename is None:
            import glob
            if archetypes_dir is None:
                archetypes_dir = os.environ.get('RR_ARCHETYPE_DIR')
            if archetypes_dir is None:
                raise IOError("ERROR: can't find archetypes_dir or $RR_ARCHETYPE_DIR")
            lstfilename = sorted(glob.glob(os.path.join(archetypes_dir, 'rrarchetype-*.fits')))
        for f in lstfilename:
            a = Archetype(f)
            if verbose:
                print('DEBUG: Found {} archetypes for SPECTYPE {} in file {}'.format(
                    a._narch, a._rrtype, f))
            self.archetypes[a._rrtype] = a
