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
``Archetype.from_synth``) or from a redrock-format archetype file (read
with astropy when it is installed, else with ``redrock_b200.fits``).  redrock's own ``Archetype`` also runs on the
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


def per_camera_order(c, n_nbh, nleg, bands):
    """Coefficients of one per-camera fit in redrock's order
    (zscan.py:322-347): the n_nbh archetype terms, then for each band in
    order of first appearance in ``bands`` the Legendre block of its last
    occurrence."""
    c = np.asarray(c)
    out = [c[:n_nbh]]
    if nleg >= 1:
        blocks = np.split(c[n_nbh:], len(bands))
        by_band = {b: blocks[i] for i, b in enumerate(bands)}
        out += [by_band[b] for b in dict.fromkeys(bands)]
    return np.concatenate(out)


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
    """(wave, flux, rrtype, subtypes, version) of a redrock archetype file
    (archetypes.py:35-58): astropy when installed, else the FITS table
    reader of redrock_b200.fits."""
    filename = os.path.expandvars(filename)
    try:
        from astropy.io import fits
        with fits.open(filename, memmap=False) as h:
            hdr = h['ARCHETYPES'].header
            flux = np.asarray(h['ARCHETYPES'].data['ARCHETYPE']).astype('float64')
            sub = np.asarray(h['ARCHETYPES'].data['SUBTYPE'])
    except ImportError:
        from .fits import read_table
        hdr, rows = read_table(filename, 'ARCHETYPES')
        flux = np.asarray(rows['ARCHETYPE']).astype('float64')
        sub = rows['SUBTYPE']
    sub = [str(s).strip() for s in np.char.strip(np.asarray(sub).astype(str))]
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

    def best_archetypes(self, items, per_camera, n_nearest, solve_method='bvls', prior=None,
                        max_bytes=1 << 31):
        """get_best_archetype for many (target, z, trans) items at once:
        the rebin of every archetype at every item's redshift (one launch
        per grid), the basis assembly and the fits of all archetypes of
        all items in one ``rr_archetype_fit`` launch, and with n_nearest a
        second launch for the nearest-archetype combinations.  ``trans`` is
        a dict of 1-D transmissions (or None) per grid, or None to compute
        it.  ``prior`` is the prior of the n_nearest combination when
        n_nearest is given (redrock's argument), else of the single fit.
        Returns [(chi2, coefficients, fulltype)] in item order."""
        out = [None] * len(items)
        # items are processed in groups whose archetype columns fit max_bytes
        from .engine import GridLayout
        dwave_all = {}
        for t, _, _ in items:
            for s in t.spectra:
                dwave_all.setdefault(s.wavehash, s.wave)
        layout = GridLayout.from_dwave(dwave_all)
        per_item = self._narch * layout.pix_stride * 8
        step = max(1, int(max_bytes // max(per_item, 1)))
        for i0 in range(0, len(items), step):
            sub = items[i0:i0 + step]
            res = self._fit_group(sub, layout, per_camera, n_nearest, solve_method, prior)
            out[i0:i0 + len(sub)] = res
        return out

    def _fit_group(self, items, layout, per_camera, n_nearest, solve_method, prior):
        from . import _lib
        from .device import device, ptr, stream_handle, struct_bytes
        from .engine import PlainTarget
        from .templates import solve_code_of
        from .zscan import HUGE_CHI2
        dev = device()
        L = _lib.lib()
        npair = len(items)
        # targets: band rows, weights and flux, concatenated
        tix, tlist = {}, []
        for t, _, _ in items:
            if id(t) not in tix:
                tix[id(t)] = len(tlist)
                tlist.append(t)
        # band rows of every target's spectra in one pack (rows are per pixel)
        allspec = [sp for t in tlist for sp in t.spectra]
        pt_all = PlainTarget(allspec, layout)
        pt_all._status.check("rr_pack_band_rows")
        npix_t = [sum(len(sp.wave) for sp in t.spectra) for t in tlist]
        offs = np.cumsum([0] + npix_t)
        band, pixb, w, fl, wf = (pt_all.band, pt_all.pix_basis, pt_all.w, pt_all.flux,
                                 pt_all.wflux)
        wsum = [float(np.sum(np.concatenate([s.ivar for s in t.spectra]))) for t in tlist]
        # archetype columns (npair, narch, pix_stride): rebin x IGM
        zs = np.array([float(z) for _, z, _ in items])
        arch = torch.zeros((npair, self._narch, layout.pix_stride), dtype=torch.float64,
                           device=dev)
        for g, hs in enumerate(layout.keys):
            wv = next(s.wave for t, _, _ in items for s in t.spectra if s.wavehash == hs)
            n = layout.npix[g]
            b = trapz_rebin(self.wave, self.dflux, wv, myz=zs, use_gpu=True)  # (npair, n, narch)
            # IGM: given per item, or redrock's transmission_Lyman(z, wave) for
            # the items without one, all their redshifts in one call
            tr = np.ones((npair, n))
            need = [i for i, (_, _, trans) in enumerate(items) if trans is None]
            if need:
                tr[need] = np.asarray(transmission_Lyman(zs[need], wv, use_gpu=False,
                                                         model=self.igm_model)).reshape(len(need), n)
            for i, (_, _, trans) in enumerate(items):
                if trans is not None and trans.get(hs) is not None:
                    T = np.asarray(trans[hs])
                    tr[i] = T[0] if T.ndim == 2 else T
            b = b * to_device(tr)[:, :, None]
            off = layout.pix_offset[g]
            arch[:, :, off:off + n] = b.permute(0, 2, 1)
        # Legendre columns, one set per distinct grid order of the targets
        nleg = tlist[0].nleg
        if any(t.nleg != nleg for t in tlist):
            raise ValueError("targets with different numbers of Legendre terms in one "
                             "archetype batch")
        sets, set_of = {}, []
        for t, _, _ in items:
            hs_order = tuple(dict.fromkeys(s.wavehash for s in t.spectra))
            key = (hs_order, tuple(t.bands) if per_camera else None)
            if key not in sets:
                leg = t.legendre(nleg)
                ncam = len(t.bands) if per_camera else 1
                nl = nleg * ncam
                a = np.zeros((max(nl, 1), layout.pix_stride))
                for i, hs in enumerate(hs_order):
                    g = layout.index[hs]
                    off, n = layout.pix_offset[g], layout.npix[g]
                    for k in range(nleg):
                        col = (i * nleg + k) if per_camera else k
                        if col < nl:
                            a[col, off:off + n] = leg[hs][k]
                sets[key] = (len(sets), a, nl)
            set_of.append(sets[key][0])
        nls = {v[2] for v in sets.values()}
        if len(nls) != 1:
            raise ValueError("targets with different numbers of cameras in one archetype batch")
        nl = nls.pop()
        legs = [None] * len(sets)
        for _, (k, a, _) in sets.items():
            legs[k] = a
        dleg = to_device(np.concatenate([a.ravel() for a in legs]))
        leg_stride = max(nl, 1) * layout.pix_stride

        def launch(m, jobs, njob, method, bounds, pri):
            nb = m + nl
            pairs = [_lib.ArchPair(int(offs[tix[id(t)]]), int(npix_t[tix[id(t)]]),
                                   i * self._narch * layout.pix_stride, set_of[i] * leg_stride)
                     for i, (t, _, _) in enumerate(items)]
            dpairs = to_device(struct_bytes(pairs), torch.uint8)
            djobs = to_device(np.ascontiguousarray(jobs, dtype=np.int32), torch.int32)
            chi2 = torch.empty(npair * njob, dtype=torch.float64, device=dev)
            co = torch.empty((npair * njob, nb), dtype=torch.float64, device=dev)
            if pri is not None and np.shape(pri) != (nb, nb):
                raise ValueError(f"prior of shape {np.shape(pri)} for {nb} coefficients")
            dpri = None if pri is None else to_device(np.ascontiguousarray(pri, np.float64))
            hb = None if bounds is None else np.ascontiguousarray(bounds, dtype=np.float64)
            max_npix = max(npix_t)
            nwork = int(L.rr_archetype_fit_work_bytes(npair, njob, m, nl, max_npix))
            work = torch.empty(max(nwork, 8), dtype=torch.uint8, device=dev)
            rc = L.rr_archetype_fit(ptr(dpairs), npair, ptr(band), ptr(pixb), ptr(w), ptr(wf),
                                    ptr(fl), max_npix, ptr(arch), self._narch, ptr(dleg),
                                    layout.pix_stride,
                                    ptr(djobs), njob, m, nl, ptr(dpri), method,
                                    None if hb is None else hb.ctypes.data, ptr(chi2), ptr(co),
                                    ptr(work), work.numel(), stream_handle())
            _lib.check(rc, "rr_archetype_fit")
            return (chi2.cpu().numpy().reshape(npair, njob),
                    co.cpu().numpy().reshape(npair, njob, nb))

        # every archetype with the Legendre terms (archetypes.py:369-393)
        nb1 = 1 + nl
        p1 = prior
        if n_nearest is not None and prior is not None:
            p1 = prior[n_nearest - 1:, ][:, n_nearest - 1:]
        b1 = np.zeros((2, nb1))
        b1[0][1:] = -np.inf
        b1[1] = np.inf
        code = solve_code_of(solve_method)
        jobs = np.tile(np.arange(self._narch, dtype=np.int32), npair)
        c2, co = launch(1, jobs, self._narch, code, b1 if code == _lib.RR_SOLVE_BVLS else None,
                        p1 if per_camera else None)
        for i, (t, _, _) in enumerate(items):
            if wsum[tix[id(t)]] == 0:
                c2[i] = HUGE_CHI2
                co[i] = 0.0
        if n_nearest is None:
            res = []
            for i, (t, _, _) in enumerate(items):
                k = int(np.argmin(c2[i]))
                c = per_camera_order(co[i, k], 1, nleg, t.bands) if per_camera else co[i, k]
                res.append((c2[i, k], c, self._full_type[k]))
            return res
        # the n_nearest archetypes of lowest chi2 together (archetypes.py:228-294)
        best = np.stack([np.argsort(c2[i])[0:n_nearest] for i in range(npair)])
        nb2 = n_nearest + nl
        if per_camera:
            b2 = np.zeros((2, nb2))
            b2[0][n_nearest:] = -np.inf
            b2[1] = np.inf
            c2n, con = launch(n_nearest, best.ravel(), 1, _lib.RR_SOLVE_BVLS, b2, prior)
        else:
            c2n, con = launch(n_nearest, best.ravel(), 1, _lib.RR_SOLVE_PCA, None, None)
        res = []
        for i, (t, _, _) in enumerate(items):
            c = con[i, 0]
            if wsum[tix[id(t)]] == 0:
                c2n[i, 0] = HUGE_CHI2
                c = np.zeros_like(c)
            if per_camera:
                c = per_camera_order(c, n_nearest, nleg, t.bands)
            ft = make_fulltype(self._rrtype, ';'.join('%s' % self._subtype[k] for k in best[i]))
            res.append((c2n[i, 0], c, ft))
        return res

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
        Legendre terms in one batched launch (``best_archetypes``).  The
        fit uses the target's own spectra (weights, flux and wflux are
        redrock's concatenation of them).  ``trans`` (the IGM transmission
        per grid at z, as (1, npix) arrays or None) is reduced to 1-D in
        place, as redrock does.  Returns (chi2, coefficients, fulltype)."""
        if trans is not None:
            for hs in trans:
                if trans[hs] is not None:
                    trans[hs] = trans[hs][0, :]
        return self.best_archetypes([(target, z, trans)], per_camera, n_nearest,
                                    solve_method=solve_method, prior=prior)[0]


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
