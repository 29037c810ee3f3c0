"""Coadd of each target's exposures on the GPU (redrock 0.22
targets.py:267-373, ``Target.compute_coadd``).

``coadd_targets(targets)`` coadds every target of a list in one launch of
``rr_coadd``: per target, the exposures of each wavelength grid (redrock's
"wavehash", in order of first appearance) become one spectrum with
  ivar = sum ivar,  flux = sum ivar flux / sum ivar (the plain mean where
  sum ivar == 0),  R = sum R ivar / sum ivar (columns of the DIA data),
bit-identical to redrock's numpy.  The coadded spectra are built with the
class of the input spectra (redrock's own ``Spectrum`` or the mirror), which
applies redrock's 0.99 resolution-integral ivar mask.  ``compute_coadd`` is
the per-target method form (installed on redrock's ``Target`` by
``redrock_b200.install``).

With ``cosmics_nsig > 0`` (off by default in redrock's DESI driver) the
exposures' outlier pixels are first masked by ``rr_coadd_cosmics`` --
gradient chi2 across the exposures of a grid against nsig^2, the worst
exposure of each flagged pixel gets ivar 0 (targets.py:310-354) -- and the
coadd then weights flux by the masked ivar and the resolution data by the
exposures' own ivar, as redrock does.  Both steps are bit-identical to
redrock's numpy.
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse
import torch

from . import _lib
from .device import StatusWord, device, ptr, stream_handle, struct_bytes, to_device


def _groups(target):
    keys = []
    for s in target.spectra:
        if s.wavehash not in keys:
            keys.append(s.wavehash)
    return [(k, [s for s in target.spectra if s.wavehash == k]) for k in keys]


def coadd_targets(targets, cache_Rcsr=False, cosmics_nsig=0.):
    """Replace each target's spectra by its per-grid coadds (in place)."""
    plan = []
    descs, rdata, ivar, flux, exp_data, exp_pix, gwave = [], [], [], [], [], [], []
    d_off = p_off = out_pix = out_data = 0
    for t in targets:
        for key, specs in _groups(t):
            s0 = specs[0]
            npix = len(s0.wave)
            data0 = np.asarray(s0.R.data)
            ndiag = data0.shape[0]
            first = len(exp_data)
            for s in specs:
                d = np.asarray(s.R.data, dtype=np.float64)
                if len(s.wave) != npix or d.shape != data0.shape:
                    raise ValueError("exposures on one wavelength grid must have the same "
                                     "length and resolution shape")
                rdata.append(d.ravel())
                ivar.append(np.asarray(s.ivar, dtype=np.float64))
                flux.append(np.asarray(s.flux, dtype=np.float64))
                exp_data.append(d_off)
                exp_pix.append(p_off)
                d_off += d.size
                p_off += npix
            descs.append(_lib.CoaddGroup(npix, ndiag, len(specs), first, out_pix, out_data))
            gwave.append(np.asarray(s0.wave, dtype=np.float64))
            plan.append((t, specs, npix, ndiag, out_pix, out_data))
            out_pix += npix
            out_data += ndiag * npix
    if not plan:
        return targets
    L = _lib.lib()
    dev = device()
    dg = to_device(struct_bytes(descs), torch.uint8)
    ded = to_device(np.asarray(exp_data, dtype=np.int64), torch.int64)
    dep = to_device(np.asarray(exp_pix, dtype=np.int64), torch.int64)
    drd = to_device(np.concatenate(rdata))
    div = to_device(np.concatenate(ivar))
    dfl = to_device(np.concatenate(flux))
    ord_ = torch.empty(max(out_data, 1), dtype=torch.float64, device=dev)
    oiv = torch.empty(max(out_pix, 1), dtype=torch.float64, device=dev)
    ofl = torch.empty(max(out_pix, 1), dtype=torch.float64, device=dev)
    max_npix = max(p[2] for p in plan)
    div_w = div
    if cosmics_nsig > 0:
        # the cosmic-ray mask first; redrock's threshold is cosmics_nsig**2
        div_w = torch.empty_like(div)
        work = torch.empty(2 * div.numel(), dtype=torch.float64, device=dev)
        dwv = to_device(np.concatenate(gwave))
        st = StatusWord()
        rc = L.rr_coadd_cosmics(ptr(dg), len(descs), ptr(dep), ptr(dwv), ptr(div), ptr(dfl),
                                float(cosmics_nsig ** 2), ptr(div_w), ptr(work), div.numel(),
                                st.ptr, stream_handle())
        _lib.check(rc, "rr_coadd_cosmics")
        if int(st.t.item()):
            raise ValueError("cosmic-ray rejection: an exposure has no pixel with ivar > 0 "
                             "(numpy.interp: array of sample points is empty)")
    for g0 in range(0, len(descs), 65535):
        # groups in slices of the grid's y limit; offsets stay global
        n = min(65535, len(descs) - g0)
        gsize = ctypes.sizeof(_lib.CoaddGroup)
        rc = L.rr_coadd_ex(dg.data_ptr() + g0 * gsize, n, max_npix, ptr(ded), ptr(dep), ptr(drd),
                           ptr(div), ptr(div_w), ptr(dfl), ptr(ord_), ptr(oiv), ptr(ofl),
                           stream_handle())
        _lib.check(rc, "rr_coadd_ex")
    hrd, hiv, hfl = ord_.cpu().numpy(), oiv.cpu().numpy(), ofl.cpu().numpy()
    new = {}
    for t, specs, npix, ndiag, op, od in plan:
        s_last = specs[-1]
        rdiags = hrd[od:od + ndiag * npix].reshape(ndiag, npix).copy()
        R = scipy.sparse.dia_matrix((rdiags, specs[0].R.offsets), shape=(npix, npix))
        Rcsr = R.tocsr() if cache_Rcsr else None
        cls = type(specs[0])
        sp = cls(specs[0].wave, hfl[op:op + npix].copy(), hiv[op:op + npix].copy(), R, Rcsr,
                 band=s_last.band)
        new.setdefault(id(t), (t, []))[1].append(sp)
    for t, sp in new.values():
        t.spectra = sp
    return targets


def compute_coadd(self, cache_Rcsr=False, cosmics_nsig=0.):
    """Target.compute_coadd (targets.py:267): replaces the target's spectra
    with their per-grid coadds."""
    coadd_targets([self], cache_Rcsr=cache_Rcsr, cosmics_nsig=cosmics_nsig)
