"""Oracle: CPU restatement of redrock's redshift-scan hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker for the CUDA path:
only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import it, and never as the thing measured or shipped.  The product package
(redrock_b200/) does not import it.

Restates, in numpy/scipy (and a small C file for the rebin), redrock 0.22:
  centers2edges         py/redrock/rebin.py:100-118
  trapz_rebin           py/redrock/rebin.py:126-209, 212-378 (C restatement in
                        trapz_oracle.c, bit-for-bit the same operation order)
  rebin_template        py/redrock/rebin.py:453-517
  transmission_Lyman    py/redrock/igm.py:369-439 (Inoue14 igm.py:105-318,
                        Calura12/Kamble20 igm.py:321-364)
  DistTemplate basis    py/redrock/templates.py:584-597
  spectral_data         py/redrock/zscan.py:192-209
  Target.compute_coadd  py/redrock/targets.py:267-373 (with the cosmic-ray
                        rejection of :310-354)
  calc_zchi2_batch      py/redrock/zscan.py:626-781 (CPU branch :747-780)
  solve_matrices        py/redrock/zscan.py:1107-1201 (PCA, NMF/NNLS, BVLS)
  calc_negOII_penalty   py/redrock/zscan.py:783-800
  calc_zchi2            py/redrock/zscan.py:807-889
  calc_zchi2_one        py/redrock/zscan.py:169-190, 213-243
  per_camera_coeff      py/redrock/zscan.py:245-348 (CPU branch)
  get_best_archetype,   py/redrock/archetypes.py:228-400 (trapz rebin, CPU)
  nearest_neighbour_model
  prior_on_coeffs       py/redrock/fitz.py:113-130
  legendre_dict         py/redrock/targets.py:237-254, utils.py:260-271

Pinned against fixtures generated by running redrock itself
(tests/golden/make_*golden.py, tests/test_oracle.py).
"""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import scipy.sparse

HERE = os.path.dirname(os.path.abspath(__file__))
HUGE_CHI2 = 9999999.0
LYA = 1215.67
MIN_RESOLUTION_INTEGRAL = 0.99

# ---------------------------------------------------------------------------
# rebin
# ---------------------------------------------------------------------------
_lib = None


def _trapz_lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "libtrapz_oracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _lib = ctypes.CDLL(path)
        _lib.oracle_trapz_rebin.restype = None
        _lib.oracle_trapz_rebin.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p]
    return _lib


def centers2edges(centers):
    centers = np.asarray(centers)
    edges = np.zeros(len(centers) + 1)
    edges[1:-1] = (centers[0:-1] + centers[1:]) / 2.0
    edges[0] = centers[0] - (centers[1] - edges[1])
    edges[-1] = centers[-1] + (centers[-1] - edges[-2])
    return edges


def trapz_rebin(x, y, xnew=None, edges=None, myz=None):
    """Same contract and output shapes as redrock's CPU trapz_rebin."""
    if edges is None:
        edges = centers2edges(xnew)
    edges = np.ascontiguousarray(edges, dtype=np.float64)
    nbins = len(edges) - 1
    scalar_z = myz is None or np.isscalar(myz)
    myz = np.atleast_1d(np.asarray(0.0 if myz is None else myz, dtype=np.float64))
    nz = len(myz)
    if nz == 0:
        return np.zeros((0, nbins, 1))
    x = np.ascontiguousarray(x, dtype=np.float64)
    if edges[0] < x[0] * (1 + myz.max()) or edges[-1] > x[-1] * (1 + myz.min()):
        raise ValueError('edges must be within input x range')
    y = np.asarray(y, dtype=np.float64)
    scalar_basis = y.ndim == 1
    y2 = np.ascontiguousarray(y[None, :] if scalar_basis else y)
    nb = y2.shape[0]
    out = np.zeros((nz, nbins, nb))
    xs = np.zeros(len(x))
    myz = np.ascontiguousarray(myz)
    _trapz_lib().oracle_trapz_rebin(x.ctypes.data, len(x), y2.ctypes.data, nb, edges.ctypes.data,
                                    nbins, myz.ctypes.data, nz, out.ctypes.data, xs.ctypes.data)
    shape = (nbins,) + (() if scalar_basis else (nb,))
    if not scalar_z:
        shape = (nz,) + shape
    return out.reshape(shape)


def rebin_template(wave, flux, myz, dwave):
    return {hs: trapz_rebin(wave, flux, xnew=w, myz=myz) for hs, w in dwave.items()}


# ---------------------------------------------------------------------------
# IGM
# ---------------------------------------------------------------------------
_INOUE = None


def _inoue_table():
    """39-line Inoue et al. (2014) table, read from the kernel's own header."""
    global _INOUE
    if _INOUE is None:
        hdr = open(os.path.join(HERE, "..", "redrock_b200", "csrc", "rr_igm_table.h")).read()

        def block(name):
            body = hdr[hdr.index(name):]
            body = body[body.index("{") + 1:body.index("};")]
            vals = re.findall(r"-?0x[0-9a-fA-F.]+p[-+]?\d+", body)
            return np.array([float.fromhex(v) for v in vals])

        lam = block("rr_inoue14_lam_h")
        laf = block("rr_inoue14_laf_h").reshape(-1, 3)
        dla = block("rr_inoue14_dla_h").reshape(-1, 2)
        _INOUE = (lam, laf, dla)
    return _INOUE


def _inoue14(zS, lobs):
    """full_IGM for z (nz,) and a (nz, nw) observed grid (igm.py:105-267)."""
    lam, laf, dla = _inoue_table()
    l2 = lam[:, None, None]
    lrest_lt = (lobs / (1 + zS)[:, None])[None] < l2
    # Lyman series, LAF
    z1LAF, z2LAF = 1.2, 4.7
    x1 = lrest_lt & (lobs < l2 * (1 + z1LAF))
    x2 = lrest_lt & ((lobs >= l2 * (1 + z1LAF)) & (lobs < l2 * (1 + z2LAF)))
    x3 = lrest_lt & (lobs >= l2 * (1 + z2LAF))
    v = np.zeros(lrest_lt.shape)
    v[x1] += (laf[:, 0][:, None, None] * lobs ** 1.2)[x1]
    v[x2] += (laf[:, 1][:, None, None] * lobs ** 3.7)[x2]
    v[x3] += (laf[:, 2][:, None, None] * lobs ** 5.5)[x3]
    t_lslaf = v.sum(axis=0)
    # Lyman series, DLA
    z1DLA = 2.0
    x0 = lrest_lt & (lobs < l2 * (1. + z1DLA))
    x1 = lrest_lt & ~(lobs < l2 * (1. + z1DLA))
    v = np.zeros(lrest_lt.shape)
    v[x0] += (dla[:, 0][:, None, None] * lobs ** 2)[x0]
    v[x1] += (dla[:, 1][:, None, None] * lobs ** 3)[x1]
    t_lsdla = v.sum(axis=0)
    # Lyman continuum, DLA
    lamL = 911.8
    zc = zS[:, None] * np.ones_like(lobs)
    opz = 1.0 + zc
    r = lobs / lamL
    t_lcdla = np.zeros_like(lobs)
    x0 = lobs < lamL * (1. + zS)[:, None]
    y0 = x0 & (zc < z1DLA)
    t_lcdla[y0] = (0.2113 * np.power(opz[y0], 2) - 0.07661 * np.power(opz[y0], 2.3)
                   * np.power(r[y0], -3e-1) - 0.1347 * np.power(r[y0], 2))
    y0 = x0 & (zc >= z1DLA)
    xx = lobs >= lamL * (1. + z1DLA)
    m = y0 & xx
    t_lcdla[m] = (0.04696 * np.power(opz[m], 3) - 0.01779 * np.power(opz[m], 3.3)
                  * np.power(r[m], -3e-1) - 0.02916 * np.power(r[m], 3))
    m = y0 & ~xx
    t_lcdla[m] = (0.6340 + 0.04696 * np.power(opz[m], 3) - 0.01779 * np.power(opz[m], 3.3)
                  * np.power(r[m], -3e-1) - 0.1347 * np.power(r[m], 2)
                  - 0.2905 * np.power(r[m], -3e-1))
    # Lyman continuum, LAF.  redrock's z < 1.2 assignment is overwritten by
    # the z < 4.7 one for every element it touches, so it is not restated.
    t_lclaf = np.zeros_like(lobs)
    y0 = x0 & (zc < z2LAF)
    xx = lobs >= lamL * (1 + z1LAF)
    m = y0 & xx
    t_lclaf[m] = 2.545e-2 * (np.power(opz[m], 1.6) * np.power(r[m], 2.1) - np.power(r[m], 3.7))
    m = y0 & ~xx
    t_lclaf[m] = (2.545e-2 * np.power(opz[m], 1.6) * np.power(r[m], 2.1)
                  + 0.3248 * np.power(r[m], 1.2) - 0.2496 * np.power(r[m], 2.1))
    y0 = x0 & (zc >= z2LAF)
    xa = lobs > lamL * (1. + z2LAF)
    xb = (lobs >= lamL * (1. + z1LAF)) & (lobs < lamL * (1. + z2LAF))
    xc = lobs < lamL * (1. + z1LAF)
    m = y0 & xa
    t_lclaf[m] = 5.221e-4 * (np.power(opz[m], 3.4) * np.power(r[m], 2.1) - np.power(r[m], 5.5))
    m = y0 & xb
    t_lclaf[m] = (5.221e-4 * np.power(opz[m], 3.4) * np.power(r[m], 2.1)
                  + 0.2182 * np.power(r[m], 2.1) - 2.545e-2 * np.power(r[m], 3.7))
    m = y0 & xc
    t_lclaf[m] = (5.221e-4 * np.power(opz[m], 3.4) * np.power(r[m], 2.1)
                  + 0.3248 * np.power(r[m], 1.2) - 3.140e-2 * np.power(r[m], 2.1))
    tau_ls = t_lslaf + t_lsdla
    tau_lc = t_lclaf + t_lcdla
    return np.exp(-1.0 * (tau_lc + tau_ls + 0.))


_CALURA = [(LYA, 0.0023, 3.64), (1025.72, 0.0023 / 5.2615, 3.64), (972.537, 0.0023 / 14.356, 3.64),
           (949.7431, 0.0023 / 29.85984, 3.64), (937.8035, 0.0023 / 53.36202, 3.64)]
_KAMBLE = [(LYA, 0.00554, 3.182)]
IGM_MODELS = ('Calura12', 'Kamble20', 'Inoue14', 'None', None)


def transmission_Lyman(zObj, lObs, model='Calura12', always_return_array=True):
    """Same contract as redrock's igm.transmission_Lyman (CPU)."""
    if model not in IGM_MODELS:
        raise ValueError(f'Unrecognized model {model}; should be one of {IGM_MODELS}')
    if (model == 'None' or model is None) and not always_return_array:
        return None
    min_wave = np.min(lObs) / (1. + np.max(zObj))
    if min_wave > LYA and not always_return_array:
        return None
    scalar_z = np.isscalar(zObj)
    scalar_l = np.isscalar(lObs)
    z = np.atleast_1d(np.asarray(zObj, dtype=np.float64))
    lo = np.atleast_1d(np.asarray(lObs, dtype=np.float64))
    if always_return_array and (min_wave > LYA or model is None or model == 'None'):
        T = np.ones((len(z), len(lo)))
    elif model in ('Calura12', 'Kamble20'):
        lrest = np.outer(1.0 / (1.0 + z), lo)
        lobs2 = np.tile(lo, (z.size, 1))
        T = np.ones(lrest.shape)
        for line, A, B in (_CALURA if model == 'Calura12' else _KAMBLE):
            if lrest.min() > line:
                continue
            w = lrest < line
            zpix = lobs2[w] / line - 1.
            T[w] *= np.exp(-(A * (1. + zpix) ** B))
    else:
        lobs2 = np.tile(lo, (z.size, 1))
        T = np.ones(lobs2.shape)
        ii = np.nonzero(lobs2.min() / (1. + z) < LYA)[0]
        # a few redshifts at a time: the restatement keeps redrock's
        # (39, nz, nwave) temporaries, which are large for long z grids
        for i0 in range(0, len(ii), 8):
            sel = ii[i0:i0 + 8]
            T[sel, :] = _inoue14(z[sel], lobs2[sel, :])
    if scalar_z and scalar_l:
        return T[0, 0]
    if scalar_z:
        return T[0]
    if scalar_l:
        return T[:, 0]
    return T


def template_basis(wave, flux, redshifts, dwave, igm_model):
    """DistTemplate.local.data for one template (templates.py:584-597)."""
    data = rebin_template(wave, flux, redshifts, dwave)
    for k, w in dwave.items():
        T = transmission_Lyman(redshifts, w, always_return_array=False, model=igm_model)
        if T is None:
            continue
        data[k] *= T[:, :, None]
    return data


# ---------------------------------------------------------------------------
# scan
# ---------------------------------------------------------------------------

def spectrum_rcsr(rdata, roffsets, npix):
    return scipy.sparse.dia_matrix((rdata, roffsets), shape=(npix, npix)).tocsr()


def masked_ivar(ivar, rdata, roffsets):
    """Spectrum.__init__: pixels whose R row integral < 0.99 get ivar 0."""
    npix = len(ivar)
    R = scipy.sparse.dia_matrix((rdata, roffsets), shape=(npix, npix))
    ivar = np.array(ivar, dtype=np.float64)
    ivar[np.asarray(R.sum(axis=1))[:, 0] < MIN_RESOLUTION_INTEGRAL] = 0.
    return ivar


class OSpectrum:
    """Minimal spectrum record: wave, flux, ivar (already masked), Rcsr."""

    def __init__(self, wavehash, wave, flux, ivar, rdata, roffsets):
        self.wavehash = wavehash
        self.wave = wave
        self.flux = np.asarray(flux, dtype=np.float64)
        self.ivar = masked_ivar(ivar, rdata, roffsets)
        self.Rcsr = spectrum_rcsr(rdata, roffsets, len(wave))


def _cosmic_grad(wave, flux, ivar):
    """One exposure's flux gradient and its variance (targets.py:310-332):
    ivar == 0 pixels interpolated from ivar > 0 ones, ivar <= 0 left over
    set to the smallest positive ivar."""
    good = ivar > 0
    bad = ivar == 0
    tflux = flux.copy()
    tivar = ivar.copy()
    tflux[bad] = np.interp(wave[bad], wave[good], flux[good])
    tivar[bad] = np.interp(wave[bad], wave[good], ivar[good])
    bad = tivar <= 0
    tivar[bad] = np.min(tivar[tivar > 0])
    tvar = 1 / tivar
    tflux[1:] = tflux[1:] - tflux[:-1]
    tvar[1:] = tvar[1:] + tvar[:-1]
    tflux[0] = 0
    return tflux, tvar


def cosmic_mask(wave, flux, ivar, nsig):
    """ivar (nspec, npix) with the cosmic-ray outliers set to 0
    (targets.py:337-354): gradient chi2 across exposures against nsig^2;
    the exposure with the largest term of a flagged pixel is masked."""
    ivar = np.array(ivar, dtype=np.float64)
    grads = [_cosmic_grad(wave, f, v) for f, v in zip(flux, ivar)]
    if len(grads) > 1 and nsig > 0:
        grad = np.array([g[0] for g in grads])
        gradivar = 1 / np.array([g[1] for g in grads])
        nspec = grad.shape[0]
        meangrad = np.sum(gradivar * grad, axis=0) / np.sum(gradivar)
        deltagrad = grad - meangrad
        chi2 = np.sum(gradivar * deltagrad ** 2, axis=0) / (nspec - 1)
        for j in np.where(chi2 > nsig ** 2)[0]:
            k = np.argmax(gradivar[:, j] * deltagrad[:, j] ** 2)
            ivar[k][j] = 0.
    return ivar


def compute_coadd(exposures, cosmics_nsig=0.):
    """Target.compute_coadd (targets.py:267-373).

    exposures: list of (band, wave, flux, ivar, rdata, roffsets), ivar already
    masked by its own resolution (Spectrum.__init__).  Returns one
    (band, wave, flux, ivar, rdata, roffsets) per grid in order of first
    appearance; the coadd's ivar is masked by the coadded resolution
    (Spectrum.__init__ of the coadd, targets.py:33-35)."""
    keys = []
    for e in exposures:
        if e[0] not in keys:
            keys.append(e[0])
    out = []
    for key in keys:
        group = [e for e in exposures if e[0] == key]
        rdiags = None
        for e in group:
            if rdiags is None:
                rdiags = np.asarray(e[4]) * e[3]
            else:
                rdiags += np.asarray(e[4]) * e[3]
        flux = np.array([e[2] for e in group])
        ivar = np.array([e[3] for e in group])
        if cosmics_nsig > 0:
            ivar = cosmic_mask(group[0][1], flux, ivar, cosmics_nsig)
        unweighted = np.sum(flux, axis=0)
        weights = np.sum(ivar, axis=0)
        weighted = np.sum(ivar * flux, axis=0)
        isbad = (weights == 0)
        f = weighted / (weights + isbad)
        f[isbad] = unweighted[isbad] / len(group)
        rdiags /= (weights + isbad)
        out.append((group[-1][0], group[0][1], f, masked_ivar(weights, rdiags, group[0][5]),
                    rdiags, group[0][5]))
    return out


def spectral_data(spectra):
    weights = np.concatenate([s.ivar for s in spectra])
    flux = np.concatenate([s.flux for s in spectra])
    return weights, flux, weights * flux


def solve_pca(M, y):
    return np.linalg.solve(M, y.reshape(y.shape + (1,))).reshape(y.shape)


def solve_matrices(M, y, method='PCA', solver_args=None):
    """solve_matrices, CPU branch (zscan.py:1107-1201): PCA linear solve;
    NMF / NNLS: scipy.optimize.nnls(M, y); BVLS: lsq_linear(M, y, bounds,
    method='bvls'); other names: NotImplementedError."""
    from scipy.optimize import lsq_linear, nnls
    m = method.upper()
    if m == 'PCA':
        return solve_pca(M, y)
    if m in ('NMF', 'NNLS'):
        try:
            return nnls(M, y)[0]
        except Exception:
            raise np.linalg.LinAlgError
    if m == 'BVLS':
        if solver_args is not None and 'bounds' in solver_args:
            bounds = solver_args['bounds']
        else:
            bounds = np.zeros((2, y.shape[-1]))
            bounds[0] = -np.inf
            bounds[1] = np.inf
        return lsq_linear(M, y, bounds=bounds, method='bvls').x
    raise NotImplementedError(method)


def calc_zchi2_batch(spectra, tdata, weights, flux, wflux, nz, nbasis, method='PCA', prior=None,
                     solver_args=None):
    zchi2 = np.zeros(nz)
    if weights.sum() == 0:
        zchi2[:] = HUGE_CHI2
        return zchi2, np.zeros((nz, nbasis))
    zcoeff = np.zeros((nz, nbasis))
    for i in range(nz):
        Tb = np.vstack([s.Rcsr.dot(tdata[s.wavehash][i, :, :]) for s in spectra])
        M = Tb.T.dot(np.multiply(weights[:, None], Tb))
        y = Tb.T.dot(wflux)
        if prior is not None:
            M += prior
        try:
            zcoeff[i, :] = solve_matrices(M, y, method, solver_args)
        except (np.linalg.LinAlgError, NotImplementedError):
            zchi2[i] = HUGE_CHI2
            continue
        model = Tb.dot(zcoeff[i, :])
        zchi2[i] = np.dot((flux - model) ** 2, weights)
    return zchi2, zcoeff


def calc_negOII_penalty(OIItemplate, coeff):
    OIIflux = np.sum(coeff @ OIItemplate, axis=1)
    return -OIIflux * (OIIflux < 0)


def calc_zchi2(targets, tdata, nz, nbasis, method='PCA', OIItemplate=None):
    """targets: list of lists of OSpectrum.  Returns (zchi2, zcoeff, penalty)."""
    nt = len(targets)
    zchi2 = np.zeros((nt, nz))
    pen = np.zeros((nt, nz))
    zcoeff = np.zeros((nt, nz, nbasis))
    for j, spectra in enumerate(targets):
        weights, flux, wflux = spectral_data(spectra)
        if np.sum(weights) == 0:
            zchi2[j, :] = HUGE_CHI2
            continue
        zchi2[j], zcoeff[j] = calc_zchi2_batch(spectra, tdata, weights, flux, wflux, nz, nbasis,
                                              method)
        if OIItemplate is not None:
            pen[j] = calc_negOII_penalty(OIItemplate, zcoeff[j])
    return zchi2, zcoeff, pen


def calc_zchi2_one(spectra, weights, flux, wflux, tdata, method='PCA'):
    Tb = np.vstack([s.Rcsr.dot(tdata[s.wavehash]) for s in spectra])
    nbasis = Tb.shape[1]
    zcoeff = np.zeros(nbasis)
    M = Tb.T.dot(np.multiply(weights[:, None], Tb))
    y = Tb.T.dot(wflux)
    if method.upper() != 'PCA':
        return HUGE_CHI2, zcoeff
    try:
        zcoeff[:] = solve_pca(M, y)
    except np.linalg.LinAlgError:
        return HUGE_CHI2, zcoeff
    model = Tb.dot(zcoeff)
    return np.dot((flux - model) ** 2, weights), zcoeff


def oii_template(wave, flux):
    """Template.OIItemplate (templates.py:172-174)."""
    isOII = (3724 <= wave) & (wave <= 3733)
    return flux[:, isOII]


# ---------------------------------------------------------------------------
# reference gradient (checker for the adjoint kernel)
# ---------------------------------------------------------------------------

def basis_and_dz(wave, flux, z, dwave, igm_model, h_igm=1e-7):
    """T(z) per grid (npix, nb) and dT/dz: the trapezoid average of the
    piecewise-linear template over a bin of width w obeys
    dT/dz = (T - (e_hi y(e_hi) - e_lo y(e_lo)) / w) / (1+z) with y the
    redshifted interpolant at the edges; the IGM factor's z derivative is a
    central difference of transmission_Lyman (step h_igm)."""
    T = template_basis(wave, flux, np.array([z]), dwave, igm_model)
    out = {}
    for k, w in dwave.items():
        e = centers2edges(w)
        Tr = trapz_rebin(wave, flux, edges=e, myz=np.array([z]))[0]     # (npix, nb)
        xs = wave * (1 + z)
        ye = np.stack([np.interp(e, xs, fb) for fb in flux], axis=1)   # (npix+1, nb)
        dT = (Tr - (e[1:, None] * ye[1:] - e[:-1, None] * ye[:-1]) / np.diff(e)[:, None]) / (1 + z)
        tr = transmission_Lyman(np.array([z]), w, model=igm_model, always_return_array=True)[0]
        tp = transmission_Lyman(np.array([z + h_igm]), w, model=igm_model,
                                always_return_array=True)[0]
        tm = transmission_Lyman(np.array([z - h_igm]), w, model=igm_model,
                                always_return_array=True)[0]
        dtr = (tp - tm) / (2 * h_igm)
        out[k] = (T[k][0], dT * tr[:, None] + Tr * dtr[:, None])
    return out


def chi2_grad_z(spectra, wave, flux, z, dwave, igm_model):
    """(chi2, dchi2/dz) at z from the normal equations and stationarity."""
    bd = basis_and_dz(wave, flux, z, dwave, igm_model)
    Tb = np.vstack([s.Rcsr.dot(bd[s.wavehash][0]) for s in spectra])
    dTb = np.vstack([s.Rcsr.dot(bd[s.wavehash][1]) for s in spectra])
    w, f, wf = spectral_data(spectra)
    M = Tb.T.dot(w[:, None] * Tb)
    c = solve_pca(M, Tb.T.dot(wf))
    r = f - Tb.dot(c)
    return np.dot(w * r, r), -2.0 * np.dot(w * r, dTb.dot(c))


# ---------------------------------------------------------------------------
# archetypes
# ---------------------------------------------------------------------------

def reduced_wavelength(wave):
    """utils.py:260-271: wavelengths mapped linearly onto [-1, 1]."""
    return 2 * (wave - wave.min()) / (wave.max() - wave.min()) - 1


def legendre_dict(dwave, nleg):
    """Target.legendre (targets.py:237-254): P_0..P_{nleg-1} per grid."""
    import scipy.special
    return {hs: np.array([scipy.special.legendre(i)(reduced_wavelength(w)) for i in range(nleg)])
            .reshape(nleg, len(w)) for hs, w in dwave.items()}


def prior_on_coeffs(n_nbh, deg_legendre, sigma, ncamera):
    """fitz.py:113-130: 1/sigma^2 on the Legendre terms, 0 on archetypes."""
    nbasis = n_nbh + deg_legendre * ncamera
    prior = np.zeros((nbasis, nbasis))
    np.fill_diagonal(prior, 1 / (sigma ** 2))
    for i in range(n_nbh):
        prior[i][i] = 0.
    return prior


def per_camera_coeff(spectra, tdata, weights, flux, wflux, nleg, narch, method, n_nbh, prior,
                     bands):
    """per_camera_coeff_with_least_square_batch, CPU branch (zscan.py:245-348):
    one fit per archetype with each camera's Legendre terms in their own
    columns; coefficients in [archetypes, Legendre per band] order."""
    ncam = len(bands)
    nbasis = n_nbh + nleg * ncam
    method = method.upper()
    solver_args = {}
    if method == 'BVLS':
        bounds = np.zeros((2, nbasis))
        bounds[0][n_nbh:] = -np.inf
        bounds[1] = np.inf
        solver_args['bounds'] = bounds
    zzchi2 = np.zeros(narch)
    zzcoeff = np.zeros((narch, nbasis))
    for j in range(narch):
        t2 = {}
        for i, hs in enumerate(tdata):
            a = np.zeros((tdata[hs].shape[1], nbasis))
            a[:, :n_nbh] = tdata[hs][j, :, :n_nbh]
            a[:, n_nbh + i * nleg:n_nbh + (i + 1) * nleg] = tdata[hs][j, :, n_nbh:]
            t2[hs] = a[None]
        c2, co = calc_zchi2_batch(spectra, t2, weights, flux, wflux, 1, nbasis, method, prior,
                                  solver_args)
        zzchi2[j] = c2[0]
        zzcoeff[j] = co[0]
    if n_nbh > 1:
        alpha = zzcoeff[0:1, :n_nbh]
    else:
        alpha = zzcoeff[:, :1]
    blocks = np.split(zzcoeff[:, n_nbh:], ncam, axis=1) if nleg >= 1 else []
    # one block per distinct band, in order of first appearance in bands
    seen = {}
    for i, b in enumerate(bands):
        seen[b] = blocks[i] if blocks else None
    cols = [alpha] + ([seen[b] for b in seen] if nleg >= 1 else [])
    return zzchi2, np.concatenate(cols, axis=1)


class OArchetype:
    """Archetype set: wave (nwave,), flux (narch, nwave), rrtype, and the
    subtypes with the row number appended (archetypes.py:35-70)."""

    def __init__(self, wave, flux, rrtype, subtype):
        self.wave = np.asarray(wave, dtype=np.float64)
        self.flux = np.asarray(flux, dtype=np.float64)
        self.narch = self.flux.shape[0]
        self.rrtype = rrtype
        self.subtype = np.array([f"{s}_{i}" for i, s in enumerate(subtype)])
        self.full_type = np.array([f"{rrtype}:::{s}" for s in self.subtype])
        self.igm_model = 'Inoue14'

    def rebin(self, z, dwave, indx=None):
        """rebin_template_batch, trapz (archetypes.py:129-183):
        dict -> (nbin, narch)."""
        flux = self.flux if indx is None else self.flux[indx]
        return {hs: trapz_rebin((1. + z) * self.wave, flux, w) for hs, w in dwave.items()}


def nearest_neighbour_model(arch, spectra, bands, legendre, weights, flux, wflux, dwave, z,
                            n_nearest, zzchi2, per_camera, binned, prior):
    """archetypes.py:228-294 with binned (already x IGM) passed in."""
    nleg = legendre[next(iter(legendre))].shape[0]
    iBest = np.argsort(zzchi2)[0:n_nearest]
    tdata = {}
    for hs in dwave:
        a = binned[hs][:, iBest][None]
        if nleg > 0:
            a = np.append(a, legendre[hs].T[None], axis=2)
        tdata[hs] = a
    nbasis = tdata[hs].shape[2]
    if per_camera:
        c2, co = per_camera_coeff(spectra, tdata, weights, flux, wflux, nleg, 1, 'bvls',
                                  n_nearest, prior, bands)
    else:
        c2, co = calc_zchi2_batch(spectra, tdata, weights, flux, wflux, 1, nbasis)
    return c2[0], co[0], arch.rrtype + ':::' + ';'.join(arch.subtype[k] for k in iBest)


def get_best_archetype(arch, spectra, bands, legendre, weights, flux, wflux, dwave, z,
                       per_camera, n_nearest, trans=None, solve_method='bvls', prior=None):
    """Archetype.get_best_archetype, CPU branch (archetypes.py:295-400).
    ``trans``: dict of 1-D transmissions (or None) per grid at z."""
    nleg = legendre[next(iter(legendre))].shape[0]
    if trans is None:
        trans = {hs: transmission_Lyman(z, w, model=arch.igm_model) for hs, w in dwave.items()}
    binned = arch.rebin(z, dwave)
    nn_prior = None
    if n_nearest is not None:
        nn_prior = prior.copy()
        prior = prior[n_nearest - 1:, n_nearest - 1:]
    tdata = {}
    for hs in dwave:
        if trans[hs] is not None:
            binned[hs] = binned[hs] * trans[hs][:, None]
        a = binned[hs].T[:, :, None]
        if nleg > 0:
            a = np.append(a, np.tile(legendre[hs].T[None], (arch.narch, 1, 1)), axis=2)
        tdata[hs] = a
    nbasis = tdata[hs].shape[2]
    if per_camera:
        c2, co = per_camera_coeff(spectra, tdata, weights, flux, wflux, nleg, arch.narch,
                                  solve_method, 1, prior, bands)
    else:
        bounds = np.zeros((2, nbasis))
        bounds[0][1:] = -np.inf
        bounds[1] = np.inf
        c2, co = calc_zchi2_batch(spectra, tdata, weights, flux, wflux, arch.narch, nbasis,
                                  solve_method.upper(), None, {'bounds': bounds})
    if n_nearest is not None:
        return nearest_neighbour_model(arch, spectra, bands, legendre, weights, flux, wflux,
                                       dwave, z, n_nearest, c2, per_camera, binned, nn_prior)
    i = np.argmin(c2)
    return c2[i], co[i], arch.full_type[i]
