"""Seeded synthetic DESI-like workloads for the redshift scan.

Everything here is plain numpy and deterministic for a given seed, so the
same arrays can be regenerated on any machine.  Nothing in this module runs
the scan; it only produces the raw inputs (camera grids, banded resolution
matrices in DIA form, flux/ivar, template bases and redshift grids).

Workload shapes:

* cameras b/r/z: ``np.arange(lo, hi + 0.01, 0.8)`` for (3600, 5800),
  (5760, 7620), (7520, 9824) -> 2751 / 2326 / 2881 pixels (P = 7958).
* resolution: 11 diagonals (offsets -5..5), Gaussian kernel with sigma drawn
  per (target, camera) from U(0.8, 1.2) pixels; every row of the truncated
  band matrix is normalised to sum 1, so no row falls under redrock's 0.99
  row-integral cut (``targets.py:33-35`` of the reference).
* ivar = 1/sigma^2 with sigma ~ U(0.5, 2); a random fraction of pixels is
  masked (ivar = 0).
* GALAXY template: rest 1200-10000 A at 0.2 A (44 001 samples), 10 bases:
  power law, Legendre P1-P4, and five sigma = 2 A Gaussian line modes
  ([OII], Hb, [OIII], Ha+[NII], [SII]).  Each line mode also carries a weak
  sinusoidal continuum ripple (periods 350-950 A) so that the basis stays
  full rank in every observed-frame window, as real PCA eigenvectors do;
  the ten functions are then orthonormalised (QR) and scaled to unit RMS.
  z grid: z_k = exp(ln 0.995 + 3e-4 k) - 1, k = 0..3310.
* QSO template: rest 500-10000 A at 0.5 A, 4 bases (continuum + broad
  Lya/CIV/CIII]/MgII with sigma = 20 A), z_k = exp(ln 1.05 + 5e-4 k) - 1,
  k = 0..3793, Inoue14 IGM.
* STAR templates: 5 subtypes, rest 3500-10000 A at 0.2 A, 5 bases each,
  z = linspace(-0.002, 0.002, 100), no IGM.
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field

import numpy as np

CAMERAS = (("b", 3600.0, 5800.0), ("r", 5760.0, 7620.0), ("z", 7520.0, 9824.0))
DWAVE = 0.8
NDIAG = 11


def camera_wave(lo, hi, step=DWAVE):
    return np.arange(lo, hi + 0.01, step)


def camera_grids():
    return {name: camera_wave(lo, hi) for name, lo, hi in CAMERAS}


def galaxy_zgrid(nz=3311):
    return np.exp(np.log(0.995) + 3e-4 * np.arange(nz)) - 1.0


def qso_zgrid(nz=3794):
    return np.exp(np.log(1.05) + 5e-4 * np.arange(nz)) - 1.0


def star_zgrid(nz=100):
    return np.linspace(-0.002, 0.002, nz)


# --------------------------------------------------------------------------
# resolution matrices
# --------------------------------------------------------------------------

def resolution_dia(npix, sigma, ndiag=NDIAG):
    """Banded Gaussian resolution in scipy DIA layout, rows normalised.

    Returns (data, offsets) with data[k, j] = R[j - offsets[k], j], the
    scipy ``dia_matrix`` convention.
    """
    half = ndiag // 2
    offsets = np.arange(-half, half + 1)
    kern = np.exp(-0.5 * (offsets / sigma) ** 2)
    # dense band by rows: band[i, k] = R[i, i + offsets[k]]
    band = np.tile(kern, (npix, 1))
    i = np.arange(npix)[:, None]
    col = i + offsets[None, :]
    band[(col < 0) | (col >= npix)] = 0.0
    band /= band.sum(axis=1, keepdims=True)
    data = np.zeros((ndiag, npix))
    for k, off in enumerate(offsets):
        rows = np.arange(npix)
        cols = rows + off
        ok = (cols >= 0) & (cols < npix)
        data[k, cols[ok]] = band[rows[ok], k]
    return data, offsets


def dia_to_dense(data, offsets, npix):
    R = np.zeros((npix, npix))
    for k, off in enumerate(offsets):
        for j in range(max(0, off), min(npix, npix + off)):
            R[j - off, j] = data[k, j]
    return R


def dia_matvec(data, offsets, x):
    """y = R x for a DIA matrix, x of shape (npix,) or (npix, m)."""
    npix = data.shape[1]
    y = np.zeros_like(x, dtype=np.float64)
    for k, off in enumerate(offsets):
        if off >= 0:
            n = npix - off
            if n <= 0:
                continue
            d = data[k, off:off + n]
            y[:n] += (d[:, None] * x[off:off + n]) if x.ndim == 2 else d * x[off:off + n]
        else:
            n = npix + off
            if n <= 0:
                continue
            d = data[k, :n]
            y[-off:] += (d[:, None] * x[:n]) if x.ndim == 2 else d * x[:n]
    return y


# --------------------------------------------------------------------------
# templates
# --------------------------------------------------------------------------

def _legendre(x, deg):
    return np.polynomial.legendre.legval(x, [0] * deg + [1])


def _gauss(wave, center, sigma):
    return np.exp(-0.5 * ((wave - center) / sigma) ** 2)


def _orthonormal(funcs):
    A = np.stack(funcs, axis=1)
    q, _ = np.linalg.qr(A)
    q *= np.sqrt(A.shape[0])
    # fix the sign so each basis correlates positively with its raw function
    for i in range(q.shape[1]):
        if np.dot(q[:, i], A[:, i]) < 0:
            q[:, i] = -q[:, i]
    return np.ascontiguousarray(q.T)


def galaxy_basis(step=0.2, lo=1200.0, hi=10000.0):
    wave = np.arange(lo, hi + step / 2, step)
    x = 2 * (wave - lo) / (hi - lo) - 1
    funcs = [(wave / 5000.0) ** -1.5]
    funcs += [_legendre(x, d) for d in range(1, 5)]
    lines = [
        [(3726.0, 1.0), (3728.8, 1.3)],
        [(4861.3, 1.0)],
        [(4958.9, 0.35), (5006.8, 1.0)],
        [(6548.0, 0.3), (6562.8, 1.0), (6583.4, 0.9)],
        [(6716.4, 1.0), (6730.8, 0.8)],
    ]
    periods = (350.0, 480.0, 610.0, 770.0, 950.0)
    for i, ln in enumerate(lines):
        g = sum(a * _gauss(wave, c, 2.0) for c, a in ln)
        funcs.append(g + 0.05 * np.sin(2 * np.pi * wave / periods[i] + 0.7 * i))
    return wave, _orthonormal(funcs)


def qso_basis(step=0.5, lo=500.0, hi=10000.0):
    wave = np.arange(lo, hi + step / 2, step)
    x = 2 * (wave - lo) / (hi - lo) - 1
    lines = (1215.67, 1549.06, 1908.73, 2798.75)
    strength = np.array([[1.0, 0.5, 0.25, 0.35],
                         [0.2, 1.0, 0.3, 0.1],
                         [0.1, 0.2, 1.0, 0.6],
                         [0.4, 0.1, 0.2, 1.0]])
    funcs = []
    for i in range(4):
        cont = (wave / 1500.0) ** (-0.5 - 0.3 * i) * (1 + 0.2 * np.sin(2 * np.pi * wave / (700.0 + 450.0 * i) + i))
        ln = sum(strength[i, j] * 3.0 * _gauss(wave, c, 20.0) for j, c in enumerate(lines))
        funcs.append(cont + ln)
    return wave, _orthonormal(funcs)


STAR_SUBTYPES = ("A", "F", "G", "K", "M")
_STAR_TEFF = {"A": 9000.0, "F": 6800.0, "G": 5700.0, "K": 4500.0, "M": 3300.0}


def star_basis(subtype, step=0.2, lo=3500.0, hi=10000.0):
    wave = np.arange(lo, hi + step / 2, step)
    x = 2 * (wave - lo) / (hi - lo) - 1
    teff = _STAR_TEFF[subtype]
    lam_cm = wave * 1e-8
    bb = 1.0 / (lam_cm ** 5 * (np.exp(1.4388 / (lam_cm * teff)) - 1.0))
    bb /= bb.max()
    absl = [3933.7, 3968.5, 4101.7, 4340.5, 4861.3, 5175.0, 5892.9, 6562.8, 8542.1]
    depth = 0.5 * sum(_gauss(wave, c, 3.0) for c in absl)
    funcs = [bb * (1 - depth),
             bb * _legendre(x, 1),
             bb * _legendre(x, 2) + 0.1 * depth,
             _legendre(x, 3) + 0.2 * _gauss(wave, 6562.8, 5.0),
             _legendre(x, 4) - 0.3 * depth * (1 + 0.5 * _legendre(x, 5))]
    return wave, _orthonormal(funcs)


@dataclass
class ArchetypeSpec:
    """A redrock-format archetype set: ``flux`` (narch, nwave) on a linear
    rest grid, one subtype name per row, spectral class ``rrtype``."""
    rrtype: str
    wave: np.ndarray
    flux: np.ndarray
    subtype: list
    version: str = "synthetic"


def archetype_set(narch=24, seed=5, rrtype="GALAXY", step=0.5, lo=800.0, hi=10000.0):
    """Positive rest-frame galaxy-like spectra: a power-law continuum with a
    4000 A break and a weak ripple, plus the [OII], Hb, [OIII], Ha+[NII],
    [SII], Lya and MgII lines (sigma 2-6 A) with random strengths."""
    rng = np.random.default_rng(seed)
    wave = np.arange(lo, hi + step / 2, step)
    lines = (1215.67, 2798.75, 3727.0, 4861.3, 4958.9, 5006.8, 6562.8, 6583.4, 6716.4, 6730.8)
    flux = np.zeros((narch, len(wave)))
    for i in range(narch):
        slope = rng.uniform(-2.5, -0.5)
        cont = (wave / 5000.0) ** slope
        cont *= 1.0 - rng.uniform(0.0, 0.5) / (1.0 + np.exp((wave - 4000.0) / 30.0))
        cont *= 1.0 + 0.05 * np.sin(2 * np.pi * wave / rng.uniform(300.0, 900.0))
        amp = rng.uniform(0.0, 3.0, size=len(lines)) * (rng.uniform(size=len(lines)) < 0.8)
        sig = rng.uniform(2.0, 6.0)
        flux[i] = cont + sum(a * _gauss(wave, c, sig) for a, c in zip(amp, lines))
    sub = ["ELG" if i % 3 == 0 else ("LRG" if i % 3 == 1 else "BGS") for i in range(narch)]
    return ArchetypeSpec(rrtype, wave, flux, sub)


@dataclass
class TemplateSpec:
    spectype: str
    subtype: str
    wave: np.ndarray
    flux: np.ndarray
    redshifts: np.ndarray
    igm_model: str
    method: str = "PCA"

    @property
    def full_type(self):
        return f"{self.spectype}:::{self.subtype}" if self.subtype else self.spectype


def template_set(nz_galaxy=3311, nz_qso=3794, nz_star=100, stars=STAR_SUBTYPES,
                 zsub=None):
    """GALAXY + QSO + STAR subtypes.  ``zsub`` keeps every zsub-th redshift."""
    out = []
    gw, gf = galaxy_basis()
    out.append(TemplateSpec("GALAXY", "", gw, gf, galaxy_zgrid(nz_galaxy), "Inoue14"))
    qw, qf = qso_basis()
    out.append(TemplateSpec("QSO", "", qw, qf, qso_zgrid(nz_qso), "Inoue14"))
    for st in stars:
        sw, sf = star_basis(st)
        out.append(TemplateSpec("STAR", st, sw, sf, star_zgrid(nz_star), "None"))
    if zsub:
        for t in out:
            t.redshifts = np.ascontiguousarray(t.redshifts[::zsub])
    return out


# --------------------------------------------------------------------------
# targets
# --------------------------------------------------------------------------

@dataclass
class SpectrumSpec:
    band: str
    wave: np.ndarray
    flux: np.ndarray
    ivar: np.ndarray
    rdata: np.ndarray      # (ndiag, npix) DIA data
    roffsets: np.ndarray   # (ndiag,)


@dataclass
class TargetSpec:
    targetid: int
    spectra: list = field(default_factory=list)
    ztrue: float = 0.0


def trapz_rebin_np(x, y, edges):
    """Small numpy trapezoid rebin used only to render synthetic flux.

    Integrates the piecewise-linear y(x) over each bin (exact for linear
    interpolation) via the cumulative integral; (nbin,) or (nbin, m)."""
    y2 = y if y.ndim == 2 else y[:, None]
    cum = np.concatenate([np.zeros((1, y2.shape[1])),
                          np.cumsum(0.5 * (y2[1:] + y2[:-1]) * np.diff(x)[:, None], axis=0)])

    def cumint(e):
        j = np.clip(np.searchsorted(x, e, side="right") - 1, 0, len(x) - 2)
        t = (e - x[j])
        slope = (y2[j + 1] - y2[j]) / (x[j + 1] - x[j])[:, None]
        return cum[j] + t[:, None] * (y2[j] + 0.5 * slope * t[:, None])

    ce = cumint(np.asarray(edges, dtype=np.float64))
    out = (ce[1:] - ce[:-1]) / np.diff(edges)[:, None]
    return out if y.ndim == 2 else out[:, 0]


def centers_to_edges(c):
    c = np.asarray(c, dtype=np.float64)
    e = np.zeros(len(c) + 1)
    e[1:-1] = (c[:-1] + c[1:]) / 2.0
    e[0] = c[0] - (c[1] - e[1])
    e[-1] = c[-1] + (c[-1] - e[-2])
    return e


def make_targets(ntarget, seed=0, template=None, zrange=(0.0, 1.5), amp=1.0,
                 snr_range=None, mask_frac=0.05, mask_range=None,
                 drop_camera_frac=0.0, sigma_r=(0.8, 1.2), cameras=CAMERAS,
                 first_id=1000, transmission=None):
    """Seeded synthetic targets.

    Flux = R . rebin(template(z_true) . c) + N(0, sigma) with random
    coefficients c ~ N(0, 1) * amp (or amp drawn log-uniform from
    ``snr_range`` when given), sigma ~ U(0.5, 2), a random fraction of masked
    pixels, optionally one camera dropped for a fraction of targets.
    ``transmission(z, wave) -> T`` (e.g. an IGM model) multiplies the
    rendered template before the resolution is applied.
    """
    rng = np.random.default_rng(seed)
    if template is None:
        gw, gf = galaxy_basis()
        template = (gw, gf)
    twave, tflux = template
    grids = {name: camera_wave(lo, hi) for name, lo, hi in cameras}
    edges = {k: centers_to_edges(w) for k, w in grids.items()}
    out = []
    for it in range(ntarget):
        z = rng.uniform(*zrange)
        a = amp if snr_range is None else np.exp(rng.uniform(np.log(snr_range[0]), np.log(snr_range[1])))
        c = rng.normal(size=tflux.shape[0]) * a
        mf = mask_frac if mask_range is None else rng.uniform(*mask_range)
        drop = None
        if drop_camera_frac > 0 and rng.uniform() < drop_camera_frac:
            drop = int(rng.integers(len(cameras)))
        tg = TargetSpec(first_id + it, ztrue=z)
        model_rest = tflux.T @ c
        for ic, (name, lo, hi) in enumerate(cameras):
            wave = grids[name]
            npix = len(wave)
            sig_r = rng.uniform(*sigma_r)
            rdata, roff = resolution_dia(npix, sig_r)
            noise = rng.uniform(0.5, 2.0, size=npix)
            ivar = 1.0 / noise ** 2
            ivar[rng.uniform(size=npix) < mf] = 0.0
            if ic == drop:
                continue
            m = trapz_rebin_np(twave * (1 + z), model_rest, edges[name])
            if transmission is not None:
                m = m * np.asarray(transmission(z, wave), dtype=np.float64)
            flux = dia_matvec(rdata, roff, m) + rng.normal(size=npix) * noise
            tg.spectra.append(SpectrumSpec(name, wave, flux, ivar, rdata, roff))
        out.append(tg)
    return out


def multi_exposure_targets(ntarget, seed=0, nexp=(1, 3), cosmics=0):
    """Targets with 1-3 exposures per camera -- the input of redrock's
    Target.compute_coadd.  Each exposure has its own resolution width,
    noise, extra noise on the flux and 5 % random masking; about 1 % of the
    pixels of each camera are masked in every exposure (the all-masked
    branch of the coadd).  ``cosmics`` > 0 adds that many cosmic-ray hits
    per exposure: 1-3 adjacent pixels raised by 20-200 sigma."""
    rng = np.random.default_rng(seed)
    base = make_targets(ntarget, seed=seed + 1, mask_frac=0.0)
    out = []
    for t in base:
        tg = TargetSpec(t.targetid, ztrue=t.ztrue)
        for s in t.spectra:
            npix = len(s.wave)
            dead = rng.uniform(size=npix) < 0.01
            for _ in range(int(rng.integers(nexp[0], nexp[1] + 1))):
                rdata, roff = resolution_dia(npix, rng.uniform(0.8, 1.2))
                noise = rng.uniform(0.5, 2.0, size=npix)
                ivar = 1.0 / noise ** 2
                ivar[(rng.uniform(size=npix) < 0.05) | dead] = 0.0
                flux = s.flux + rng.normal(size=npix) * noise
                for _ in range(cosmics):
                    j = int(rng.integers(npix - 3))
                    w = int(rng.integers(1, 4))
                    flux[j:j + w] += rng.uniform(20.0, 200.0) * noise[j:j + w]
                tg.spectra.append(SpectrumSpec(s.band, s.wave, flux, ivar, rdata, roff))
        out.append(tg)
    return out


def make_population(ntarget, seed=0, qso_frac=0.0, snr_range=None, mask_range=None,
                    drop_camera_frac=0.0, transmission=None, first_id=1000):
    """Mixed GALAXY / QSO-like targets, shuffled: a fraction qso_frac drawn
    from the QSO basis at z ~ U(0.05, 6) (rendered with ``transmission``,
    e.g. an IGM model), the rest GALAXY at z ~ U(0, 1.5)."""
    rng = np.random.default_rng(seed)
    nq = int(round(qso_frac * ntarget))
    kw = dict(snr_range=snr_range, mask_range=mask_range, drop_camera_frac=drop_camera_frac)
    gal = make_targets(ntarget - nq, seed=seed + 1, first_id=first_id, **kw)
    qso = make_targets(nq, seed=seed + 2, template=qso_basis(), zrange=(0.05, 6.0),
                       first_id=first_id + ntarget - nq, transmission=transmission, **kw)
    out = gal + qso
    order = rng.permutation(len(out))
    return [out[i] for i in order]


def checksum(arrays):
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def targets_checksum(targets):
    arrs = []
    for t in targets:
        for s in t.spectra:
            arrs += [s.wave, s.flux, s.ivar, s.rdata, s.roffsets]
    return checksum(arrs)


# --------------------------------------------------------------------------
# the fake template/target of redrock's own test utilities
# (py/redrock/test/util.py:12-75): 3 bases on 100-9000 A at 5 A, two
# cameras at 5 A with two exposures each, R from a sampled Gaussian with
# exp(-x^2 / (2 sigma)) (sic) normalised to sum 1.
# --------------------------------------------------------------------------

def util_template(wavemin=100, wavemax=9000, wavestep=5):
    wave = np.arange(wavemin, wavemax + wavestep / 2.0, wavestep)
    flux = np.zeros((3, len(wave)))
    wavemid = (wavemin + wavemax) / 2.0
    wx = np.pi * (2 * (wave - wavemin) / (wavemax - wavemin) - 1)
    flux[0] = 1.0
    flux[1] = np.arange(len(wave)) / len(wave)
    flux[2] = np.exp(-(wave - wavemid) ** 2 / (2 * 20 ** 2)) + 0.1 * np.sin(wx)
    return wave, flux


def util_R(n, sigma=2.0):
    x = np.arange(-5, 6)
    y = np.exp(-x ** 2 / (2.0 * sigma))
    y = y / np.sum(y)
    data = np.zeros((11, n))
    for i in range(n):
        data[:, i] = y
    return data, x


def util_target(z, seed, targetid, wavestep=5):
    rng = np.random.default_rng(seed)
    twave, tflux = util_template()
    c = np.array([1.0, 2.0, 3.0])
    tg = TargetSpec(targetid, ztrue=z)
    for band, wave in (("b", np.arange(4000, 6700, wavestep, dtype=np.float64)),
                       ("r", np.arange(6502, 8001, wavestep, dtype=np.float64))):
        flux = trapz_rebin_np(twave * (1 + z), tflux.T @ c, centers_to_edges(wave))
        sigma = np.clip(rng.normal(loc=1, scale=0.1, size=len(wave)), 0.5, 1.5)
        ivar = 1 / sigma ** 2
        rdata, roff = util_R(len(wave), 2.0)
        for _ in range(2):
            noisy = flux + rng.normal(size=len(wave)) * sigma
            # R is not applied to the model, as in the reference's fixture
            tg.spectra.append(SpectrumSpec(band, wave, noisy, ivar.copy(), rdata, roff))
    return tg
