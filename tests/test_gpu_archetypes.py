"""Archetype fits on the GPU against redrock's own (fixture made by
tests/golden/make_archetype_golden.py) and against the oracle.

Tolerances: best archetype names identical; chi2 relative 1e-8;
coefficients |dc| <= 1e-6 max(1, max|c|) (the solves are FP64 on the same
normal equations; the batched Gram sums run in another order).  fitz with
archetypes: redshifts |dz| <= 1e-7 and ZWARN identical (the template part,
as in test_gpu_fitz), archetype names identical, chi2 relative 1e-8.
zfind with archetypes: the columns of test_gpu_zfind with its tolerances,
plus the archetype columns (fitmethod, pca_* identical; coefficients
|dc| <= 1e-5 max(1, max|c|) per row).
"""
import os

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from redrock_b200 import synth  # noqa: E402
from tests.archetype_cases import (CASES, FITZ_CASES, ZFIND_CASES, archetype_targets,  # noqa: E402
                                   fitz_targets)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "archetype_golden.npz")


@pytest.fixture(scope="module")
def ag():
    return dict(np.load(GOLDEN))


def _close_coeff(a, b):
    b = np.asarray(b)
    assert np.asarray(a).shape == b.shape
    tol = 1e-6 * max(1.0, np.abs(b).max() if b.size else 1.0)
    assert np.all(np.abs(np.asarray(a) - b) <= tol), np.abs(np.asarray(a) - b).max()


def _fit_inputs(t, z):
    from redrock_b200.igm import transmission_Lyman
    from redrock_b200.zscan import spectral_data
    dwave = {s.wavehash: s.wave for s in t.spectra}
    w, f, wf = spectral_data(t.spectra)
    trans = {hs: transmission_Lyman(np.array([z]), wv, always_return_array=False,
                                    model='Inoue14') for hs, wv in dwave.items()}
    return dwave, w, f, wf, trans


@pytest.mark.parametrize("name", list(CASES))
def test_get_best_archetype_vs_redrock(ag, name):
    from redrock_b200 import archetypes as A, fitz, targets as T
    per_camera, nleg, nn, psig, method = CASES[name]
    spec, tg = archetype_targets()
    assert synth.targets_checksum(tg) == str(ag["arch_targets_sha"])
    arch = A.Archetype.from_synth(spec)
    for j, t in enumerate(T.from_synth(tg)):
        z = tg[j].ztrue
        t.legendre(nleg)
        dwave, w, f, wf, trans = _fit_inputs(t, z)
        ncam = len(dwave) if per_camera else 1
        prior = (None if psig is None else
                 fitz.prior_on_coeffs(1 if nn is None else nn, nleg, psig, ncam))
        c2, co, ft = arch.get_best_archetype(t, w, f, wf, dwave, z, per_camera, nn, trans=trans,
                                             solve_method=method, prior=prior)
        assert ft == str(ag[f"arch_{name}_{j}_fulltype"]), (name, j)
        np.testing.assert_allclose(c2, ag[f"arch_{name}_{j}_chi2"], rtol=1e-8)
        _close_coeff(co, ag[f"arch_{name}_{j}_coeff"])


def test_per_camera_nnls_and_nearest_pca_vs_oracle():
    """Cases outside the fixture, against the oracle: per-camera fits with
    NNLS on every archetype, and nearest archetypes with one Legendre set
    for the whole spectrum (solved with PCA here; redrock passes no solve
    method there and fails)."""
    from oracle import oracle as O
    from redrock_b200 import archetypes as A, targets as T
    from redrock_b200.zscan import per_camera_coeff_with_least_square_batch
    spec, tg = archetype_targets()
    arch = A.Archetype.from_synth(spec)
    oarch = O.OArchetype(spec.wave, spec.flux, spec.rrtype, spec.subtype)
    for j, (ts, t) in enumerate(zip(tg[:2], T.from_synth(tg[:2]))):
        z = ts.ztrue
        t.legendre(2)
        dwave, w, f, wf, trans = _fit_inputs(t, z)
        osp = [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
               for s in ts.spectra]
        leg = O.legendre_dict(dwave, 2)
        binned = oarch.rebin(z, dwave)
        tdata = {hs: np.append(binned[hs].T[:, :, None],
                               np.tile(leg[hs].T[None], (oarch.narch, 1, 1)), axis=2)
                 for hs in dwave}
        bands = [s.band for s in ts.spectra]
        oc2, oco = O.per_camera_coeff(osp, tdata, w, f, wf, 2, oarch.narch, 'nnls', 1, None,
                                      bands)
        c2, co = per_camera_coeff_with_least_square_batch(t, tdata, w, f, wf, 2, oarch.narch,
                                                          method='nnls', n_nbh=1, bands=bands)
        np.testing.assert_allclose(c2, oc2, rtol=1e-8)
        _close_coeff(co, oco)
        prior = O.prior_on_coeffs(2, 2, 0.1, 1)
        otr = {hs: (None if trans[hs] is None else trans[hs][0]) for hs in trans}
        oc2, oco, oft = O.get_best_archetype(oarch, osp, bands, leg, w, f, wf, dwave, z, False, 2,
                                             otr, 'bvls', prior)
        c2, co, ft = arch.get_best_archetype(t, w, f, wf, dwave, z, False, 2, trans=trans,
                                             prior=prior)
        assert ft == oft
        np.testing.assert_allclose(c2, oc2, rtol=1e-8)
        _close_coeff(co, oco)


@pytest.mark.parametrize("name", list(FITZ_CASES))
def test_fitz_with_archetypes_vs_redrock(golden, ag, name):
    from redrock_b200 import archetypes as A, fitz, targets as T, templates as TM
    per_camera, nn, psig = FITZ_CASES[name]
    spec, _ = archetype_targets()
    arch = A.Archetype.from_synth(spec)
    ts = synth.template_set()[0]
    ts.redshifts = golden["scan_GALAXY_z"]
    tg = T.from_synth(fitz_targets())
    chi2 = [golden["scan_GALAXY_zchi2"][j] + golden["scan_GALAXY_penalty"][j]
            for j in range(len(tg))]
    out = fitz.fitz_targets(chi2, ts.redshifts, tg, TM.from_synth(ts), nminima=3,
                            archetype=arch, deg_legendre=2, per_camera=per_camera,
                            n_nearest=nn, prior_sigma=psig)
    for j, r in enumerate(out):
        g = {k: ag[f"afitz_{name}_{j}_{k}"] for k in ("z", "zerr", "zwarn", "chi2", "coeff",
                                                      "legcoeff", "fulltype", "pca_coeff",
                                                      "npixels")}
        assert list(r.keys())[:13] == ["z", "zerr", "zwarn", "chi2", "zz", "zzchi2", "coeff",
                                       "legcoeff", "fulltype", "fitmethod", "pca_coeff",
                                       "pca_spectype", "pca_subtype"]
        np.testing.assert_array_equal(r["fulltype"], g["fulltype"])
        np.testing.assert_array_equal(r["zwarn"], g["zwarn"])
        np.testing.assert_array_equal(r["npixels"], g["npixels"])
        np.testing.assert_allclose(r["z"], g["z"], rtol=0, atol=1e-7)
        np.testing.assert_allclose(r["chi2"], g["chi2"], rtol=1e-8)
        _close_coeff(r["coeff"], g["coeff"])
        _close_coeff(r["legcoeff"], g["legcoeff"])
        _close_coeff(r["pca_coeff"], g["pca_coeff"])
        assert np.all(r["fitmethod"] == "ARCH")


@pytest.mark.parametrize("name", list(ZFIND_CASES))
def test_zfind_with_archetypes_vs_redrock(ag, name):
    """zfind with GALAXY archetypes (per camera, prior 0.1) on the zfind
    fixture: the archetype columns, NEGATIVE_MODEL bits and the final
    coefficient width follow redrock's finalisation."""
    from redrock_b200 import archetypes as A, targets as T, templates as TM
    from redrock_b200.zfind import zfind
    spec, _ = archetype_targets()
    arch = A.Archetype.from_synth(spec)
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    dz = T.DistTargetsCopy(T.from_synth(ztg))
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    dts = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
    _, zfit = zfind(dz, dts, nminima=3, archetypes={"GALAXY": arch}, per_camera=True,
                    deg_legendre=2, n_nearest=ZFIND_CASES[name], prior_sigma=0.1, ncamera=3)
    g = {k: ag[f"azfind_{name}_{k}"] for k in ag[f"azfind_{name}_columns"]}
    assert list(zfit.keys()) == list(g.keys())
    for k in ("targetid", "spectype", "subtype", "zwarn", "znum", "ncoeff", "npixels",
              "fitmethod", "pca_spectype", "pca_subtype"):
        np.testing.assert_array_equal(zfit[k], g[k], err_msg=k)
    np.testing.assert_allclose(zfit["z"], g["z"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(zfit["zz"], g["zz"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(zfit["zerr"], g["zerr"], rtol=1e-5)
    for k in ("chi2", "deltachi2", "zzchi2"):
        assert np.max(np.abs(zfit[k] - g[k])) <= 1e-3, k
    for k in ("coeff", "pca_coeff", "legcoeff"):
        assert zfit[k].shape == g[k].shape, k
        scale = np.maximum(np.abs(g[k]).reshape(len(g[k]), -1).max(axis=1), 1.0)
        d = np.abs(zfit[k] - g[k]).reshape(len(g[k]), -1).max(axis=1)
        assert np.all(d <= 1e-5 * scale), (k, d.max())


@pytest.mark.parametrize("name", ["pc", "nc", "pcnn", "pc0"])
def test_best_archetypes_batch_vs_oracle(name):
    """best_archetypes: all targets' fits in one rr_archetype_fit launch (and
    in groups of two through a small max_bytes) against the oracle's
    per-target get_best_archetype."""
    from oracle import oracle as O
    from redrock_b200 import archetypes as A, fitz, targets as T
    per_camera, nleg, nn, psig, method = CASES[name]
    spec, tg = archetype_targets()
    arch = A.Archetype.from_synth(spec)
    oarch = O.OArchetype(spec.wave, spec.flux, spec.rrtype, spec.subtype)
    rt = T.from_synth(tg)
    items, want = [], []
    for ts, t in zip(tg, rt):
        for dz in (0.0, 0.01):
            z = ts.ztrue + dz
            t.legendre(nleg)
            dwave, w, f, wf, trans = _fit_inputs(t, z)
            items.append((t, z, trans))
            ncam = len(dwave) if per_camera else 1
            prior = (None if psig is None else
                     fitz.prior_on_coeffs(1 if nn is None else nn, nleg, psig, ncam))
            osp = [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
                   for s in ts.spectra]
            otr = {hs: (None if trans[hs] is None else trans[hs][0]) for hs in trans}
            want.append(O.get_best_archetype(oarch, osp, [s.band for s in ts.spectra],
                                             O.legendre_dict(dwave, nleg), w, f, wf, dwave, z,
                                             per_camera, nn, otr, method, prior))
    for max_bytes in (1 << 31, 2 * arch._narch * 8200 * 8):
        got = arch.best_archetypes(items, per_camera, nn, solve_method=method, prior=prior,
                                   max_bytes=max_bytes)
        for (c2, co, ft), (oc2, oco, oft) in zip(got, want):
            assert ft == oft
            np.testing.assert_allclose(c2, oc2, rtol=1e-8)
            _close_coeff(co, oco)


@pytest.mark.parametrize("per_camera,nleg", [(True, 2), (False, 2), (False, 0)])
def test_archetype_multi_exposure_target_vs_oracle(per_camera, nleg):
    """redrock's own archetype unit case (test_archetypes.py:55-95): a
    target with two exposures per camera (util.get_target), bands set to
    ['b', 'r'], z = 0.5, with and without Legendre terms: coefficient
    counts 1 + nleg * 2 (per camera) / 1 + nleg, and the fit against the
    oracle."""
    from oracle import oracle as O
    from redrock_b200 import archetypes as A, fitz, targets as T
    from redrock_b200.zscan import spectral_data
    spec, _ = archetype_targets()
    arch = A.Archetype.from_synth(spec)
    oarch = O.OArchetype(spec.wave, spec.flux, spec.rrtype, spec.subtype)
    ut = synth.util_target(0.5, seed=23, targetid=123)
    t = T.from_synth([ut])[0]
    t.bands = ['b', 'r']
    t.nleg = nleg
    dwave = {s.wavehash: s.wave for s in t.spectra}
    w, f, wf = spectral_data(t.spectra)
    prior = fitz.prior_on_coeffs(1, nleg, 0.1, len(dwave)) if nleg else None
    c2, co, ft = arch.get_best_archetype(t, w, f, wf, dwave, 0.5, per_camera, None, trans=None,
                                         solve_method='bvls', prior=prior)
    assert len(co) == (1 + nleg * len(t.bands) if per_camera else 1 + nleg)
    osp = [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets) for s in ut.spectra]
    oc2, oco, oft = O.get_best_archetype(oarch, osp, ['b', 'r'], O.legendre_dict(dwave, nleg),
                                         w, f, wf, dwave, 0.5, per_camera, None, None, 'bvls',
                                         prior)
    assert ft == oft
    np.testing.assert_allclose(c2, oc2, rtol=1e-8)
    _close_coeff(co, oco)
