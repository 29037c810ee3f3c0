"""The oracle (CPU restatement) against fixtures produced by redrock itself."""
import os
import numpy as np
import pytest

from oracle import oracle as O
from redrock_b200 import synth


def test_rebin_known_answers(golden):
    x = np.arange(10.)
    y = np.ones((2, 10))
    y[1] = np.arange(10)
    np.testing.assert_array_equal(O.trapz_rebin(x, y, edges=[0, 2, 4, 6, 8], myz=[0.0, 0.5]),
                                  golden["rebin_doc"])
    xu = np.linspace(0, 10, 100) ** 2
    np.testing.assert_array_equal(O.trapz_rebin(xu, np.sqrt(xu), edges=np.linspace(0, 100, 21)),
                                  golden["rebin_uneven"])
    xs = np.linspace(0, 2 * np.pi, 100)
    np.testing.assert_array_equal(
        O.trapz_rebin(xs, np.sin(xs), edges=[0, 0.5 * np.pi, np.pi, 1.5 * np.pi, 2 * np.pi]),
        golden["rebin_sin"])


def test_rebin_redrock_unit_cases():
    # redrock test_rebin.py: constant density stays exactly 1
    x = np.arange(10) * 1.1
    y = np.ones(10)
    for nedge in range(3, 10):
        assert np.all(O.trapz_rebin(x, y, edges=np.linspace(x.min(), x.max(), nedge)) == 1.0)
    assert np.allclose(O.trapz_rebin(np.arange(10), np.ones(10), np.linspace(0.5, 8.5)), 1.0)
    with pytest.raises(ValueError):
        O.trapz_rebin(np.arange(10), np.ones(10), edges=np.arange(-1, 9))
    with pytest.raises(ValueError):
        O.trapz_rebin(np.arange(10), np.ones(10), edges=np.arange(1, 11))


@pytest.mark.parametrize("key", ["GALAXY", "QSO", "STAR_G"])
def test_basis_bit_exact(golden, key):
    grids = synth.camera_grids()
    ts = {t.full_type.replace(":::", "_"): t for t in synth.template_set()}[key]
    zz = golden[f"basis_{key}_z"]
    r = O.trapz_rebin(ts.wave, ts.flux, xnew=grids["b"], myz=zz)
    assert synth.checksum([r]) == str(golden[f"rebin_{key}_b_sha"])
    data = O.template_basis(ts.wave, ts.flux, zz, grids, ts.igm_model)
    for cam in grids:
        d = data[cam]
        np.testing.assert_allclose(d[:, ::13], golden[f"basis_{key}_{cam}_sample"], rtol=1e-13,
                                   atol=0)


@pytest.mark.parametrize("model", ["Inoue14", "Calura12", "Kamble20"])
def test_igm(golden, model):
    T = O.transmission_Lyman(golden["igm_z"], golden["igm_lobs"], model=model)
    np.testing.assert_allclose(T, golden[f"igm_{model}"], rtol=1e-14, atol=1e-300)


def test_igm_shapes_and_high_z(golden):
    np.testing.assert_allclose(O.transmission_Lyman(4.2, golden["igm_lobs"], model="Inoue14"),
                               golden["igm_Inoue14_scalar_z"], rtol=1e-14)
    np.testing.assert_allclose(O.transmission_Lyman(golden["igm_z"], 3650.0, model="Inoue14"),
                               golden["igm_Inoue14_scalar_l"], rtol=1e-14)
    np.testing.assert_allclose(
        O.transmission_Lyman(golden["igm_hi_z"], golden["igm_hi_lobs"], model="Inoue14"),
        golden["igm_hi_Inoue14"], rtol=1e-14, atol=1e-300)
    assert O.transmission_Lyman(np.array([0.1, 0.2]), np.array([5000.0, 6000.0]), model="Inoue14",
                                always_return_array=False) is None
    with pytest.raises(ValueError):
        O.transmission_Lyman(1.0, 1000.0, model="bogus")


def _ospectra(t):
    return [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets) for s in t.spectra]


def _scan_targets():
    tg = synth.make_targets(4, seed=11, amp=1.0)
    tg += synth.make_targets(1, seed=12, mask_range=(0.4, 0.4), first_id=2000)
    tg += synth.make_targets(1, seed=13, drop_camera_frac=1.0, first_id=3000)
    tg += synth.make_targets(1, seed=14, first_id=4000)
    for s in tg[-1].spectra:
        s.ivar[:] = 0.0
    return tg


@pytest.mark.parametrize("key", ["GALAXY", "QSO", "STAR_G"])
def test_calc_zchi2(golden, key):
    tg = _scan_targets()
    assert synth.targets_checksum(tg) == str(golden["scan_targets_sha"])
    ts = {t.full_type.replace(":::", "_"): t for t in synth.template_set()}[key]
    zz = golden[f"scan_{key}_z"]
    grids = synth.camera_grids()
    tdata = O.template_basis(ts.wave, ts.flux, zz, grids, ts.igm_model)
    oii = O.oii_template(ts.wave, ts.flux) if ts.spectype == "GALAXY" else None
    zc, co, pe = O.calc_zchi2([_ospectra(t) for t in tg], tdata, len(zz), ts.flux.shape[0],
                              OIItemplate=oii)
    np.testing.assert_allclose(zc, golden[f"scan_{key}_zchi2"], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(co, golden[f"scan_{key}_zcoeff"], rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(pe, golden[f"scan_{key}_penalty"], rtol=1e-8, atol=1e-10)
    assert np.all(zc[-1] == O.HUGE_CHI2)


def test_util_fixture(golden):
    ut = [synth.util_target(0.2, seed=21, targetid=111),
          synth.util_target(0.25, seed=22, targetid=222)]
    assert synth.targets_checksum(ut) == str(golden["util_targets_sha"])
    uw, uf = synth.util_template()
    zz = np.linspace(0.15, 0.3, 50)
    dwave = {s.band: s.wave for t in ut for s in t.spectra}
    tdata = O.template_basis(uw, uf, zz, dwave, "Inoue14")
    zc, co, pe = O.calc_zchi2([_ospectra(t) for t in ut], tdata, len(zz), 3,
                              OIItemplate=O.oii_template(uw, uf))
    for i, t in enumerate(ut):
        np.testing.assert_allclose(zc[i], golden[f"util_{t.targetid}_zchi2"], rtol=1e-10)
        np.testing.assert_allclose(co[i], golden[f"util_{t.targetid}_zcoeff"], rtol=1e-8)
        np.testing.assert_allclose(pe[i], golden[f"util_{t.targetid}_penalty"], atol=1e-10)


def test_prior_one_singular(golden):
    tg = _scan_targets()
    gal = synth.template_set()[0]
    grids = synth.camera_grids()
    zb = golden["prior_z"]
    tdata = O.template_basis(gal.wave, gal.flux, zb, grids, gal.igm_model)
    sp = _ospectra(tg[0])
    w, f, wf = O.spectral_data(sp)
    zc, co = O.calc_zchi2_batch(sp, tdata, w, f, wf, len(zb), 10, prior=golden["prior_matrix"])
    np.testing.assert_allclose(zc, golden["prior_zchi2"], rtol=1e-10)
    np.testing.assert_allclose(co, golden["prior_zcoeff"], rtol=1e-8)
    for i in range(len(zb)):
        c2, c = O.calc_zchi2_one(sp, w, f, wf, {k: v[i] for k, v in tdata.items()})
        np.testing.assert_allclose(c2, golden["one_zchi2"][i], rtol=1e-10)
        np.testing.assert_allclose(c, golden["one_zcoeff"][i], rtol=1e-8)
    sflux = gal.flux.copy()
    sflux[3] = 0.0
    tdata = O.template_basis(gal.wave, sflux, zb, grids, gal.igm_model)
    zc, co, pe = O.calc_zchi2([sp], tdata, len(zb), 10, OIItemplate=O.oii_template(gal.wave, sflux))
    np.testing.assert_array_equal(zc, golden["singular_zchi2"])
    np.testing.assert_array_equal(co, golden["singular_zcoeff"])


def test_coadd_oracle_vs_redrock_golden():
    """The oracle's compute_coadd reproduces redrock's Target(coadd=True)
    bit for bit (checksums of flux, ivar and resolution data)."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "coadd_golden.npz"))
    tg = synth.multi_exposure_targets(4, seed=61)
    assert synth.targets_checksum(tg) == str(g["coadd_targets_sha"])
    for it, t in enumerate(tg):
        exps = [(s.band, s.wave, s.flux, O.masked_ivar(s.ivar, s.rdata, s.roffsets), s.rdata,
                 s.roffsets) for s in t.spectra]
        out = O.compute_coadd(exps)
        assert len(out) == int(g[f"coadd_{it}_nspec"][1])
        for j, (band, wave, f, w, rd, ro) in enumerate(out):
            assert band == str(g[f"coadd_{it}_{j}_band"])
            assert synth.checksum([f, w, rd]) == str(g[f"coadd_{it}_{j}_sha"])


def test_bounded_solves_oracle_vs_redrock_golden():
    """The oracle's NNLS / BVLS branches of solve_matrices reproduce
    redrock's calc_zchi2_batch and its NMF calc_zchi2."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "lsq_golden.npz"))
    tg = synth.make_targets(2, seed=11, amp=1.0)
    assert synth.targets_checksum(tg) == str(g["lsq_targets_sha"])
    gal = synth.template_set()[0]
    zb = g["lsq_z"]
    nb = gal.flux.shape[0]
    tdata = O.template_basis(gal.wave, gal.flux, zb, synth.camera_grids(), gal.igm_model)
    lo, hi = g["lsq_bounds"]
    for it, t in enumerate(tg):
        sp = [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets) for s in t.spectra]
        w, f, wf = O.spectral_data(sp)
        for name, alg, args in (("nnls", "NNLS", None),
                                ("bvls", "BVLS", {"bounds": (np.full(nb, lo), np.full(nb, hi))}),
                                ("bvls_free", "BVLS", None)):
            zc, co = O.calc_zchi2_batch(sp, tdata, w, f, wf, len(zb), nb, alg, solver_args=args)
            np.testing.assert_allclose(zc, g[f"lsq_{name}_{it}_zchi2"], rtol=1e-10, atol=1e-8)
            np.testing.assert_allclose(co, g[f"lsq_{name}_{it}_zcoeff"], rtol=1e-8, atol=1e-10)
    osp = [[O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets) for s in t.spectra]
           for t in tg]
    # redrock caches the [OII] template for GALAXY PCA templates only
    # (templates.py:170-174), so an NMF template has no penalty
    zc, co, pe = O.calc_zchi2(osp, tdata, len(zb), nb, "NMF", OIItemplate=None)
    np.testing.assert_allclose(zc, g["lsq_nmf_zchi2"], rtol=1e-10, atol=1e-8)
    np.testing.assert_allclose(co, g["lsq_nmf_zcoeff"], rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(pe, g["lsq_nmf_penalty"], rtol=1e-8, atol=1e-10)


def _archetype_golden():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "archetype_golden.npz"))


def test_archetype_oracle_vs_redrock():
    """The oracle's archetype fit (rebin x IGM, Legendre terms, batched
    bounded solves, nearest archetypes) reproduces redrock's
    get_best_archetype on every case of the fixture."""
    from tests.archetype_cases import CASES, archetype_targets
    g = _archetype_golden()
    spec, tg = archetype_targets()
    assert synth.targets_checksum(tg) == str(g["arch_targets_sha"])
    assert synth.checksum([spec.wave, spec.flux]) == str(g["arch_flux_sha"])
    arch = O.OArchetype(spec.wave, spec.flux, spec.rrtype, spec.subtype)
    for name, (per_camera, nleg, nn, psig, method) in CASES.items():
        for j, t in enumerate(tg):
            sp = _ospectra(t)
            z = t.ztrue
            dwave = {s.wavehash: s.wave for s in sp}
            w, f, wf = O.spectral_data(sp)
            trans = {}
            for hs, wv in dwave.items():
                T = O.transmission_Lyman(np.array([z]), wv, model='Inoue14',
                                         always_return_array=False)
                trans[hs] = None if T is None else T[0]
            ncam = len(dwave) if per_camera else 1
            prior = (None if psig is None else
                     O.prior_on_coeffs(1 if nn is None else nn, nleg, psig, ncam))
            c2, co, ft = O.get_best_archetype(arch, sp, [s.band for s in t.spectra],
                                              O.legendre_dict(dwave, nleg), w, f, wf, dwave, z,
                                              per_camera, nn, trans, method, prior)
            assert ft == str(g[f"arch_{name}_{j}_fulltype"]), (name, j)
            np.testing.assert_allclose(c2, g[f"arch_{name}_{j}_chi2"], rtol=1e-10)
            gc = g[f"arch_{name}_{j}_coeff"]
            np.testing.assert_allclose(co, gc, rtol=0, atol=1e-8 * max(1.0, np.abs(gc).max()))


@pytest.mark.parametrize("nsig", [4.0, 2.5])
def test_coadd_cosmics_oracle_vs_redrock_golden(nsig):
    """Cosmic-ray rejection in the oracle's coadd matches redrock's
    Target(coadd=True, cosmics_nsig=nsig) bit for bit, and it masks pixels
    (the coadds differ from the ones without rejection)."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "coadd_golden.npz"))
    ct = synth.multi_exposure_targets(4, seed=62, cosmics=4)
    assert synth.targets_checksum(ct) == str(g["cosmic_targets_sha"])
    changed = 0
    for it, t in enumerate(ct):
        exps = [(s.band, s.wave, s.flux, O.masked_ivar(s.ivar, s.rdata, s.roffsets), s.rdata,
                 s.roffsets) for s in t.spectra]
        out = O.compute_coadd(exps, cosmics_nsig=nsig)
        plain = O.compute_coadd(exps)
        key = f"cosmic{nsig:g}_{it}"
        assert len(out) == int(g[f"{key}_nspec"][1])
        for j, ((band, wave, f, w, rd, ro), p) in enumerate(zip(out, plain)):
            assert synth.checksum([f, w, rd]) == str(g[f"{key}_{j}_sha"]), (it, j)
            changed += int(not np.array_equal(w, p[3]))
    assert changed > 0
