"""Bounded solves of solve_matrices on the GPU (rr_zchi2_batch_plain_ex:
NNLS / NMF and BVLS in redrock's scipy sense, min ||M c - y|| under bounds,
chi2 the direct residual) against redrock's own outputs
(tests/golden/make_lsq_golden.py).

Tolerances: |dchi2| <= 1e-3 (the acceptance bar) and 1e-6 relative,
coefficients 1e-5 of max|c| per z, identical active sets (coefficients at
zero for NNLS, at +-0.5 for the bounded BVLS case)."""

import os

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from oracle import oracle as O  # noqa: E402
from redrock_b200 import synth  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "lsq_golden.npz")


def _close(zc, co, gz, gc):
    zc, co = np.asarray(zc), np.asarray(co)
    assert np.max(np.abs(zc - gz)) <= 1e-3
    assert np.all(np.abs(zc - gz) <= 1e-6 * np.maximum(1.0, np.abs(gz)))
    scale = np.maximum(np.abs(gc).max(axis=-1, keepdims=True), 1e-300)
    assert np.all(np.abs(co - gc) <= 1e-5 * scale)


def test_nnls_bvls_batch_vs_redrock():
    from redrock_b200 import targets as T
    from redrock_b200 import zscan
    g = np.load(GOLDEN)
    tg = synth.make_targets(2, seed=11, amp=1.0)
    assert synth.targets_checksum(tg) == str(g["lsq_targets_sha"])
    gal = synth.template_set()[0]
    zb = g["lsq_z"]
    nb = gal.flux.shape[0]
    tdata = O.template_basis(gal.wave, gal.flux, zb, synth.camera_grids(), gal.igm_model)
    lo, hi = g["lsq_bounds"]
    for it, t in enumerate(T.from_synth(tg)):
        w, f, wf = zscan.spectral_data(t.spectra)
        for name, alg, args in (("nnls", "NNLS", None),
                                ("bvls", "BVLS", {"bounds": (np.full(nb, lo), np.full(nb, hi))}),
                                ("bvls_free", "BVLS", None)):
            zc, co = zscan.calc_zchi2_batch(t.spectra, tdata, w, f, wf, len(zb), nb, alg,
                                            solver_args=args)
            gz, gc = g[f"lsq_{name}_{it}_zchi2"], g[f"lsq_{name}_{it}_zcoeff"]
            _close(zc, co, gz, gc)
            if name == "nnls":
                np.testing.assert_array_equal(co == 0, gc == 0)
                assert np.all(co >= 0)
            if name == "bvls":
                np.testing.assert_array_equal(np.abs(np.abs(co) - hi) < 1e-9,
                                              np.abs(np.abs(gc) - hi) < 1e-9)
                assert np.all((co >= lo - 1e-12) & (co <= hi + 1e-12))


def test_nmf_template_scan_vs_redrock():
    """calc_zchi2 with an NMF template: each target through the plain chain
    with the NNLS solve (no [OII] penalty: redrock keeps that for PCA)."""
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    from redrock_b200 import zscan
    g = np.load(GOLDEN)
    tg = synth.make_targets(2, seed=11, amp=1.0)
    gal = synth.template_set()[0]
    zb = g["lsq_z"]
    dtg = T.DistTargetsCopy(T.from_synth(tg))
    tm = TM.Template(spectype="GALAXY", subtype="NMF", redshifts=zb, wave=gal.wave, flux=gal.flux,
                     method="NMF", igm_model=gal.igm_model)
    dt = TM.DistTemplate(tm, dtg.wavegrids())
    zc, co, pe = zscan.calc_zchi2([t.id for t in dtg.local()], dtg.local(), dt)
    _close(zc, co, g["lsq_nmf_zchi2"], g["lsq_nmf_zcoeff"])
    np.testing.assert_array_equal(pe, g["lsq_nmf_penalty"])
    # the all-templates entry point routes it the same way
    res = zscan.calc_zchi2_targets(dtg, [dt])
    for i, t in enumerate(dtg.local()):
        r = res[t.id][tm.full_type]
        _close(r["zchi2"][None], r["zcoeff"][None], g["lsq_nmf_zchi2"][i][None],
               g["lsq_nmf_zcoeff"][i][None])


def test_nmf_template_fitz_vs_redrock():
    """fitz on the NMF template's coarse scan: the fine grids and the fits at
    the parabola minima in batched pair launches with the kernel's NNLS (the
    template rebinned per pair, chi2 the direct residual), against redrock's
    fitz (rebin + IGM + calc_zchi2_batch per minimum).  z |dz| <= 1e-7, ZWARN identical, chi2 |d| <= 1e-3,
    coefficients |dc| <= 1e-5 max|c|."""
    from redrock_b200 import fitz, targets as T, templates as TM
    g = np.load(GOLDEN)
    tg = synth.make_targets(2, seed=11, amp=1.0)
    gal = synth.template_set()[0]
    zb = g["lsq_z"]
    tm = TM.Template(spectype="GALAXY", subtype="NMF", redshifts=zb, wave=gal.wave, flux=gal.flux,
                     method="NMF", igm_model=gal.igm_model)
    rt = T.from_synth(tg)
    chi2 = [g["lsq_nmf_zchi2"][j] + g["lsq_nmf_penalty"][j] for j in range(len(rt))]
    out = fitz.fitz_targets(chi2, zb, rt, tm, nminima=3)
    for j, r in enumerate(out):
        gz = {k: g[f"lsq_nmf_fitz_{j}_{k}"] for k in ("z", "zerr", "zwarn", "chi2", "coeff",
                                                      "npixels")}
        np.testing.assert_array_equal(r["zwarn"], gz["zwarn"])
        np.testing.assert_array_equal(r["npixels"], gz["npixels"])
        np.testing.assert_allclose(r["z"], gz["z"], rtol=0, atol=1e-7)
        np.testing.assert_allclose(r["zerr"], gz["zerr"], rtol=1e-5)
        assert np.max(np.abs(r["chi2"] - gz["chi2"])) <= 1e-3
        scale = np.maximum(np.abs(gz["coeff"]).max(axis=-1, keepdims=True), 1e-300)
        assert np.all(np.abs(r["coeff"] - gz["coeff"]) <= 1e-5 * scale)


def test_pair_scan_bounded_solves_vs_redrock():
    """rr_zscan_pairs with NNLS and BVLS (bounded and free): every (target,
    redshift) pair of the fixture in one launch per method, each pair's
    template rebinned inside the kernel, against redrock's calc_zchi2_batch
    at the same redshifts; same bars and active sets as the plain chain."""
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    from redrock_b200.adjoint import PairContext
    from redrock_b200.engine import TemplateSource, run_pairs
    g = np.load(GOLDEN)
    tg = synth.make_targets(2, seed=11, amp=1.0)
    gal = synth.template_set()[0]
    zb = g["lsq_z"]
    nb = gal.flux.shape[0]
    lo, hi = g["lsq_bounds"]
    rt = T.from_synth(tg)
    tm = TM.Template(spectype="GALAXY", subtype="NMF", redshifts=zb, wave=gal.wave, flux=gal.flux,
                     method="NMF", igm_model=gal.igm_model)
    ctx = PairContext(rt, tm)
    pt = np.repeat(np.arange(len(rt), dtype=np.int32), len(zb))
    pz = np.tile(zb, len(rt))
    for name, alg, bounds in (("nnls", "NNLS", None),
                              ("bvls", "BVLS", (np.full(nb, lo), np.full(nb, hi))),
                              ("bvls_free", "BVLS", None)):
        src = TemplateSource(gal.wave, gal.flux, zb, gal.igm_model, method=TM.solve_code_of(alg))
        c2, co, pe = run_pairs(ctx.rows, src, pt, pz, bounds=bounds)
        c2 = c2.cpu().numpy().reshape(len(rt), len(zb))
        co = co.cpu().numpy().reshape(len(rt), len(zb), nb)
        for it in range(len(rt)):
            gz, gc = g[f"lsq_{name}_{it}_zchi2"], g[f"lsq_{name}_{it}_zcoeff"]
            _close(c2[it], co[it], gz, gc)
            if name == "nnls":
                np.testing.assert_array_equal(co[it] == 0, gc == 0)
            if name == "bvls":
                np.testing.assert_array_equal(np.abs(np.abs(co[it]) - hi) < 1e-9,
                                              np.abs(np.abs(gc) - hi) < 1e-9)
        assert not np.any(pe.cpu().numpy())
