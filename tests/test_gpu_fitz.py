"""fitz refinement on the GPU (rr_zscan_pairs) against redrock's own fitz.

Input: redrock's coarse chi2 + penalty for the fixture targets (so the test
isolates the refinement).  Tolerances: redshift |dz| <= 1e-7, zerr relative
1e-5, chi2 |d| <= 1e-3, ZWARN bits and npixels identical, coefficients
|dc| <= 1e-5 max|c|.
"""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from redrock_b200 import synth  # noqa: E402


def scan_case():
    tg = synth.make_targets(4, seed=11, amp=1.0)
    tg += synth.make_targets(1, seed=12, mask_range=(0.4, 0.4), first_id=2000)
    tg += synth.make_targets(1, seed=13, drop_camera_frac=1.0, first_id=3000)
    tg += synth.make_targets(1, seed=14, first_id=4000)
    for s in tg[-1].spectra:
        s.ivar[:] = 0.0
    return tg


@pytest.mark.parametrize("key", ["GALAXY", "QSO", "STAR_G"])
def test_fitz_targets_vs_redrock(golden, key):
    from redrock_b200 import fitz, targets as T, templates as TM
    tg = scan_case()
    ts = {t.full_type.replace(":::", "_"): t for t in synth.template_set()}[key]
    ts.redshifts = golden[f"scan_{key}_z"]
    tm = TM.from_synth(ts)
    rtg = T.from_synth(tg)
    chi2 = [golden[f"scan_{key}_zchi2"][j] + golden[f"scan_{key}_penalty"][j]
            for j in range(len(tg))]
    out = fitz.fitz_targets(chi2, ts.redshifts, rtg, tm, nminima=3)
    for j, r in enumerate(out):
        g = {k: golden[f"fitz_{key}_{j}_{k}"] for k in ("z", "zerr", "zwarn", "chi2", "coeff",
                                                         "npixels")}
        assert r["z"].shape == g["z"].shape
        np.testing.assert_array_equal(r["zwarn"], g["zwarn"])
        np.testing.assert_array_equal(r["npixels"], g["npixels"])
        np.testing.assert_allclose(r["z"], g["z"], rtol=0, atol=1e-7)
        np.testing.assert_allclose(r["zerr"], g["zerr"], rtol=1e-5, atol=1e-12)
        assert np.max(np.abs(r["chi2"] - g["chi2"])) <= 1e-3
        scale = np.maximum(np.abs(g["coeff"]).max(axis=-1, keepdims=True), 1e-300)
        assert np.all(np.abs(r["coeff"] - g["coeff"]) <= 1e-5 * scale)


def test_fitz_single_target_signature(golden):
    from redrock_b200 import fitz, targets as T, templates as TM
    tg = scan_case()[:1]
    ts = synth.template_set()[0]
    ts.redshifts = golden["scan_GALAXY_z"]
    r = fitz.fitz(golden["scan_GALAXY_zchi2"][0] + golden["scan_GALAXY_penalty"][0],
                  ts.redshifts, T.from_synth(tg)[0], TM.from_synth(ts), nminima=3)
    np.testing.assert_allclose(r["z"], golden["fitz_GALAXY_0_z"], atol=1e-7)


def test_fitz_newton_refinement(golden):
    """refine="newton" replaces the parabola: the refined z stays within a
    fine-grid step of the parabola's, and its chi2 (a real evaluation, unlike
    the parabola's fitted minimum) is not above the best fine-grid point."""
    from redrock_b200 import fitz, targets as T, templates as TM
    tg = scan_case()[:4]
    ts = synth.template_set()[0]
    ts.redshifts = golden["scan_GALAXY_z"]
    chi2 = [golden["scan_GALAXY_zchi2"][j] + golden["scan_GALAXY_penalty"][j] for j in range(4)]
    rtg = T.from_synth(tg)
    par = fitz.fitz_targets(chi2, ts.redshifts, rtg, TM.from_synth(ts), nminima=3)
    new = fitz.fitz_targets(chi2, ts.redshifts, rtg, TM.from_synth(ts), nminima=3,
                            refine="newton")
    step = np.diff(ts.redshifts).max() * 2 / 14
    for a, b in zip(par, new):
        good = (a["zwarn"].ravel() == 0) & (b["zwarn"].ravel() == 0)
        assert good.sum() >= 1
        assert np.all(np.abs(a["z"].ravel() - b["z"].ravel())[good] <= step)
        best_grid = b["zzchi2"].min(axis=1)
        assert np.all((b["chi2"].ravel() <= best_grid + 1e-6)[good])
        assert np.all(b["zerr"].ravel()[good] > 0)
