"""zfind end to end (fused coarse scan -> batched GPU fitz -> finalisation)
against redrock's own zfind on the same inputs.

Tolerances: row order, targetid, spectype, subtype, ZWARN, znum, ncoeff and
npixels identical; redshift |dz| <= 1e-7; chi2 and delta-chi2 |d| <= 1e-3;
zerr relative 1e-5; coefficients |dc| <= 1e-5 max|c|.
"""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from redrock_b200 import synth  # noqa: E402


def test_zfind_vs_redrock(golden):
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.zfind import zfind
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    assert synth.targets_checksum(ztg) == str(golden["zfind_targets_sha"])
    dz = T.DistTargetsCopy(T.from_synth(ztg))
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    dts = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
    _, zfit = zfind(dz, dts, nminima=3)
    assert list(zfit.keys()) == list(golden["zfind_columns"])
    for k in ("targetid", "spectype", "subtype", "zwarn", "znum", "ncoeff", "npixels"):
        np.testing.assert_array_equal(zfit[k], golden[f"zfind_{k}"], err_msg=k)
    np.testing.assert_allclose(zfit["z"], golden["zfind_z"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(zfit["zerr"], golden["zfind_zerr"], rtol=1e-5)
    assert np.max(np.abs(zfit["chi2"] - golden["zfind_chi2"])) <= 1e-3
    assert np.max(np.abs(zfit["deltachi2"] - golden["zfind_deltachi2"])) <= 1e-3
    g = golden["zfind_coeff"]
    scale = np.maximum(np.abs(g).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(zfit["coeff"] - g) <= 1e-5 * scale)


@pytest.mark.parametrize("name", ["gaussian", "tophat"])
def test_zfind_with_priors_vs_redrock(name):
    """Redshift priors (Gaussian, top-hat; one target without a prior) added
    to the coarse chi2 before the refinement, as redrock's zfind does."""
    import os
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.priors import Priors
    from redrock_b200.zfind import zfind
    from tests.prior_cases import prior_arrays, zfind_inputs
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "prior_golden.npz"))
    ztg, sel = zfind_inputs()
    tid, z0, sig, func = prior_arrays(name, ztg)
    dz = T.DistTargetsCopy(T.from_synth(ztg))
    dts = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
    _, zfit = zfind(dz, dts, nminima=3, priors=Priors(targetid=tid, z=z0, sigma=sig,
                                                      function=func))
    cols = list(g[f"prior_{name}_columns"])
    assert list(zfit.keys()) == cols
    for k in ("targetid", "spectype", "subtype", "zwarn", "znum", "ncoeff", "npixels"):
        np.testing.assert_array_equal(zfit[k], g[f"prior_{name}_{k}"], err_msg=k)
    np.testing.assert_allclose(zfit["z"], g[f"prior_{name}_z"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(zfit["zerr"], g[f"prior_{name}_zerr"], rtol=1e-5)
    assert np.max(np.abs(zfit["chi2"] - g[f"prior_{name}_chi2"])) <= 1e-3
    d = zfit["deltachi2"] - g[f"prior_{name}_deltachi2"]
    assert np.max(np.abs(d[np.isfinite(d)])) <= 1e-3
    np.testing.assert_array_equal(np.isfinite(zfit["deltachi2"]),
                                  np.isfinite(g[f"prior_{name}_deltachi2"]))


def test_zfind_details_file_resume(golden, tmp_path):
    """zfind -> write_zscan -> zfind(chi2_scan=file): the resumed run reads
    the float32 coarse scans from the details file instead of scanning and
    finds the same best redshifts (redrock's --chi2-scan path)."""
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.results import read_zfit, write_zscan
    from redrock_b200.zfind import zfind
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}

    def inputs():
        dz = T.DistTargetsCopy(T.from_synth(ztg))
        dts = []
        for ts in synth.template_set():
            if ts.full_type in sel:
                ts.redshifts = ts.redshifts[::sel[ts.full_type]]
                dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
        return dz, dts

    res, zfit = zfind(*inputs(), nminima=3)
    fn = str(tmp_path / "rrdetails.h5")
    write_zscan(fn, res, zfit)
    back = read_zfit(fn)
    np.testing.assert_array_equal(back['targetid'], zfit['targetid'])
    # redrock's test_io.py:45-85 checks on the same round trip
    from redrock_b200.results import read_zscan
    zfit1 = {k: v for k, v in zfit.items() if k != 'fitmethod'}
    fn1 = str(tmp_path / "rrdetails1.h5")
    write_zscan(fn1, res, zfit1)
    write_zscan(fn1, res, zfit1, clobber=True)
    zscan2, zfit2 = read_zscan(fn1)
    assert list(zfit2.keys()) == list(zfit1.keys())
    assert zfit2['z'].dtype == zfit1['z'].dtype
    assert zfit2['targetid'].dtype == zfit1['targetid'].dtype
    for cn in zfit1:
        d2 = zfit2[cn]
        np.testing.assert_equal(np.asarray(zfit1[cn]).astype(d2.dtype), d2)
    for tid in res:
        for ft in res[tid]:
            for key in ('redshifts', 'zchi2', 'penalty', 'zcoeff'):
                d1 = np.asarray(res[tid][ft][key])
                if key != 'redshifts':
                    d1 = d1.astype(np.float32)
                np.testing.assert_equal(d1, zscan2[tid][ft][key])
    _, zfit2 = zfind(*inputs(), nminima=3, chi2_scan=fn)
    best = zfit['znum'] == 0
    best2 = zfit2['znum'] == 0
    np.testing.assert_array_equal(zfit2['targetid'][best2], zfit['targetid'][best])
    np.testing.assert_array_equal(zfit2['spectype'][best2], zfit['spectype'][best])
    np.testing.assert_allclose(zfit2['z'][best2], zfit['z'][best], rtol=0, atol=1e-6)


def test_zfind_newton_refinement(golden):
    """zfind(refine="newton"): every template's minima refined by batched
    Newton steps on chi2(z) (one pair-gradient launch per iteration for all
    candidates) instead of the parabola.  Same targets and row structure as
    the parabola path; each good redshift within a fine-grid step of the
    parabola's, with a chi2 (a real evaluation at that z) no higher than the
    best fine-grid point it started from."""
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.zfind import zfind
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    dz = T.DistTargetsCopy(T.from_synth(ztg))
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    dts = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
    _, par = zfind(dz, dts, nminima=3)
    _, new = zfind(dz, dts, nminima=3, refine="newton")
    assert list(new.keys()) == list(par.keys())
    np.testing.assert_array_equal(new["targetid"], par["targetid"])
    best = new["znum"] == 0
    np.testing.assert_array_equal(new["spectype"][best], par["spectype"][best])
    good = (new["zwarn"] == 0) & (par["zwarn"] == 0) & (new["spectype"] == par["spectype"])
    assert good.sum() >= 5
    for st, step in (("GALAXY", 23 * 3e-4), ("QSO", 31 * 5e-4), ("STAR", 4 * 4e-5)):
        m = good & (new["spectype"] == st)
        # a fine-grid step: the 15-point grid spans two coarse steps
        assert np.all(np.abs(np.log1p(new["z"][m]) - np.log1p(par["z"][m])) <= step * 2 / 14
                      + 1e-12)
    assert np.all(new["zerr"][good] > 0)
