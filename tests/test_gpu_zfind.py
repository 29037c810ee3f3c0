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
    # rows are ranked by chi2, which the two refinements give slightly
    # differently: match each good Newton minimum to the parabola minima of
    # the same target and spectral type
    steps = {"GALAXY": 23 * 3e-4, "QSO": 31 * 5e-4, "STAR": 4 * 4e-5}
    good = np.nonzero(new["zwarn"] == 0)[0]
    assert len(good) >= 5
    for r in good:
        same = (par["targetid"] == new["targetid"][r]) & (par["spectype"] == new["spectype"][r])
        dlnz = np.abs(np.log1p(par["z"][same]) - np.log1p(new["z"][r]))
        # a fine-grid step: the 15-point grid spans two coarse steps
        assert dlnz.min() <= steps[new["spectype"][r]] * 2 / 14 + 1e-12
        assert new["zerr"][r] > 0
    # each good GALAXY Newton minimum: never above the best fine-grid point
    # of the cell it searched (the three points around the best one), and a
    # true minimum of fitz's objective -- a dense FP64 scan (201 points) of
    # a neighbourhood 1 % of the cell wide finds nothing lower.  (On these
    # 23x-subsampled grids a cell can hold several local minima; on the full
    # grids bench.py --zfind finds Newton at the cell's lowest point for every
    # target.)
    from redrock_b200.engine import RowPack, TemplateSource, run_pairs
    gal = [t for t in dts if t.template.full_type == "GALAXY"][0]
    local = list(dz.local())
    rows = RowPack.from_targets(local, gal.basis.layout)
    src = TemplateSource.from_template(gal.template)
    idx = {t.id: i for i, t in enumerate(local)}
    m = np.nonzero((new["zwarn"] == 0) & (new["spectype"] == "GALAXY"))[0]
    assert len(m) >= 2
    k = np.clip(np.argmin(new["zzchi2"][m], axis=1), 1, new["zz"].shape[1] - 2)
    lo = new["zz"][m, k - 1]
    hi = new["zz"][m, k + 1]
    zn = new["z"][m]
    assert np.all((lo <= zn) & (zn <= hi))
    cell = np.stack([new["zzchi2"][m, k - 1], new["zzchi2"][m, k], new["zzchi2"][m, k + 1]])
    assert np.all(new["chi2"][m] <= cell.min(axis=0) + 1e-9 * np.abs(cell.min(axis=0)))
    half = 0.005 * (hi - lo)
    zd = np.linspace(zn - half, zn + half, 201, axis=1)
    pt = np.repeat([idx[t] for t in new["targetid"][m]], 201).astype(np.int32)
    c2, _, pen = run_pairs(rows, src, pt, zd.ravel())
    c2 = (c2 + pen).cpu().numpy().reshape(len(m), 201)
    assert np.all(c2.min(axis=1) >= new["chi2"][m] - 1e-4), new["chi2"][m] - c2.min(axis=1)


def test_fitz_candidates_kernel_vs_find_minima():
    """rr_fitz_candidates against find_minima + np.linspace on rows with
    plateaus, edge minima, exact ties and a constant (all-masked) row:
    identical candidates and grids where the order is determined, the tie
    flag where numpy's unstable sort decides it."""
    import torch
    from redrock_b200.engine import FitzCandidates
    from redrock_b200.fitz import find_minima
    rng = np.random.default_rng(3)
    nz, K, nfine = 200, 5, 15
    z = np.sort(rng.uniform(0.0, 2.0, nz))
    rows = [rng.uniform(0, 100, nz) for _ in range(20)]
    r = rng.uniform(0, 100, nz)
    r[0] = -1.0                      # edge minimum
    rows.append(r)
    r = np.round(rng.uniform(0, 5, nz))   # many exact ties
    rows.append(r)
    rows.append(np.full(nz, 9999999.0))   # HUGE_CHI2 row
    r = np.linspace(10, 0, nz)       # monotone: only the last index
    rows.append(r)
    zc = np.stack(rows)
    pen = np.where(rng.uniform(size=zc.shape) < 0.1, rng.uniform(0, 3, zc.shape), 0.0)
    pen[-1] = 0.0
    fc = FitzCandidates(torch.tensor(zc, device="cuda"), torch.tensor(pen, device="cuda"),
                        torch.tensor(z, device="cuda"), K, nfine)
    torch.cuda.synchronize()
    cand, count, tie = fc.cand.cpu().numpy(), fc.count.cpu().numpy(), fc.tie.cpu().numpy()
    pz = fc.pair_z.cpu().numpy().reshape(len(rows), K, nfine)
    for j in range(len(rows)):
        eff = zc[j] + pen[j]
        ref = find_minima(eff)
        assert count[j] == min(K, len(ref))
        vals = eff[ref[:count[j] + 1]]
        determined = len(np.unique(vals)) == len(vals)
        if not determined:
            assert tie[j] == 1
            continue
        assert tie[j] == 0
        np.testing.assert_array_equal(cand[j, :count[j]], ref[:count[j]])
        for k, im in enumerate(ref[:count[j]]):
            lo, hi = z[max(0, im - 1)], z[min(im + 1, nz - 1)]
            np.testing.assert_array_equal(pz[j, k], np.linspace(lo, hi, nfine))
    assert tie[len(rows) - 2] == 1 and count[-1] == 1


def test_zfind_graph_equals_eager():
    """zfind(graph=True) -- scan, candidates and fine-grid scans of the whole
    batch captured as one CUDA graph -- gives the eager zfind's table bit
    for bit, with masked, dropped-camera and all-masked targets in two
    target blocks."""
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.zfind import zfind
    tg = synth.make_targets(40, seed=47, amp=1.5, mask_range=(0.0, 0.4), drop_camera_frac=0.15,
                            first_id=9000)
    for s in tg[7].spectra:
        s.ivar[:] = 0.0
    dz = T.DistTargetsCopy(T.from_synth(tg))
    sel = {"GALAXY": 11, "QSO": 13, "STAR:::K": 2, "STAR:::A": 2}
    dts = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            ts.redshifts = ts.redshifts[::sel[ts.full_type]]
            dts.append(TM.DistTemplate(TM.from_synth(ts), dz.wavegrids()))
    res_e, eager = zfind(dz, dts, nminima=3)
    res_g, graph = zfind(dz, dts, nminima=3, graph=True)
    assert list(graph.keys()) == list(eager.keys())
    for k in eager:
        np.testing.assert_array_equal(graph[k], eager[k], err_msg=k)
    for tid in res_e:
        for ft in res_e[tid]:
            np.testing.assert_array_equal(res_g[tid][ft]["zchi2"], res_e[tid][ft]["zchi2"])
    # a repeated call on the same objects replays the cached plan's graph
    from redrock_b200 import zscan
    plan = next(iter(zscan._plan_cache.d.values()))[1]
    _, graph2 = zfind(dz, dts, nminima=3, graph=True)
    assert next(iter(zscan._plan_cache.d.values()))[1] is plan
    for k in eager:
        np.testing.assert_array_equal(graph2[k], eager[k], err_msg=k)
    # after an in-place change of a target and clear_caches(), both paths
    # see the new contents (and agree again)
    t0 = dz.local()[0]
    for s in t0.spectra:
        s.flux[:] = s.flux * 1.5
    zscan.clear_caches()
    _, eager3 = zfind(dz, dts, nminima=3)
    _, graph3 = zfind(dz, dts, nminima=3, graph=True)
    assert not np.array_equal(eager3["chi2"], eager["chi2"])
    for k in eager3:
        np.testing.assert_array_equal(graph3[k], eager3[k], err_msg=k)
