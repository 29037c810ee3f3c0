"""The drop-in on redrock's own objects: the unmodified redrock (its install
at baseline/_ref, or $REDROCK_PY) with redrock_b200.install() applied, fed
redrock's own Spectrum / Target / DistTargetsCopy / Template objects, and
redrock's own DistTemplate class and zfind driving the GPU functions, checked
against the outputs redrock produced on the same inputs without the GPU
(tests/golden/redrock_golden.npz).

Tolerances as in test_gpu_parity / test_gpu_zfind: |dchi2| <= 2e-5 on the
scan, identical argmin, |dc| <= 1e-5 max|c|; zfind columns identical where
discrete, |dz| <= 1e-7, |dchi2| <= 1e-3.
"""
import sys

import numpy as np
import pytest

from tests.conftest import cuda_available, redrock_dir

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU"),
              pytest.mark.skipif(redrock_dir() is None,
                                 reason="redrock not installed at baseline/_ref and "
                                        "REDROCK_PY unset")]

from redrock_b200 import synth  # noqa: E402
from tests.redrock_ref import ref_targets, ref_template  # noqa: E402

DCHI2_TIGHT = 2e-5
COEFF_REL = 1e-5


@pytest.fixture(scope="module")
def installed():
    """redrock imported fresh, its own DistTemplate and calc_zchi2_targets
    kept aside, then redrock_b200.install(redrock); redrock and its
    stand-ins are dropped from sys.modules afterwards."""
    before = set(sys.modules)
    path0 = list(sys.path)
    from tests.redrock_ref import import_redrock, install_table_stubs
    rr = import_redrock(redrock_dir())
    install_table_stubs()
    import redrock.zfind  # noqa: F401
    own = {"DistTemplate": rr.templates.DistTemplate,
           "calc_zchi2": rr.zscan.calc_zchi2}
    import redrock_b200
    done = redrock_b200.install(rr)
    # the package-level entry point keeps working after the first call
    assert callable(redrock_b200.install)
    yield rr, own, done
    for name in set(sys.modules) - before:
        if name.split(".")[0] in ("redrock", "astropy", "fitsio"):
            del sys.modules[name]
    sys.path[:] = path0


def scan_case():
    tg = synth.make_targets(4, seed=11, amp=1.0)
    tg += synth.make_targets(1, seed=12, mask_range=(0.4, 0.4), first_id=2000)
    tg += synth.make_targets(1, seed=13, drop_camera_frac=1.0, first_id=3000)
    tg += synth.make_targets(1, seed=14, first_id=4000)
    for s in tg[-1].spectra:
        s.ivar[:] = 0.0
    return tg


def test_install_rebinds_redrock(installed):
    rr, own, done = installed
    assert "zscan.calc_zchi2" in done and "templates.rebin_template" in done
    assert "fitz.calc_zchi2_batch" in done and "zfind.calc_zchi2_targets" in done
    assert rr.zscan.calc_zchi2 is not own["calc_zchi2"]
    assert rr.zscan.calc_zchi2.__module__ == "redrock_b200.zscan"
    assert rr.templates.transmission_Lyman.__module__ == "redrock_b200.igm"


@pytest.mark.parametrize("key", ["GALAXY", "QSO", "STAR_G"])
def test_calc_zchi2_on_redrock_objects(installed, golden, key):
    """redrock's own DistTemplate class (its rebin and IGM calls now reach the
    GPU through the rebound names) and redrock Targets, through the rebound
    calc_zchi2 -- the call redrock's calc_zchi2_targets makes per template."""
    rr, own, _ = installed
    tg = scan_case()
    assert synth.targets_checksum(tg) == str(golden["scan_targets_sha"])
    rtg = ref_targets(rr, tg)
    dtg = rr.targets.DistTargetsCopy(rtg)
    ts = {t.full_type.replace(":::", "_"): t for t in synth.template_set()}[key]
    tmpl = ref_template(rr, ts)
    tmpl._redshifts = golden[f"scan_{key}_z"]
    dt = own["DistTemplate"](tmpl, dtg.wavegrids())
    assert type(dt).__module__ == "redrock.templates"
    zc, co, pe = rr.zscan.calc_zchi2([t.id for t in rtg], rtg, dt)
    g = golden[f"scan_{key}_zchi2"]
    assert zc.shape == g.shape
    assert np.max(np.abs(zc - g)) <= DCHI2_TIGHT
    np.testing.assert_array_equal(np.argmin(zc, axis=1), np.argmin(g, axis=1))
    gc = golden[f"scan_{key}_zcoeff"]
    scale = np.maximum(np.abs(gc[:-1]).max(axis=-1, keepdims=True), 1e-300)
    assert np.all(np.abs(co[:-1] - gc[:-1]) <= COEFF_REL * scale)
    np.testing.assert_allclose(pe, golden[f"scan_{key}_penalty"], rtol=1e-8, atol=1e-8)
    # the installed DistTemplate name (the GPU-resident one) gives the same
    dt2 = rr.templates.DistTemplate(tmpl, dtg.wavegrids())
    res = rr.zscan.calc_zchi2_targets(dtg, [dt2])
    for i, t in enumerate(rtg):
        assert np.max(np.abs(res[t.id][tmpl.full_type]["zchi2"] - g[i])) <= DCHI2_TIGHT


def test_redrock_zfind_drives_the_gpu(installed, golden):
    """redrock's own zfind (coarse scan and fitz rebound, its own
    finalisation) on redrock Targets against redrock's CPU zfind."""
    rr, own, _ = installed
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    assert synth.targets_checksum(ztg) == str(golden["zfind_targets_sha"])
    dz = rr.targets.DistTargetsCopy(ref_targets(rr, ztg))
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    zt = []
    for ts in synth.template_set():
        if ts.full_type in sel:
            tm = ref_template(rr, ts)
            tm._redshifts = ts.redshifts[::sel[ts.full_type]]
            zt.append(rr.templates.DistTemplate(tm, dz.wavegrids()))
    _, zfit = rr.zfind.zfind(dz, zt, mp_procs=1, nminima=3)
    assert list(zfit.keys()) == list(golden["zfind_columns"])
    for k in ("targetid", "spectype", "subtype", "zwarn", "znum", "ncoeff", "npixels"):
        np.testing.assert_array_equal(np.asarray(zfit[k]), golden[f"zfind_{k}"], err_msg=k)
    np.testing.assert_allclose(np.asarray(zfit["z"]), golden["zfind_z"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(np.asarray(zfit["zerr"]), golden["zfind_zerr"], rtol=1e-5)
    assert np.max(np.abs(np.asarray(zfit["chi2"]) - golden["zfind_chi2"])) <= 1e-3
    assert np.max(np.abs(np.asarray(zfit["deltachi2"]) - golden["zfind_deltachi2"])) <= 1e-3
    g = golden["zfind_coeff"]
    scale = np.maximum(np.abs(g).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(np.asarray(zfit["coeff"]) - g) <= 1e-5 * scale)
