"""Generate the golden fixtures in this directory by running redrock itself.

Run with REDROCK_PY set to the directory that holds redrock's ``redrock``
package (a source checkout's ``py/`` directory, or an install target);
astropy and fitsio are stubbed because redrock only uses them for file I/O
(tests/redrock_ref.py).  The fixtures hold redrock's outputs (and checksums
of the generated inputs) for seeded synthetic inputs from
redrock_b200.synth, so the tests can regenerate the inputs without redrock.

    REDROCK_PY=<dir> python tests/golden/make_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from redrock_b200 import synth  # noqa: E402
from tests.redrock_ref import import_redrock, install_table_stubs  # noqa: E402,F401

rr = import_redrock()
install_table_stubs()
import redrock.zfind  # noqa: E402
import scipy.sparse  # noqa: E402


def ref_targets(specs):
    out = []
    for t in specs:
        spectra = []
        for s in t.spectra:
            npix = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(npix, npix))
            spectra.append(rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R,
                                               band=s.band))
        out.append(rr.targets.Target(t.targetid, spectra))
    return out


def ref_template(ts):
    return rr.templates.Template(spectype=ts.spectype, subtype=ts.subtype,
                                 redshifts=ts.redshifts, wave=ts.wave, flux=ts.flux,
                                 method=ts.method, igm_model=ts.igm_model)


def sample(a, step=13):
    return np.ascontiguousarray(a[:, ::step])


def main():
    out = {}
    # --- rebin: redrock's own known answers -------------------------------
    x = np.arange(10.)
    y = np.ones((2, 10))
    y[1] = np.arange(10)
    out["rebin_doc"] = rr.rebin.trapz_rebin(x, y, edges=[0, 2, 4, 6, 8], myz=[0.0, 0.5])
    xu = np.linspace(0, 10, 100) ** 2
    out["rebin_uneven"] = rr.rebin.trapz_rebin(xu, np.sqrt(xu), edges=np.linspace(0, 100, 21))
    xs = np.linspace(0, 2 * np.pi, 100)
    out["rebin_sin"] = rr.rebin.trapz_rebin(xs, np.sin(xs), edges=[0, 0.5 * np.pi, np.pi,
                                                                    1.5 * np.pi, 2 * np.pi])
    # --- rebin + IGM bases on the DESI-like grids --------------------------
    grids = synth.camera_grids()
    tmpls = synth.template_set()
    zsel = {"GALAXY": np.array([0, 1, 700, 1650, 2900, 3310]),
            "QSO": np.array([0, 5, 1200, 2201, 2600, 3100, 3793]),
            "STAR:::G": np.array([0, 37, 99])}
    for ts in tmpls:
        if ts.full_type not in zsel:
            continue
        key = ts.full_type.replace(":::", "_")
        zz = ts.redshifts[zsel[ts.full_type]]
        out[f"basis_{key}_z"] = zz
        tmpl = ref_template(ts)
        tmpl._redshifts = zz
        dt = rr.templates.DistTemplate(tmpl, grids)
        for cam in grids:
            d = dt.local.data[cam]
            out[f"basis_{key}_{cam}_sha"] = np.array(synth.checksum([d]))
            out[f"basis_{key}_{cam}_sample"] = sample(d)
        # rebin alone (no IGM) for one camera: bit-exactness of the rebin
        r = rr.rebin.trapz_rebin(ts.wave, ts.flux, xnew=grids["b"], myz=zz)
        out[f"rebin_{key}_b_sha"] = np.array(synth.checksum([r]))
        out[f"rebin_{key}_b_sample"] = sample(r)
    # --- IGM ---------------------------------------------------------------
    zigm = np.linspace(1.5, 6.6, 24)
    lob = np.ascontiguousarray(grids["b"][::7])
    out["igm_z"] = zigm
    out["igm_lobs"] = lob
    for model in ("Inoue14", "Calura12", "Kamble20"):
        out[f"igm_{model}"] = rr.igm.transmission_Lyman(zigm, lob, model=model)
    out["igm_Inoue14_scalar_z"] = rr.igm.transmission_Lyman(4.2, lob, model="Inoue14")
    out["igm_Inoue14_scalar_l"] = rr.igm.transmission_Lyman(zigm, 3650.0, model="Inoue14")
    # z >= 4.7 branches at wavelengths below the Lyman limit
    lob2 = np.linspace(3000.0, 9000.0, 301)
    zhi = np.array([4.69, 4.7, 5.2, 6.0, 7.5, 9.0])
    out["igm_hi_z"] = zhi
    out["igm_hi_lobs"] = lob2
    out["igm_hi_Inoue14"] = rr.igm.transmission_Lyman(zhi, lob2, model="Inoue14")
    # --- scan: calc_zchi2 ---------------------------------------------------
    tg = synth.make_targets(4, seed=11, amp=1.0)
    tg += synth.make_targets(1, seed=12, mask_range=(0.4, 0.4), first_id=2000)
    tg += synth.make_targets(1, seed=13, drop_camera_frac=1.0, first_id=3000)
    tg += synth.make_targets(1, seed=14, first_id=4000)
    for s in tg[-1].spectra:
        s.ivar[:] = 0.0  # all-masked target -> HUGE_CHI2 row
    out["scan_targets_sha"] = np.array(synth.targets_checksum(tg))
    rtg = ref_targets(tg)
    dtg = rr.targets.DistTargetsCopy(rtg)
    dwave = dtg.wavegrids()
    scan_sel = {"GALAXY": np.arange(0, 3311, 69), "QSO": np.arange(0, 3794, 79),
                "STAR:::G": np.arange(0, 100, 5)}
    for ts in tmpls:
        if ts.full_type not in scan_sel:
            continue
        key = ts.full_type.replace(":::", "_")
        tmpl = ref_template(ts)
        tmpl._redshifts = ts.redshifts[scan_sel[ts.full_type]]
        dt = rr.templates.DistTemplate(tmpl, dwave)
        zc, co, pe = rr.zscan.calc_zchi2([t.id for t in rtg], rtg, dt)
        out[f"scan_{key}_z"] = tmpl.redshifts
        out[f"scan_{key}_zchi2"] = zc
        out[f"scan_{key}_zcoeff"] = co
        out[f"scan_{key}_penalty"] = pe
        # fitz on the coarse results (zfind.py:356-363 passes zchi2 + penalty)
        for j, tg_ in enumerate(rtg):
            zf = rr.fitz.fitz(zc[j] + pe[j], tmpl.redshifts, tg_, tmpl, nminima=3)
            for k in ("z", "zerr", "zwarn", "chi2", "coeff", "npixels"):
                out[f"fitz_{key}_{j}_{k}"] = np.asarray(zf[k])
    # --- scan: redrock's test-utility fixture (2 exposures per camera) -------
    ut = [synth.util_target(0.2, seed=21, targetid=111), synth.util_target(0.25, seed=22,
                                                                            targetid=222)]
    out["util_targets_sha"] = np.array(synth.targets_checksum(ut))
    rut = []
    for t in ut:
        spectra = []
        for s in t.spectra:
            npix = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(npix, npix))
            spectra.append(rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R,
                                               R.tocsr()))
        rut.append(rr.targets.Target(t.targetid, spectra))
    dut = rr.targets.DistTargetsCopy(rut)
    uw, uf = synth.util_template()
    utm = rr.templates.Template(spectype="GALAXY", redshifts=np.linspace(0.15, 0.3, 50), wave=uw,
                                flux=uf, subtype="")
    udt = rr.templates.DistTemplate(utm, dut.wavegrids())
    res = rr.zscan.calc_zchi2_targets(dut, [udt], mp_procs=1)
    for t in rut:
        r = res[t.id][utm.full_type]
        out[f"util_{t.id}_zchi2"] = r["zchi2"]
        out[f"util_{t.id}_zcoeff"] = r["zcoeff"]
        out[f"util_{t.id}_penalty"] = r["penalty"]
    # --- calc_zchi2_batch with a prior, calc_zchi2_one, singular ------------
    gal = tmpls[0]
    tmpl = ref_template(gal)
    zb = gal.redshifts[[10, 400, 1500]]
    tmpl._redshifts = zb
    dt = rr.templates.DistTemplate(tmpl, dwave)
    t0 = rtg[0]
    w, f, wf = rr.zscan.spectral_data(t0.spectra)
    prior = np.diag(np.linspace(0.5, 5.0, gal.flux.shape[0]))
    zc, co = rr.zscan.calc_zchi2_batch(t0.spectra, dt.local.data, w, f, wf, len(zb),
                                       gal.flux.shape[0], "PCA", prior=prior)
    out["prior_z"] = zb
    out["prior_matrix"] = prior
    out["prior_zchi2"] = zc
    out["prior_zcoeff"] = co
    one = [rr.zscan.calc_zchi2_one(t0.spectra, w, f, wf,
                                   {k: v[i] for k, v in dt.local.data.items()}, "PCA")
           for i in range(len(zb))]
    out["one_zchi2"] = np.array([o[0] for o in one])
    out["one_zcoeff"] = np.array([o[1] for o in one])
    sflux = gal.flux.copy()
    sflux[3] = 0.0
    stm = rr.templates.Template(spectype="GALAXY", redshifts=zb, wave=gal.wave, flux=sflux,
                                subtype="")
    sdt = rr.templates.DistTemplate(stm, dwave)
    zc, co, pe = rr.zscan.calc_zchi2([t0.id], [t0], sdt)
    out["singular_zchi2"] = zc
    out["singular_zcoeff"] = co
    out["singular_penalty"] = pe
    # --- zfind end to end (coarse scan, fitz, finalisation) ------------------
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    out["zfind_targets_sha"] = np.array(synth.targets_checksum(ztg))
    rz = ref_targets(ztg)
    dz = rr.targets.DistTargetsCopy(rz)
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    zt = []
    for ts in tmpls:
        if ts.full_type in sel:
            tm = ref_template(ts)
            tm._redshifts = ts.redshifts[::sel[ts.full_type]]
            zt.append(rr.templates.DistTemplate(tm, dz.wavegrids()))
    _, zfit = rr.zfind.zfind(dz, zt, mp_procs=1, nminima=3)
    for k in ("targetid", "z", "zerr", "zwarn", "chi2", "deltachi2", "spectype", "subtype",
              "ncoeff", "znum", "npixels", "coeff"):
        out[f"zfind_{k}"] = np.asarray(zfit[k])
    out["zfind_columns"] = np.array(list(zfit.keys()))
    path = os.path.join(HERE, "redrock_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
