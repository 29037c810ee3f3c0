"""Golden vectors for the archetype fits, made by running redrock itself
(archetypes.py:228-400, zscan.py:245-348, fitz.py:113-395).

Inputs are regenerated by the tests (tests/archetype_cases.py).
Cases of Archetype.get_best_archetype per target (at its true z):
  pc    per camera, 2 Legendre terms, prior sigma 0.1          (BVLS)
  nc    one Legendre set for the spectrum, no prior            (BVLS)
  pcnn  per camera, 3 nearest archetypes, prior sigma 0.1
  pcnn2 per camera, 2 nearest archetypes, prior sigma 0.1
  pc0   per camera without Legendre terms
  pcpca per camera, solve method PCA
and fitz with archetypes (per camera, prior 0.1; one Legendre set for the
spectrum, prior 0.1) on the GALAXY coarse scan of redrock_golden.npz, and
zfind with GALAXY archetypes on the zfind fixture of redrock_golden.npz (per
camera, prior 0.1; with and without 2 nearest archetypes).
(Nearest archetypes with one Legendre set for the spectrum is not a case:
redrock calls calc_zchi2_batch without a solve method there
(archetypes.py:287) and solve_matrices fails on None.)

    REDROCK_PY=<dir> python tests/golden/make_archetype_golden.py
"""

import os
import sys

import numpy as np
import scipy.sparse

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
# importing make_golden imports redrock with its file-I/O modules stubbed
# (astropy.table.Table as a dict of columns, for zfind)
from make_golden import ROOT, ref_template, rr  # noqa: E402

sys.path.insert(0, ROOT)
from redrock_b200 import synth  # noqa: E402
from tests.archetype_cases import (CASES, FITZ_CASES, ZFIND_CASES, archetype_targets,  # noqa: E402
                                   fitz_targets)

def ref_archetype(rr, spec):
    import redrock.archetypes as ra
    a = object.__new__(ra.Archetype)
    a._filename = None
    a.flux = np.asarray(spec.flux, dtype=np.float64)
    a._narch, a._nwave = a.flux.shape
    a._rrtype = spec.rrtype
    a._subtype = np.char.add(np.char.add(np.array(spec.subtype), '_'),
                             np.arange(a._narch, dtype=int).astype(str))
    a._full_type = np.array([rr.templates.make_fulltype(a._rrtype, s) for s in a._subtype])
    a._version = spec.version
    a.wave = np.asarray(spec.wave)
    a.minwave = a.wave[0]
    a.maxwave = a.wave[-1]
    a._archetype = {}
    a._gpuwave = None
    a._gpuflux = None
    a.igm_model = 'Inoue14'
    a.method = 'ARCH'
    return a


def ref_targets(rr, specs):
    out = []
    for t in specs:
        sp = []
        for s in t.spectra:
            n = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(n, n))
            sp.append(rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R, band=s.band))
        out.append(rr.targets.Target(t.targetid, sp))
    return out


def main():
    import redrock.archetypes  # noqa: F401
    spec, tg = archetype_targets()
    arch = ref_archetype(rr, spec)
    out = {"arch_targets_sha": np.array(synth.targets_checksum(tg)),
           "arch_flux_sha": np.array(synth.checksum([spec.wave, spec.flux])),
           "arch_z": np.array([t.ztrue for t in tg])}
    for name, (per_camera, nleg, nn, psig, method) in CASES.items():
        rtg = ref_targets(rr, tg)
        for j, t in enumerate(rtg):
            z = tg[j].ztrue
            t.legendre(nleg)
            w, f, wf = rr.zscan.spectral_data(t.spectra)
            dwave = {s.wavehash: s.wave for s in t.spectra}
            trans = {hs: rr.igm.transmission_Lyman(np.array([z]), wv, always_return_array=False,
                                                   model='Inoue14')
                     for hs, wv in dwave.items()}
            ncam = len(dwave) if per_camera else 1
            prior = (None if psig is None else
                     rr.fitz.prior_on_coeffs(1 if nn is None else nn, nleg, psig, ncam))
            c2, co, ft = arch.get_best_archetype(t, w, f, wf, dwave, z, per_camera, nn,
                                                 trans=trans, solve_method=method, prior=prior)
            out[f"arch_{name}_{j}_chi2"] = np.array(c2)
            out[f"arch_{name}_{j}_coeff"] = np.asarray(co)
            out[f"arch_{name}_{j}_fulltype"] = np.array(ft)
    g = np.load(os.path.join(HERE, "redrock_golden.npz"))
    scan_tg = fitz_targets()
    gal = synth.template_set()[0]
    tmpl = ref_template(gal)
    tmpl._redshifts = g["scan_GALAXY_z"]
    for name, (per_camera, nn, psig) in FITZ_CASES.items():
        rtg = ref_targets(rr, scan_tg)
        for j, t in enumerate(rtg):
            chi2 = g["scan_GALAXY_zchi2"][j] + g["scan_GALAXY_penalty"][j]
            r = rr.fitz.fitz(chi2, tmpl.redshifts, t, tmpl, nminima=3, archetype=arch,
                             deg_legendre=2, per_camera=per_camera, n_nearest=nn,
                             prior_sigma=psig)
            for k in ("z", "zerr", "zwarn", "chi2", "coeff", "legcoeff", "fulltype",
                      "pca_coeff", "npixels"):
                out[f"afitz_{name}_{j}_{k}"] = np.asarray(r[k])
    # zfind end to end with archetypes for GALAXY (the zfind fixture's
    # targets and templates), per camera with prior 0.1, and with 2 nearest
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    for name, nn in ZFIND_CASES.items():
        dz = rr.targets.DistTargetsCopy(ref_targets(rr, ztg))
        zt = []
        for ts in synth.template_set():
            if ts.full_type in sel:
                tm = ref_template(ts)
                tm._redshifts = ts.redshifts[::sel[ts.full_type]]
                zt.append(rr.templates.DistTemplate(tm, dz.wavegrids()))
        _, zfit = rr.zfind.zfind(dz, zt, mp_procs=1, nminima=3, archetypes={"GALAXY": arch},
                                 per_camera=True, deg_legendre=2, n_nearest=nn,
                                 prior_sigma=0.1, ncamera=3)
        out[f"azfind_{name}_columns"] = np.array(list(zfit.keys()))
        for k in zfit.keys():
            out[f"azfind_{name}_{k}"] = np.asarray(zfit[k])
    np.savez(os.path.join(HERE, "archetype_golden.npz"), **out)
    print("wrote", len(out), "arrays;",
          {k: str(out[k]) for k in out if k.endswith("fulltype") and "_0_" in k})


if __name__ == "__main__":
    main()
