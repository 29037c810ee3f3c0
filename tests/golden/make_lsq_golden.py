"""Golden vectors for the bounded solves of redrock's solve_matrices
(zscan.py:1153-1201), made by running redrock itself: calc_zchi2_batch with
"NNLS", "BVLS" (active bounds) and "BVLS" (no bounds) for two synthetic
targets on every 150th GALAXY redshift, calc_zchi2 with an NMF GALAXY
template (chi2, coefficients, [OII] penalty), and fitz on that scan.

    REDROCK_PY=<dir> python tests/golden/make_lsq_golden.py
"""

import os
import sys

import numpy as np
import scipy.sparse

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import ROOT, import_redrock  # noqa: E402

sys.path.insert(0, ROOT)
from redrock_b200 import synth  # noqa: E402

SEED, NTARGET, ZSTEP = 11, 2, 150
BOUNDS = (-0.5, 0.5)


def main():
    rr = import_redrock()
    tg = synth.make_targets(NTARGET, seed=SEED, amp=1.0)
    rtg = []
    for t in tg:
        sp = []
        for s in t.spectra:
            n = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(n, n))
            sp.append(rr.targets.Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R, band=s.band))
        rtg.append(rr.targets.Target(t.targetid, sp))
    gal = synth.template_set()[0]
    zb = np.ascontiguousarray(gal.redshifts[::ZSTEP])
    dwave = {s.band: s.wave for s in rtg[0].spectra}
    tmpl = rr.templates.Template(spectype="GALAXY", subtype="", redshifts=zb, wave=gal.wave,
                                 flux=gal.flux, method="PCA", igm_model=gal.igm_model)
    dt = rr.templates.DistTemplate(tmpl, dwave)
    nb = gal.flux.shape[0]
    out = {"lsq_targets_sha": synth.targets_checksum(tg), "lsq_z": zb,
           "lsq_bounds": np.array(BOUNDS)}
    for it, t in enumerate(rtg):
        w, f, wf = rr.zscan.spectral_data(t.spectra)
        for name, alg, args in (("nnls", "NNLS", None),
                                ("bvls", "BVLS", {"bounds": (np.full(nb, BOUNDS[0]),
                                                             np.full(nb, BOUNDS[1]))}),
                                ("bvls_free", "BVLS", None)):
            zc, co = rr.zscan.calc_zchi2_batch(t.spectra, dt.local.data, w, f, wf, len(zb), nb,
                                               alg, solver_args=args)
            out[f"lsq_{name}_{it}_zchi2"] = zc
            out[f"lsq_{name}_{it}_zcoeff"] = co
    nmf = rr.templates.Template(spectype="GALAXY", subtype="NMF", redshifts=zb, wave=gal.wave,
                                flux=gal.flux, method="NMF", igm_model=gal.igm_model)
    ndt = rr.templates.DistTemplate(nmf, dwave)
    zc, co, pe = rr.zscan.calc_zchi2([t.id for t in rtg], rtg, ndt)
    out["lsq_nmf_zchi2"] = zc
    out["lsq_nmf_zcoeff"] = co
    out["lsq_nmf_penalty"] = pe
    # fitz on the NMF coarse scan (fitz.py:133-395 with the NNLS solver)
    for j, t in enumerate(rtg):
        zf = rr.fitz.fitz(zc[j] + pe[j], zb, t, nmf, nminima=3)
        for k in ("z", "zerr", "zwarn", "chi2", "coeff", "npixels"):
            out[f"lsq_nmf_fitz_{j}_{k}"] = np.asarray(zf[k])
    np.savez(os.path.join(HERE, "lsq_golden.npz"), **out)
    print("wrote", len(out), "arrays; NNLS zeros per target:",
          [int((out[f"lsq_nnls_{i}_zcoeff"] == 0).sum()) for i in range(NTARGET)],
          "BVLS at bounds:", [int((np.abs(np.abs(out[f"lsq_bvls_{i}_zcoeff"]) - 0.5) < 1e-9).sum())
                              for i in range(NTARGET)])


if __name__ == "__main__":
    main()
