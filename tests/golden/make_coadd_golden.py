"""Golden vectors for Target.compute_coadd, made by running redrock itself.

Inputs: redrock_b200.synth.multi_exposure_targets(4, seed=61) (1-3
exposures per camera, per-exposure resolution, noise and masks, pixels
masked in every exposure).  Each becomes a redrock ``Target(..., coadd=True)``
and the coadded spectra's flux, ivar and resolution data are recorded as
SHA-256 checksums (plus their sums, for diagnosis).  The cosmic-ray cases
coadd synth.multi_exposure_targets(4, seed=62, cosmics=4) (four hits per
exposure) with cosmics_nsig = 4 and 2.5.

    REDROCK_PY=<dir> python tests/golden/make_coadd_golden.py
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

SEED, NTARGET = 61, 4
COSMIC_SEED, COSMIC_NSIG = 62, (4.0, 2.5)


def main():
    redrock = import_redrock()
    RS, RT = redrock.targets.Spectrum, redrock.targets.Target
    tg = synth.multi_exposure_targets(NTARGET, seed=SEED)
    out = {"coadd_targets_sha": synth.targets_checksum(tg)}
    for it, t in enumerate(tg):
        specs = []
        for s in t.spectra:
            n = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata.copy(), s.roffsets.copy()), shape=(n, n))
            specs.append(RS(s.wave, s.flux.copy(), s.ivar.copy(), R, band=s.band))
        rt = RT(t.targetid, specs, coadd=True)
        out[f"coadd_{it}_bands"] = np.array(rt.bands)
        out[f"coadd_{it}_nspec"] = np.array([len(t.spectra), len(rt.spectra)])
        for j, sp in enumerate(rt.spectra):
            out[f"coadd_{it}_{j}_band"] = np.array(sp.band)
            out[f"coadd_{it}_{j}_sha"] = synth.checksum([sp.flux, sp.ivar, sp.R.data])
            out[f"coadd_{it}_{j}_sums"] = np.array([sp.flux.sum(), sp.ivar.sum(), sp.R.data.sum()])
    ct = synth.multi_exposure_targets(NTARGET, seed=COSMIC_SEED, cosmics=4)
    out["cosmic_targets_sha"] = synth.targets_checksum(ct)
    for nsig in COSMIC_NSIG:
        for it, t in enumerate(ct):
            specs = []
            for s in t.spectra:
                n = len(s.wave)
                R = scipy.sparse.dia_matrix((s.rdata.copy(), s.roffsets.copy()), shape=(n, n))
                specs.append(RS(s.wave, s.flux.copy(), s.ivar.copy(), R, band=s.band))
            rt = RT(t.targetid, specs, coadd=True, cosmics_nsig=nsig)
            key = f"cosmic{nsig:g}_{it}"
            out[f"{key}_nspec"] = np.array([len(t.spectra), len(rt.spectra)])
            for j, sp in enumerate(rt.spectra):
                out[f"{key}_{j}_sha"] = synth.checksum([sp.flux, sp.ivar, sp.R.data])
                out[f"{key}_{j}_sums"] = np.array([sp.flux.sum(), sp.ivar.sum(),
                                                    sp.R.data.sum()])
    np.savez(os.path.join(HERE, "coadd_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
