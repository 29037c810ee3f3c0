"""Golden vectors for redshift priors in zfind, made by running redrock
itself (priors.py, zfind.py:318-322) on the zfind fixture of
redrock_golden.npz (synth.make_targets(5, seed=41, amp=2.0, first_id=5000),
GALAXY / QSO / STAR K, M on subsampled grids) with the priors of
tests/prior_cases.py: Gaussian and top-hat, the last target without a
prior.  redrock's Priors reads a FITS file; the object is built directly
and handed to zfind in place of the file.

    REDROCK_PY=<dir> python tests/golden/make_prior_golden.py
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
# importing make_golden imports redrock with its file-I/O modules stubbed
from make_golden import ROOT, ref_targets, ref_template, rr  # noqa: E402

sys.path.insert(0, ROOT)
from redrock_b200 import synth  # noqa: E402
from tests.prior_cases import PRIOR_CASES, prior_arrays, zfind_inputs  # noqa: E402


def main():
    import redrock.priors as rp
    ztg, sel = zfind_inputs()
    out = {}
    for name in PRIOR_CASES:
        tid, z0, sig, func = prior_arrays(name, ztg)
        pri = object.__new__(rp.Priors)
        pri._param = {tid[i]: {'Z': z0[i], 'SIGMA': sig[i]} for i in range(len(tid))}
        pri._type = func
        pri._func = getattr(pri, func)
        rr.zfind.Priors = lambda filename, _p=pri: _p
        dz = rr.targets.DistTargetsCopy(ref_targets(ztg))
        zt = []
        for ts in synth.template_set():
            if ts.full_type in sel:
                tm = ref_template(ts)
                tm._redshifts = ts.redshifts[::sel[ts.full_type]]
                zt.append(rr.templates.DistTemplate(tm, dz.wavegrids()))
        _, zfit = rr.zfind.zfind(dz, zt, mp_procs=1, nminima=3, priors="in-memory")
        out[f"prior_{name}_columns"] = np.array(list(zfit.keys()))
        for k in zfit.keys():
            out[f"prior_{name}_{k}"] = np.asarray(zfit[k])
    np.savez(os.path.join(HERE, "prior_golden.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
