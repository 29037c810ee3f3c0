"""Inputs of the redshift-prior parity test, shared with the script that
made its golden vectors (tests/golden/make_prior_golden.py)."""
import numpy as np

from redrock_b200 import synth

PRIOR_CASES = ("gaussian", "tophat")


def zfind_inputs():
    """The zfind fixture's targets and the template subsampling."""
    ztg = synth.make_targets(5, seed=41, amp=2.0, first_id=5000)
    sel = {"GALAXY": 23, "QSO": 31, "STAR:::K": 4, "STAR:::M": 4}
    return ztg, sel


def prior_arrays(name, targets):
    """(targetid, z0, sigma, function): a prior for all but the last
    target, centred 0.02 above its true redshift; sigma 0.05 (Gaussian) or
    width 0.3 (top-hat)."""
    tid = np.array([t.targetid for t in targets[:-1]])
    z0 = np.array([t.ztrue + 0.02 for t in targets[:-1]])
    sig = np.full(len(tid), 0.05 if name == "gaussian" else 0.3)
    return tid, z0, sig, name
