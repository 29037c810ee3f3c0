"""Inputs and cases of the archetype parity tests, shared with the script
that made their golden vectors (tests/golden/make_archetype_golden.py).

  * archetypes: synth.archetype_set(24, seed=5) (rest 800-10000 A at 0.5 A);
  * targets: synth.make_targets(3, seed=21) drawn from two of the
    archetypes at z in (0.1, 1.2), plus one at z in (2.2, 2.6), where the
    IGM transmission is active in the b camera.
"""
from redrock_b200 import synth

CASES = {  # name: (per_camera, nleg, n_nearest, prior_sigma, method)
    "pc": (True, 2, None, 0.1, "bvls"),
    "nc": (False, 2, None, None, "bvls"),
    "pcnn": (True, 2, 3, 0.1, "bvls"),
    "pcnn2": (True, 2, 2, 0.1, "bvls"),
    "pc0": (True, 0, None, 0.1, "bvls"),
    "pcpca": (True, 2, None, 0.1, "pca"),
}
FITZ_CASES = {  # name: (per_camera, n_nearest, prior_sigma)
    "pc": (True, None, 0.1),
    "nc": (False, None, 0.1),
}

ZFIND_CASES = {  # name: n_nearest (per camera, 2 Legendre terms, prior 0.1)
    "best": None,
    "nn2": 2,
}


def archetype_targets():
    arch = synth.archetype_set()
    tg = synth.make_targets(3, seed=21, template=(arch.wave, arch.flux[2:4]),
                            zrange=(0.1, 1.2), first_id=7000)
    tg += synth.make_targets(1, seed=22, template=(arch.wave, arch.flux[5:6]),
                             zrange=(2.2, 2.6), first_id=7100)
    return arch, tg


def fitz_targets():
    """The first three targets of the coarse-scan fixture."""
    return synth.make_targets(3, seed=11, amp=1.0)
