"""Target.compute_coadd on the GPU (rr_coadd, rr_coadd_cosmics) against
redrock's own coadds: bit-identical flux, ivar and resolution data
(checksums recorded by tests/golden/make_coadd_golden.py from redrock's
Target(coadd=True), with and without cosmic-ray rejection)."""

import os

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from redrock_b200 import synth  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "coadd_golden.npz")


def _check(targets, g):
    for it, t in enumerate(targets):
        assert len(t.spectra) == int(g[f"coadd_{it}_nspec"][1])
        assert list(t.bands) == [str(b) for b in g[f"coadd_{it}_bands"]]
        for j, sp in enumerate(t.spectra):
            assert sp.band == str(g[f"coadd_{it}_{j}_band"])
            got = synth.checksum([sp.flux, sp.ivar, sp.R.data])
            assert got == str(g[f"coadd_{it}_{j}_sha"]), (it, j, [sp.flux.sum(), sp.ivar.sum(),
                                                                 sp.R.data.sum()],
                                                           g[f"coadd_{it}_{j}_sums"])


def test_coadd_batched_bit_identical_to_redrock():
    from redrock_b200 import targets as T
    from redrock_b200.coadd import coadd_targets
    g = np.load(GOLDEN)
    tg = synth.multi_exposure_targets(4, seed=61)
    assert synth.targets_checksum(tg) == str(g["coadd_targets_sha"])
    rt = T.from_synth(tg)
    coadd_targets(rt)          # all targets, one launch
    _check(rt, g)


def test_target_coadd_flag_and_method():
    from redrock_b200 import targets as T
    g = np.load(GOLDEN)
    tg = synth.multi_exposure_targets(4, seed=61)
    rt = T.from_synth(tg)
    # Target(..., coadd=True) coadds at construction, like redrock's
    built = [T.Target(t.id, t.spectra, coadd=True) for t in rt]
    _check(built, g)


@pytest.mark.parametrize("nsig", [4.0, 2.5])
def test_coadd_cosmics_bit_identical_to_redrock(nsig):
    from redrock_b200 import targets as T
    from redrock_b200.coadd import coadd_targets
    g = np.load(GOLDEN)
    ct = synth.multi_exposure_targets(4, seed=62, cosmics=4)
    assert synth.targets_checksum(ct) == str(g["cosmic_targets_sha"])
    rt = T.from_synth(ct)
    coadd_targets(rt, cosmics_nsig=nsig)
    for it, t in enumerate(rt):
        key = f"cosmic{nsig:g}_{it}"
        assert len(t.spectra) == int(g[f"{key}_nspec"][1])
        for j, sp in enumerate(t.spectra):
            got = synth.checksum([sp.flux, sp.ivar, sp.R.data])
            assert got == str(g[f"{key}_{j}_sha"]), (it, j, [sp.flux.sum(), sp.ivar.sum(),
                                                            sp.R.data.sum()],
                                                      g[f"{key}_{j}_sums"])


def test_coadd_cosmics_exposure_without_good_pixels_raises():
    """numpy's interp has no sample points there: redrock raises ValueError."""
    from redrock_b200 import targets as T
    ct = synth.multi_exposure_targets(1, seed=62, cosmics=1)
    rt = T.from_synth(ct)
    rt[0].spectra[0].ivar[:] = 0.0
    with pytest.raises(ValueError):
        rt[0].compute_coadd(cosmics_nsig=4.0)
