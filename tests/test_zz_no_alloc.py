"""rr_zchi2_batch_plain_noalloc: the plain per-target chain for callers that
cannot allocate device memory themselves (their own memory manager owns the
GPU's memory, or a cudaMalloc / cudaFree would synchronise a latency-bound
loop).  It runs in the library's fixed 16 MiB scratch array instead of a
caller workspace.

Checked through the C ABI against rr_zchi2_batch_plain (which is given a
workspace) on two calls in a row, with different redshift sets so the
second call runs over the first call's leftover scratch contents.
Tolerances as in test_gpu_parity: |dchi2| <= 2e-5, |dc| <= 1e-5 max|c|.

This file is collected last so a stop-at-first-failure run has already run
every other test; it needs nothing from them.
"""

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

DCHI2_TIGHT = 2e-5
COEFF_REL = 1e-5


def _setup(zsel):
    import torch
    from redrock_b200 import synth
    from redrock_b200 import targets as T
    from redrock_b200.engine import DeviceBasis, GridLayout, PlainTarget, TemplateSource
    tg = T.from_synth(synth.make_targets(1, seed=31, mask_range=(0.1, 0.1)))[0]
    gal = synth.template_set()[0]
    layout = GridLayout.from_dwave(synth.camera_grids())
    src = TemplateSource(gal.wave, gal.flux, gal.redshifts[zsel], gal.igm_model)
    basis = DeviceBasis.build(src, layout)
    pt = PlainTarget(tg.spectra, layout)
    torch.cuda.synchronize()
    return pt, basis


def _call(fn_name, pt, basis, workspace=None):
    import torch
    from redrock_b200 import _lib
    from redrock_b200.device import stream_handle
    L = _lib.lib()
    nz, nb = basis.nz, basis.nbasis
    zchi2 = torch.full((nz,), -1.0, dtype=torch.float64, device="cuda")
    zcoeff = torch.full((nz, nb), -1.0, dtype=torch.float64, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    args = [pt.band.data_ptr(), pt.w.data_ptr(), pt.wflux.data_ptr(), pt.flux.data_ptr(),
            pt.pix_basis.data_ptr(), pt.npix, basis.basis.data_ptr(), basis.layout.pix_stride,
            nz, nb, basis.stride, None, _lib.RR_SOLVE_PCA, zchi2.data_ptr(), zcoeff.data_ptr()]
    if workspace is not None:
        args += [workspace.data_ptr(), workspace.numel()]
    args += [status.data_ptr(), stream_handle()]
    rc = getattr(L, fn_name)(*args)
    assert rc == _lib.RR_OK, _lib.status_string(rc)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return zchi2.cpu().numpy(), zcoeff.cpu().numpy()


def test_noalloc_matches_workspace_path_twice():
    import torch
    from redrock_b200 import _lib
    L = _lib.lib()
    for zsel in (slice(0, 3311, 221), slice(100, 3311, 331)):
        pt, basis = _setup(zsel)
        need = L.rr_zchi2_batch_plain_workspace_bytes(pt.npix, basis.nz, basis.nbasis)
        ws = torch.empty(need, dtype=torch.uint8, device="cuda")
        ref_chi2, ref_coeff = _call("rr_zchi2_batch_plain", pt, basis, ws)
        got_chi2, got_coeff = _call("rr_zchi2_batch_plain_noalloc", pt, basis)
        assert np.all(np.isfinite(got_chi2)) and np.all(got_chi2 > 0)
        assert np.max(np.abs(got_chi2 - ref_chi2)) <= DCHI2_TIGHT
        scale = np.abs(ref_coeff).max(axis=1, keepdims=True)
        assert np.all(np.abs(got_coeff - ref_coeff) <= COEFF_REL * scale)


def test_noalloc_rejects_oversized_request():
    from redrock_b200 import _lib
    L = _lib.lib()
    cap = 16 << 20
    # 3311 redshifts x 7958 pixels x 10 bases needs ~2 GB of scratch
    assert L.rr_zchi2_batch_plain_workspace_bytes(7958, 3311, 10) > cap
    # null pointers: the size check answers first; were it ever to let the
    # request through, the null checks would refuse it before any launch
    rc = L.rr_zchi2_batch_plain_noalloc(None, None, None, None, None, 7958, None, 8000,
                                        3311, 10, 10, None, 0, None, None, None, None)
    assert rc == _lib.RR_ESCRATCH
    assert "scratch" in _lib.status_string(rc)
