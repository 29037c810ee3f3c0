"""Tensor-core y = Tb^T W f (rr_pack_g + rr_ygemm) against FP64 references.

* G = R^T W f per target: a numpy restatement from the packed rows
  (relative 1e-12 of each target's max).
* Y = G^T . basis per variant, against a torch FP64 product of the same
  operands, relative to S = sum_q |G| |T| (the natural scale of a dot
  product's rounding error):
    INT8X7 (Ozaki, exact int32 accumulation)   <= 1e-12 S
    INT8X6 (six base-256 digits, one bit less)  <= 4e-12 S
    BF16X3 / TF32X3 (FP32 accumulation in TMEM) <= K 2^-24 S with K the
      padded pixel count (~5e-4 S at K = 8064), the worst-case bound of a
      K-term FP32 sum
* The fused scan fed with either INT8 y keeps the FP64 path's bounds
  against the oracle (|dchi2| <= 2e-5, identical argmin, coefficients
  1e-5).  With the FP32-accumulated variants chi2 = f^T W f - c^T y moves
  by about 2 c^T dy (first order), so they are held to
  |dchi2| <= 4 K 2^-24 sum_i |c_i| S_i; at DESI S/N that is far above the
  1e-3 acceptance bar (bench.py --ygemm-study reports the actual errors).
"""

import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from oracle import oracle as O  # noqa: E402
from redrock_b200 import synth  # noqa: E402

VARIANTS = ["int8x7", "int8x6", "bf16x3", "tf32x3"]
I8 = ("int8x7", "int8x6")
TOL_S = {"int8x7": 1e-12, "int8x6": 4e-12}
# per-output error bound K 2^(e_t + e_n - BOUND_SHIFT) of each INT8 scheme
BOUND_SHIFT = {"int8x7": 45, "int8x6": 44}


def _case(ntarget, zsub, seed):
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    from redrock_b200.engine import (DeviceBasis, GridLayout, TargetBatch, TargetPack,
                                     TemplateSource)
    tg = synth.make_targets(ntarget, seed=seed, mask_range=(0.0, 0.4), drop_camera_frac=0.1)
    rtg = T.from_synth(tg)
    layout = GridLayout.from_dwave(synth.camera_grids())
    pack = TargetPack(TargetBatch(rtg, layout).to_device())
    tset = synth.template_set(zsub=zsub, stars=("K",))
    bases = [DeviceBasis.build(TemplateSource.from_template(TM.from_synth(ts)), layout)
             for ts in tset]
    pack.check()
    return tg, tset, layout, pack, bases


def layout_kpad(layout):
    from redrock_b200 import _lib
    return int(_lib.lib().rr_ygemm_kpad(layout.pix_stride))


def _g_reference(pack, layout):
    rw = pack.rw.cpu().numpy()  # [nblock][npix_block][12][32]
    nb, npos = rw.shape[0], rw.shape[0] * 32
    g = np.zeros((layout.pix_stride, npos))
    for sd in pack.segs:
        bo, npx, ro = sd.basis_offset, sd.npix_pad, sd.rw_offset
        f = rw[:, ro:ro + npx, 11, :]
        for k in range(11):
            q0 = bo + k - 5
            g[q0:q0 + npx] += (rw[:, ro:ro + npx, k, :] * f).transpose(1, 0, 2).reshape(npx, npos)
    return g, nb


def test_pack_g_matches_numpy():
    from redrock_b200.engine import YGemm
    tg, tset, layout, pack, bases = _case(45, 211, seed=31)
    yg = YGemm(pack, "int8x7")
    gref, nblock = _g_reference(pack, layout)
    g = yg.g.cpu().numpy()
    npos = nblock * 32
    assert yg.kpad >= layout.pix_stride and yg.kpad % 64 == 0
    assert np.all(g[layout.pix_stride:] == 0) and np.all(g[:, npos:] == 0)
    scale = np.maximum(np.abs(gref).max(axis=0), 1e-300)
    assert np.all(np.abs(g[:layout.pix_stride, :npos] - gref) <= 1e-12 * scale)
    # exponents with the digit schemes' margin: 128/127 max |G| of each
    # target in [2^(e-1), 2^e), so max |G| < 127/128 2^e
    e = yg.row_exp.cpu().numpy()[:npos].astype(np.int64)
    m = np.abs(gref).max(axis=0)
    nz = m > 0
    assert np.all(e[~nz] == 0)
    ee = e[nz] - 4096
    assert np.all(m[nz] < np.ldexp(127.0 / 128.0, ee))
    assert np.all(m[nz] * (128.0 / 127.0) >= np.ldexp(0.5, ee) * (1 - 1e-15))


@pytest.mark.parametrize("variant", VARIANTS)
def test_ygemm_matches_fp64_product(variant):
    import torch
    from redrock_b200.engine import YGemm
    tg, tset, layout, pack, bases = _case(45, 157, seed=32)
    yg = YGemm(pack, variant)
    g = yg.g[:layout.pix_stride]
    for b in bases:
        y = yg.y(b)
        t = b.basis[:, :, :b.nbasis]
        ref = torch.einsum("qp,zqi->pzi", g, t)
        s = torch.einsum("qp,zqi->pzi", g.abs(), t.abs())
        torch.cuda.synchronize()
        tol = TOL_S[variant] if variant in I8 else yg.kpad * 2.0 ** -24
        err = ((y - ref).abs() / s.clamp_min(1e-300))[:pack.nblock * 32]
        assert torch.isfinite(y[:pack.nblock * 32]).all()
        assert float(err.max()) <= tol, (variant, b.nbasis, float(err.max()))


@pytest.mark.parametrize("variant", I8)
def test_i8_digits_edge_values(variant):
    """Entries at and just below a power of two and just below the 127/128
    margin of the exponents (where the leading digit reaches +-64 in base
    128 and +-127 in base 256), of both signs: the error stays within the
    scheme's bound K 2^-45 (base 128) or K 2^-44 (base 256) times
    2^(e_t + e_n) -- rounding to 49- / 48-bit integers plus the dropped
    digit products.  A lost carry would be an error of the order of
    2^(e_t + e_n) itself."""
    import torch
    from redrock_b200 import _lib
    from redrock_b200.device import ptr
    from redrock_b200.engine import YGemm
    tg, tset, layout, pack, bases = _case(33, 401, seed=34)
    yg = YGemm(pack, variant)
    rng = np.random.default_rng(5)
    g = yg.g.cpu().numpy()
    npos = pack.nblock * 32
    for t in range(npos):
        e = int(rng.integers(-20, 20))
        q = rng.choice(layout.pix_stride, size=8, replace=False)
        if t % 2:
            # rows whose maximum sits at or just below a power of two
            g[q[0], t] = np.ldexp(1.0 - 2.0 ** -40, e)
            g[q[1], t] = -np.ldexp(1.0 - 2.0 ** -40, e)
            g[q[2], t] = np.ldexp(0.996, e)
            g[q[3], t] = -np.ldexp(0.9961, e)
        else:
            # rows whose maximum sits just below the 127/128 margin
            g[q[0], t] = np.ldexp(127.0 / 128.0 * (1.0 - 2.0 ** -40), e)
            g[q[1], t] = -np.ldexp(127.0 / 128.0 * (1.0 - 2.0 ** -40), e)
            g[q[2], t] = np.ldexp(0.9921, e)
            g[q[3], t] = -np.ldexp(0.99218, e)
        g[q[4], t] = np.ldexp(0.5, e)
        g[q[5], t] = -np.ldexp(0.75, e)
        g[q[6], t] = np.ldexp(0.5 * 127.0 / 128.0, e)
        g[q[7], t] = -np.ldexp(0.25 * (1.0 - 2.0 ** -30), e)
    gt = torch.as_tensor(g, device=yg.g.device)
    yg.g.copy_(gt)
    m = np.abs(g).max(axis=0)
    et = np.where(m > 0, np.frexp(m * (128.0 / 127.0))[1], 0)
    ex = np.where(m > 0, et + 4096, 0).astype(np.int32)
    yg.row_exp.copy_(torch.as_tensor(ex, device=yg.g.device))
    L = _lib.lib()
    assert L.rr_slice_g_i8(yg.variant, ptr(yg.g), ptr(yg.row_exp), yg.npos, yg.kpad,
                           ptr(yg.g_digits), None) == 0
    for b in bases:
        y = yg.y(b)
        t = b.basis[:, :, :b.nbasis]
        ref = torch.einsum("qp,zqi->pzi", gt[:layout.pix_stride], t)
        err = (y - ref).abs()[:npos].cpu().numpy()
        ce = b.i8_digits(yg.kpad, variant=yg.variant)[1].cpu().numpy()
        ce = ce[:b.nz * b.nbasis].reshape(b.nz, b.nbasis)
        en = np.where(ce > 0, ce - 4096, 0)
        bound = yg.kpad * np.ldexp(1.0, et[:npos, None, None] + en[None] - BOUND_SHIFT[variant])
        assert np.all(err <= bound), float(np.max(err / bound))


def test_fused_with_tensor_core_y_vs_oracle():
    from redrock_b200.engine import run_fused
    tg, tset, layout, pack, bases = _case(37, 97, seed=33)
    ref, st = run_fused(pack, bases)
    st.check("fused")
    grids = synth.camera_grids()
    pick = [0, 17, 36]
    rows = pack.rows.cpu().numpy()
    import torch
    from redrock_b200.engine import YGemm
    gabs = YGemm(pack, "bf16x3").g[:layout.pix_stride].abs()
    pos = torch.as_tensor([int(np.nonzero(rows == t)[0][0]) for t in range(len(tg))],
                          device=gabs.device)
    for variant in VARIANTS:
        res, st = run_fused(pack, bases, ygemm=variant)
        st.check(variant)
        for ts, r, r0, b in zip(tset, res, ref, bases):
            zc, co = r.zchi2.cpu().numpy(), r.zcoeff.cpu().numpy()
            zc0 = r0.zchi2.cpu().numpy()
            if variant in I8:
                tdata = O.template_basis(ts.wave, ts.flux, ts.redshifts, grids, ts.igm_model)
                oii = O.oii_template(ts.wave, ts.flux) if ts.spectype == "GALAXY" else None
                ospecs = [[O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
                           for s in tg[i].spectra] for i in pick]
                ozc, oco, ope = O.calc_zchi2(ospecs, tdata, len(ts.redshifts), ts.flux.shape[0],
                                             OIItemplate=oii)
                for j, i in enumerate(pick):
                    assert np.max(np.abs(zc[i] - ozc[j])) <= 2e-5
                    assert np.argmin(zc[i]) == np.argmin(ozc[j])
                    scale = np.maximum(np.abs(oco[j]).max(axis=-1, keepdims=True), 1e-300)
                    assert np.all(np.abs(co[i] - oco[j]) <= 1e-5 * scale)
            else:
                ok = zc0 < 9999999.0
                s_abs = torch.einsum("qp,zqi->pzi", gabs, b.basis[:, :, :b.nbasis].abs())[pos]
                bound = (4 * layout_kpad(layout) * 2.0 ** -24
                         * (r0.zcoeff.abs() * s_abs).sum(-1)).cpu().numpy()
                d = np.abs(zc - zc0)
                assert np.all(np.isfinite(zc))
                assert np.all(d[ok] <= bound[ok]), float(np.max(d[ok] / bound[ok]))


@pytest.mark.parametrize("nb", [3, 7])
def test_uncommon_nbasis_default_path_vs_oracle(nb):
    """nbasis outside {4, 5, 10} runs in the second fused instantiation; its
    y comes from the INT8 GEMM (default path) -- both against the oracle."""
    from redrock_b200 import targets as T
    from redrock_b200 import templates as TM
    from redrock_b200 import zscan
    gal = synth.template_set(zsub=61, stars=())[0]
    ts = synth.TemplateSpec("GALAXY", f"nb{nb}", gal.wave, gal.flux[:nb].copy(),
                            gal.redshifts, gal.igm_model)
    tg = synth.make_targets(5, seed=40 + nb, mask_range=(0.0, 0.3), drop_camera_frac=0.3)
    dtg = T.DistTargetsCopy(T.from_synth(tg))
    dt = TM.DistTemplate(TM.from_synth(ts), dtg.wavegrids())
    zc, co, pe = zscan.calc_zchi2([t.targetid for t in tg], dtg.local(), dt)
    grids = synth.camera_grids()
    tdata = O.template_basis(ts.wave, ts.flux, ts.redshifts, grids, ts.igm_model)
    oii = O.oii_template(ts.wave, ts.flux)
    ospecs = [[O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
               for s in t.spectra] for t in tg]
    ozc, oco, ope = O.calc_zchi2(ospecs, tdata, len(ts.redshifts), nb, OIItemplate=oii)
    assert np.max(np.abs(zc - ozc)) <= 2e-5
    np.testing.assert_array_equal(np.argmin(zc, axis=1), np.argmin(ozc, axis=1))
    scale = np.maximum(np.abs(oco).max(axis=-1, keepdims=True), 1e-300)
    assert np.all(np.abs(co - oco) <= 1e-5 * scale)
    np.testing.assert_allclose(pe, ope, rtol=1e-8, atol=1e-8)
