"""Adjoint of the pair scan: dchi2/dz against central finite differences
(dz = 1e-6) and the oracle's FP64 numpy gradient; dchi2/dflux against finite
differences and through torch.autograd; Newton refinement against a dense
grid scan.

Tolerances: |g - g_fd| <= 2e-4 |g_fd| + 20 (chi2 ~ 4e4 is accurate to
~1e-9 relative, so a central difference with dz = 1e-6 is good to ~20);
|g - g_oracle| <= 1e-6 |g| + 1; Newton z within 2e-7 of the dense-grid
parabola minimum.  Finite differences are asserted only where central
differences with steps h and 2h agree (no IGM line switching on inside the
step; chi2(z) has steps there and no derivative).
"""
import numpy as np
import pytest

from tests.conftest import cuda_available

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

from oracle import oracle as O  # noqa: E402
from redrock_b200 import synth  # noqa: E402

H = 1e-6


def _ctx(key, ntarget=3):
    from redrock_b200 import targets as T, templates as TM
    from redrock_b200.adjoint import PairContext
    tg = synth.make_targets(ntarget, seed=61, amp=2.0)
    ts = {t.full_type.replace(":::", "_"): t for t in synth.template_set()}[key]
    rtg = T.from_synth(tg)
    return tg, ts, PairContext(rtg, TM.from_synth(ts))


@pytest.mark.parametrize("key,zs", [("GALAXY", [0.05, 0.4123, 0.9, 1.31]),
                                    ("QSO", [0.8, 2.35, 3.72, 5.05]),
                                    ("STAR_G", [-0.0011, 0.0004])])
def test_dchi2_dz_fd_and_oracle(key, zs):
    from redrock_b200.adjoint import chi2_and_grad
    tg, ts, ctx = _ctx(key)
    pt = np.repeat(np.arange(len(tg)), len(zs)).astype(np.int32)
    pz = np.tile(np.array(zs), len(tg))
    c0, _, _, g, h, _ = chi2_and_grad(ctx, pt, pz)
    cp, *_ = chi2_and_grad(ctx, pt, pz + H)
    cm, *_ = chi2_and_grad(ctx, pt, pz - H)
    cp2, *_ = chi2_and_grad(ctx, pt, pz + 2 * H)
    cm2, *_ = chi2_and_grad(ctx, pt, pz - 2 * H)
    c0, g, cp, cm, cp2, cm2 = (a.cpu().numpy() for a in (c0, g, cp, cm, cp2, cm2))
    fd = (cp - cm) / (2 * H)
    fd2 = (cp2 - cm2) / (4 * H)
    smooth = np.abs(fd - fd2) <= 1e-3 * np.abs(fd) + 20.0
    assert smooth.mean() >= 0.5
    assert np.all(np.abs(g - fd)[smooth] <= 2e-4 * np.abs(fd[smooth]) + 20.0)
    grids = synth.camera_grids()
    for i, (t, z) in enumerate(zip(pt, pz)):
        sp = [O.OSpectrum(s.band, s.wave, s.flux, s.ivar, s.rdata, s.roffsets)
              for s in tg[t].spectra]
        oc, og = O.chi2_grad_z(sp, ts.wave, ts.flux, z, grids, ts.igm_model)
        assert abs(c0[i] - oc) <= 1e-6 * abs(oc)
        if smooth[i]:
            assert abs(g[i] - og) <= 1e-6 * abs(og) + 1.0, (z, g[i], og)


def test_newton_matches_dense_grid():
    """fitz's procedure with Newton in place of the parabola: coarse minimum
    -> 15-point fine grid between its neighbours -> Newton inside the best
    fine cell; compared with a dense (801-point) FP64 scan of that cell."""
    from redrock_b200.adjoint import chi2_and_grad, refine_newton
    tg, ts, ctx = _ctx("GALAXY", ntarget=4)
    zc = ts.redshifts[::5]
    nt = len(tg)
    pt = np.repeat(np.arange(nt), len(zc)).astype(np.int32)
    c, *_ = chi2_and_grad(ctx, pt, np.tile(zc, nt))
    c = c.cpu().numpy().reshape(nt, len(zc))
    imin = np.argmin(c, axis=1)
    zz = np.stack([np.linspace(zc[max(i - 1, 0)], zc[min(i + 1, len(zc) - 1)], 15) for i in imin])
    cf, *_ = chi2_and_grad(ctx, np.repeat(np.arange(nt), 15).astype(np.int32), zz.ravel())
    cf = cf.cpu().numpy().reshape(nt, 15)
    k = np.clip(np.argmin(cf, axis=1), 1, 13)
    lo = zz[np.arange(nt), k - 1]
    hi = zz[np.arange(nt), k + 1]
    z0 = zz[np.arange(nt), k]
    zn, cn, _, gn, hn, _ = refine_newton(ctx, np.arange(nt, dtype=np.int32), z0, lo, hi, niter=12)
    for j in range(nt):
        zd = np.linspace(lo[j], hi[j], 801)
        cd, *_ = chi2_and_grad(ctx, np.full(len(zd), j, dtype=np.int32), zd)
        cd = cd.cpu().numpy()
        m = int(np.clip(np.argmin(cd), 1, len(zd) - 2))
        a, b, _ = np.polyfit(zd[m - 1:m + 2], cd[m - 1:m + 2], 2)
        zbest = -b / (2 * a)
        assert abs(zn[j] - zbest) <= 2e-7 * (1 + zbest), (j, zn[j], zbest)
        assert cn[j] <= cd.min() + 1e-6
        assert abs(gn[j]) <= 1e-3 * np.sqrt(max(hn[j], 1.0)) + 1.0


def test_dchi2_dflux_fd_and_autograd():
    import torch
    from redrock_b200.adjoint import Chi2Scan, chi2_and_grad
    tg, ts, ctx = _ctx("GALAXY", ntarget=2)
    pt = np.array([0, 1, 1], dtype=np.int32)
    pz = np.array([0.41, 0.63, 0.9])
    f0 = ctx.packed_flux().clone()
    _, _, _, _, _, df = chi2_and_grad(ctx, pt, pz, want_dflux=True)
    df = df.cpu().numpy()
    sw = ctx.rows.sw.cpu().numpy()
    pix = [p for p in (100, 2000, 5300, 7700) if sw[0, p] > 0 and sw[1, p] > 0]
    for p in pix:
        for sgn, store in ((1, "p"), (-1, "m")):
            f = f0.clone()
            f[:, p] += sgn * 1e-4
            ctx.set_flux(f)
            c, *_ = chi2_and_grad(ctx, pt, pz)
            if sgn > 0:
                cpl = c.cpu().numpy()
            else:
                cmi = c.cpu().numpy()
        ctx.set_flux(f0)
        fd = (cpl - cmi) / 2e-4
        np.testing.assert_allclose(df[:, p], fd, rtol=1e-5, atol=1e-6)
    # autograd: d(sum chi2)/dz and d/dflux
    z = torch.tensor(pz, dtype=torch.float64, device="cuda", requires_grad=True)
    fl = f0.clone().requires_grad_(True)
    chi2, _ = Chi2Scan.apply(z, fl, ctx, pt)
    chi2.sum().backward()
    _, _, _, g, _, df2 = chi2_and_grad(ctx, pt, pz, want_dflux=True)
    torch.testing.assert_close(z.grad, g, rtol=1e-12, atol=1e-9)
    expect = torch.zeros_like(fl)
    expect.index_add_(0, torch.as_tensor(pt, dtype=torch.int64, device="cuda"), df2)
    torch.testing.assert_close(fl.grad, expect, rtol=1e-12, atol=1e-12)


def test_dpenalty_dz_fd():
    """The [OII] penalty's z derivative (-oii . dc/dz with dc/dz from the
    kernel's (M+P)^-1 (u - v)) against central differences of the penalty
    the kernel itself returns, where the penalty is active on both sides:
    within 1e-4 relative + 1e-3 absolute; zero where the penalty is off."""
    from redrock_b200.adjoint import objective_and_grad
    from redrock_b200.engine import run_pairs_grad
    tg, ts, ctx = _ctx("GALAXY", ntarget=6)
    z = np.linspace(0.05, 1.4, 40)
    pt = np.repeat(np.arange(len(tg)), len(z)).astype(np.int32)
    zz = np.tile(z, len(tg))
    dp = []
    _, _, pen, _, _, _ = run_pairs_grad(ctx.rows, ctx.src, pt, zz, dpen=dp)
    pen, dpen = pen.cpu().numpy(), dp[0].cpu().numpy()
    def fd(h):
        pp = run_pairs_grad(ctx.rows, ctx.src, pt, zz + h)[2].cpu().numpy()
        pm = run_pairs_grad(ctx.rows, ctx.src, pt, zz - h)[2].cpu().numpy()
        return (pp - pm) / (2 * h), (pp > 0) & (pm > 0)
    f1, on1 = fd(1e-6)
    f2, on2 = fd(2e-6)
    on = (pen > 0) & on1 & on2
    # the rebin makes chi2(z) C1, not C2: compare only where the central
    # differences with steps h and 2h agree (no kink inside the step)
    smooth = on & (np.abs(f1 - f2) <= 1e-5 * np.abs(f1) + 1e-3)
    assert smooth.sum() >= 5
    assert np.all(np.abs(dpen[smooth] - f1[smooth]) <= 1e-4 * np.abs(f1[smooth]) + 1e-3)
    assert np.all(dpen[pen == 0] == 0)
    # the objective's derivative is chi2's plus the penalty's
    f, _, g, _ = objective_and_grad(ctx, pt, zz, penalty=True)
    c, _, g0, _ = objective_and_grad(ctx, pt, zz, penalty=False)
    np.testing.assert_allclose(f, c + pen, rtol=0, atol=0)
    np.testing.assert_allclose(g, g0 + dpen, rtol=0, atol=0)
