"""Differentiable chi2(z) on the GPU and Newton redshift refinement.

The adjoint kernel (``rr_zscan_pairs_grad``) returns, per (target, z) pair,
chi2, dchi2/dz (least-squares stationarity: the coefficients drop out),
the envelope curvature d2chi2/dz2 and, on request, dchi2/dflux = 2 W r.

* ``chi2_and_grad``: those arrays for a list of pairs.
* ``Chi2Scan``: a ``torch.autograd.Function`` over (z, flux) -- z per pair,
  flux per target in the packed pixel order of ``RowPack``.
* ``refine_newton``: Newton steps in continuous z for many (target, start)
  pairs at once, bounded to a bracket -- the replacement for the parabola
  through three fine-grid points of redrock's fitz (fitz.py:255-261).
"""

from __future__ import annotations

import numpy as np
import torch

from .engine import GridLayout, RowPack, TemplateSource, pair_ranges_ok, run_pairs_grad


class PairContext:
    """Packed targets + device template for pair evaluations."""

    def __init__(self, targets, template, layout=None):
        if layout is None:
            dwave = {}
            for t in targets:
                for s in t.spectra:
                    dwave.setdefault(s.wavehash, s.wave)
            layout = GridLayout.from_dwave(dwave)
        self.layout = layout
        self.rows = RowPack.from_targets(targets, layout)
        self.src = TemplateSource.from_template(template)
        torch.cuda.current_stream().synchronize()
        self.rows.check()

    def packed_flux(self):
        """Per-target flux in the packed pixel order ([ntarget, npix_row])."""
        sw = self.rows.sw
        g = self.rows.rows[..., -1]
        return torch.where(sw > 0, g / torch.where(sw > 0, sw, torch.ones_like(sw)),
                           torch.zeros_like(g))

    def set_flux(self, flux_packed):
        """Replace the packed flux (sqrt(w) f column) and f^T W f."""
        sw = self.rows.sw
        self.rows.rows[..., -1] = sw * flux_packed
        self.rows.fwf.copy_(((sw * flux_packed) ** 2).sum(dim=1))


def chi2_and_grad(ctx, pair_target, pair_z, want_dflux=False):
    ok = pair_ranges_ok(ctx.src, ctx.layout, pair_z)
    if not np.all(ok):
        raise ValueError('edges must be within input x range')
    return run_pairs_grad(ctx.rows, ctx.src, pair_target, pair_z, want_dflux=want_dflux)


def objective_and_grad(ctx, pair_target, pair_z, penalty=False):
    """(objective, coeff, d objective / dz, envelope curvature) host arrays
    per pair: chi2, or with penalty=True chi2 + the [OII] penalty -- what
    fitz ranks its fine-grid points by -- and its exact z derivative."""
    ok = pair_ranges_ok(ctx.src, ctx.layout, pair_z)
    if not np.all(ok):
        raise ValueError('edges must be within input x range')
    dp = [] if penalty else None
    c2, co, pen, g, h, _ = run_pairs_grad(ctx.rows, ctx.src, pair_target, pair_z, dpen=dp)
    c2, co, g, h = c2.cpu().numpy(), co.cpu().numpy(), g.cpu().numpy(), h.cpu().numpy()
    if penalty:
        c2 = c2 + pen.cpu().numpy()
        g = g + dp[0].cpu().numpy()
    return c2, co, g, h


class Chi2Scan(torch.autograd.Function):
    """chi2 of pairs (target index, z) as a differentiable function of z
    (per pair) and of the packed flux (per target)."""

    @staticmethod
    def forward(fctx, z, flux_packed, ctx, pair_target):
        if flux_packed is not None:
            ctx.set_flux(flux_packed.detach())
        zc = z.detach().to(torch.float64).cpu().numpy()
        chi2, coeff, pen, g, h, df = chi2_and_grad(ctx, pair_target, zc,
                                                   want_dflux=flux_packed is not None)
        tgt = torch.as_tensor(np.asarray(pair_target, dtype=np.int64), device=chi2.device)
        fctx.save_for_backward(g, df if df is not None else g, tgt)
        fctx.has_flux = flux_packed is not None
        fctx.ntarget = ctx.rows.ntarget
        fctx.mark_non_differentiable(coeff)
        return chi2, coeff

    @staticmethod
    def backward(fctx, gchi2, gcoeff):
        g, df, tgt = fctx.saved_tensors
        gz = gchi2 * g
        gf = None
        if fctx.has_flux:
            gf = torch.zeros((fctx.ntarget, df.shape[1]), dtype=df.dtype, device=df.device)
            gf.index_add_(0, tgt, gchi2[:, None] * df)
        return gz, gf, None, None


def refine_newton(ctx, pair_target, z0, zlo, zhi, niter=24, tol=1e-10, penalty=False):
    """Minimise chi2(z) -- chi2 + [OII] penalty with penalty=True, fitz's
    objective -- for each pair inside [zlo, zhi], starting from z0
    (the best fine-grid point; zlo, zhi its neighbours), with Newton steps
    on dchi2/dz = 0.  The adjoint kernel's dchi2/dz is exact, so the
    curvature of each step comes from exact gradient differences (the
    secant of dchi2/dz across the current bracket) rather than from the
    kernel's envelope curvature, which leaves out the template's second
    derivative (narrow lines make that term large).  A bracket [a, b] with
    dchi2/dz(a) <= 0 <= dchi2/dz(b) is kept throughout; a step landing
    outside it, or a side of the bracket kept twice in a row, falls back to
    the Illinois (modified regula falsi) step, so every iteration shrinks
    the bracket.  One pair-gradient launch per iteration for the pairs still
    moving.

    Returns (z, chi2, coeff, dchi2_dz, d2chi2_dz2, iterations): z is the
    evaluated point of lowest chi2 (the root of dchi2/dz once converged),
    d2chi2_dz2 the secant curvature of the final bracket (> 0), or -1 where
    no bracket formed (the minimum lies beyond [zlo, zhi]; z is then the best
    point evaluated)."""
    t = np.asarray(pair_target, dtype=np.int32)
    n = len(t)
    z0 = np.asarray(z0, dtype=np.float64)
    zlo = np.asarray(zlo, dtype=np.float64)
    zhi = np.asarray(zhi, dtype=np.float64)
    if n == 0:
        e = np.zeros(0)
        return e, e.copy(), np.zeros((0, ctx.src.nbasis)), e.copy(), e.copy(), 0
    c3, co3, g3, h3 = objective_and_grad(ctx, np.tile(t, 3), np.concatenate([zlo, z0, zhi]),
                                         penalty)
    c3 = c3.reshape(3, n)
    g3 = g3.reshape(3, n)
    h3 = h3.reshape(3, n)
    co3 = co3.reshape(3, n, -1)
    zs = np.stack([zlo, z0, zhi])
    # best evaluated point so far
    k = np.argmin(c3, axis=0)
    cols = np.arange(n)
    zbest, cbest, gbest, hbest = zs[k, cols], c3[k, cols], g3[k, cols], h3[k, cols]
    cobest = co3[k, cols]
    # bracket on the side of z0 where dchi2/dz changes sign
    right = g3[1] < 0
    a = np.where(right, z0, zlo)
    b = np.where(right, zhi, z0)
    ga = np.where(right, g3[1], g3[0])
    gb = np.where(right, g3[2], g3[1])
    active = (ga <= 0) & (gb >= 0) & (b > a)
    # no sign change on that side although z0 is the best point: the
    # objective has a bump between z0 and the neighbour, and a minimum on
    # the way (descending from z0, then up and down again).  Probe the
    # gradient at 1/4, 1/2, 3/4 of the way to find where it turns positive
    # (negative, going left).
    probe = np.nonzero(~active & (b > a))[0]
    if len(probe):
        fr = np.array([0.25, 0.5, 0.75])
        rp = right[probe]
        zp = np.where(rp[:, None], a[probe, None] + fr[None, :] * (b - a)[probe, None],
                      b[probe, None] - fr[None, :] * (b - a)[probe, None])
        cp, cop, gp, _ = objective_and_grad(ctx, np.repeat(t[probe], 3), zp.ravel(), penalty)
        cp, gp = cp.reshape(-1, 3), gp.reshape(-1, 3)
        cop = cop.reshape(len(probe), 3, -1)
        for q, i in enumerate(probe):
            kb = np.argmin(cp[q])
            if cp[q, kb] < cbest[i]:
                zbest[i], cbest[i], gbest[i], cobest[i] = zp[q, kb], cp[q, kb], gp[q, kb], cop[q, kb]
            prev_z, prev_g = (a[i], ga[i]) if rp[q] else (b[i], gb[i])
            for k in range(3):
                turned = gp[q, k] >= 0 if rp[q] else gp[q, k] <= 0
                if turned:
                    if rp[q]:
                        a[i], ga[i], b[i], gb[i] = prev_z, prev_g, zp[q, k], gp[q, k]
                    else:
                        a[i], ga[i], b[i], gb[i] = zp[q, k], gp[q, k], prev_z, prev_g
                    active[i] = True
                    break
                prev_z, prev_g = zp[q, k], gp[q, k]
    # Illinois weights: the stored end values used for the next step (the
    # true gradients ga, gb are kept for the curvature)
    wa, wb = ga.copy(), gb.copy()
    last = np.zeros(n, dtype=np.int8)    # end replaced by the last step: -1 a, +1 b
    it = 0
    for it in range(1, niter + 1):
        idx = np.nonzero(active & ((b - a) > tol * (1 + np.abs(a))))[0]
        if len(idx) == 0:
            break
        ai, bi, wai, wbi = a[idx], b[idx], wa[idx], wb[idx]
        # the Newton step from a with the secant curvature of the bracket
        # (the regula falsi point); midpoint if it would not be inside
        den = wbi - wai
        zn = np.where(den > 0, ai - wai * (bi - ai) / np.where(den > 0, den, 1.0),
                      0.5 * (ai + bi))
        zn = np.where((zn > ai) & (zn < bi), zn, 0.5 * (ai + bi))
        c2, co, gn, _ = objective_and_grad(ctx, t[idx], zn, penalty)
        better = c2 < cbest[idx]
        upd = idx[better]
        zbest[upd], cbest[upd], gbest[upd] = zn[better], c2[better], gn[better]
        cobest[upd] = co[better]
        # the minimum lies above zn where dchi2/dz(zn) < 0, else below;
        # an end kept twice in a row has its stored value halved (Illinois)
        low = gn < 0
        la, lb = idx[low], idx[~low]
        a[la], ga[la], wa[la] = zn[low], gn[low], gn[low]
        wb[la] = np.where(last[la] == -1, 0.5 * wb[la], wb[la])
        last[la] = -1
        b[lb], gb[lb], wb[lb] = zn[~low], gn[~low], gn[~low]
        wa[lb] = np.where(last[lb] == 1, 0.5 * wa[lb], wa[lb])
        last[lb] = 1
        active[idx[gn == 0]] = False
    bracketed = (ga <= 0) & (gb >= 0) & (b > a)
    # no bracket at all: the best point is not a verified minimum (reported
    # with a negative curvature, which fitz flags as BAD_MINFIT)
    curv = np.where(bracketed, (gb - ga) / np.where(b > a, b - a, 1.0), -1.0)
    return zbest, cbest, cobest, gbest, curv, it
