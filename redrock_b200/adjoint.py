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


def refine_newton(ctx, pair_target, z0, zlo, zhi, niter=8, tol=1e-8):
    """Minimise chi2(z) for each pair from z0 inside [zlo, zhi] with
    safeguarded Newton steps (a bracket shrinks on every step that does not
    decrease chi2).  Returns (z, chi2, coeff, dchi2_dz, d2chi2_dz2, niter)."""
    z = np.asarray(z0, dtype=np.float64).copy()
    lo = np.asarray(zlo, dtype=np.float64).copy()
    hi = np.asarray(zhi, dtype=np.float64).copy()
    t = np.asarray(pair_target, dtype=np.int32)
    chi2, coeff, _, g, h, _ = chi2_and_grad(ctx, t, z)
    chi2 = chi2.cpu().numpy()
    g = g.cpu().numpy()
    h = h.cpu().numpy()
    coeff = coeff.cpu().numpy()
    active = np.ones(len(z), dtype=bool)
    it = 0
    for it in range(1, niter + 1):
        # Newton step where the curvature is positive, else a gradient step
        # to the bracket's edge; never leave the bracket
        step = np.where(h > 0, -g / np.where(h > 0, h, 1.0), -np.sign(g) * (hi - lo) / 4)
        zn = np.clip(z + step, lo, hi)
        idx = np.nonzero(active & (np.abs(zn - z) > tol * (1 + np.abs(z))))[0]
        if len(idx) == 0:
            break
        c2, co, _, gn, hn, _ = chi2_and_grad(ctx, t[idx], zn[idx])
        c2 = c2.cpu().numpy()
        better = c2 <= chi2[idx]
        acc = idx[better]
        rej = idx[~better]
        # accepted steps move the point; rejected ones shrink the bracket
        # towards the current point
        z[acc] = zn[acc]
        chi2[acc] = c2[better]
        g[acc] = gn.cpu().numpy()[better]
        h[acc] = hn.cpu().numpy()[better]
        coeff[acc] = co.cpu().numpy()[better]
        up = zn[rej] > z[rej]
        hi[rej[up]] = zn[rej[up]]
        lo[rej[~up]] = zn[rej[~up]]
        active[:] = False
        active[idx] = True
    return z, chi2, coeff, g, h, it
