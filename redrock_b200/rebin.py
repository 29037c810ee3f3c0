"""Drop-in ``trapz_rebin`` / ``rebin_template`` running on the GPU.

Same signatures, output shapes and ValueError as redrock 0.22
(rebin.py:212-378 and :453-517).  The arithmetic is the CUDA kernel in
csrc/rr_basis.cu, bit-identical to redrock's CPU rebin.  Results come back
as numpy arrays when ``use_gpu`` is false (what redrock's CPU callers expect)
and as CUDA tensors when it is true.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import StatusWord, device, ptr, stream_handle, to_device, to_numpy
from .engine import centers2edges

__all__ = ["centers2edges", "trapz_rebin", "rebin_template"]


def _host_scalar(v):
    if isinstance(v, torch.Tensor):
        return float(v.item())
    return float(v)


def trapz_rebin(x, y, xnew=None, edges=None, myz=None, use_gpu=False, xmin=None, xmax=None,
                edge_min=None, edge_max=None):
    """Rebin y(x) flux density by trapezoidal integration between bin edges."""
    if edges is None:
        edges = centers2edges(to_numpy(xnew))
    elif not isinstance(edges, torch.Tensor):
        edges = np.asarray(edges, dtype=np.float64)
    nbins = len(edges) - 1
    if edge_min is None:
        edge_min = edges[0]
    if edge_max is None:
        edge_max = edges[-1]
    scalar_z = False
    if myz is None:
        myz = np.array([0.0])
        scalar_z = True
    elif np.isscalar(myz):
        myz = np.array([myz], dtype=np.float64)
        scalar_z = True
    elif not isinstance(myz, torch.Tensor):
        myz = np.asarray(myz, dtype=np.float64)
    nz = len(myz)
    if nz == 0:
        return np.zeros((0, nbins, 1), dtype=np.float64)
    if xmin is None or xmax is None:
        zh = to_numpy(myz)
        x0 = _host_scalar(x[0])
        x1 = _host_scalar(x[-1])
        if xmin is None:
            xmin = x0 * (1 + zh.max())
        if xmax is None:
            xmax = x1 * (1 + zh.min())
    edge_min = _host_scalar(edge_min)
    edge_max = _host_scalar(edge_max)
    if edge_min < xmin or edge_max > xmax:
        raise ValueError('edges must be within input x range')
    y_ndim = len(y.shape)
    scalar_basis = y_ndim == 1
    dy = to_device(y)
    if scalar_basis:
        dy = dy[None, :]
    nbasis = dy.shape[0]
    if nbasis > 16:
        # the kernel keeps one accumulator per basis in registers; rebin
        # wider inputs in groups of 16 bases
        parts = [trapz_rebin(x, dy[i:i + 16], edges=edges, myz=myz, use_gpu=True, xmin=xmin,
                             xmax=xmax, edge_min=edge_min, edge_max=edge_max)
                 for i in range(0, nbasis, 16)]
        parts = [p if p.dim() == 3 else p[None] for p in parts]
        res = torch.cat(parts, dim=2)
        shape = (nbins,) + (() if scalar_basis else (nbasis,))
        if not scalar_z:
            shape = (nz,) + shape
        res = res.reshape(shape)
        return res if use_gpu else res.cpu().numpy()
    dx = to_device(x)
    de = to_device(edges)
    dz = to_device(myz)
    out = torch.empty((nz, nbins, nbasis), dtype=torch.float64, device=device())
    st = StatusWord()
    rc = _lib.lib().rr_trapz_rebin(ptr(dx), dx.numel(), ptr(dy), nbasis, ptr(de), nbins, ptr(dz),
                                   nz, float(xmin), float(xmax), edge_min, edge_max, ptr(out),
                                   st.ptr, stream_handle())
    _lib.check(rc, "rr_trapz_rebin")
    st.check("rr_trapz_rebin")
    shape = (nbins,) + (() if scalar_basis else (nbasis,))
    if not scalar_z:
        shape = (nz,) + shape
    out = out.reshape(shape)
    return out if use_gpu else out.cpu().numpy()


def rebin_template(template, myz, dwave=None, dedges=None, use_gpu=False, xmin=None, xmax=None):
    """dict[wavehash] -> (nz, nlambda, nbasis) rebinned template."""
    zh = to_numpy(myz)
    if xmin is None:
        xmin = template.minwave * (1 + zh.max())
    if xmax is None:
        xmax = template.maxwave * (1 + zh.min())
    result = {}
    if dwave is not None:
        for hs, wave in dwave.items():
            result[hs] = trapz_rebin(template.wave, template.flux, xnew=wave, myz=myz,
                                     use_gpu=use_gpu, xmin=xmin, xmax=xmax)
    elif dedges is not None:
        for hs, edges in dedges.items():
            minedge = maxedge = None
            if type(edges) is tuple:
                edges, minedge, maxedge = edges
            result[hs] = trapz_rebin(template.wave, template.flux, edges=edges, myz=myz,
                                     use_gpu=use_gpu, xmin=xmin, xmax=xmax, edge_min=minedge,
                                     edge_max=maxedge)
    return result
