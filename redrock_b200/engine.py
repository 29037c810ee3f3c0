"""Device-resident scan engine: wavelength-grid layout, template bases,
packed targets and the fused / plain scan launches.

HBM layout (all FP64):

* basis of one template: ``[nz][pix_stride][stride]``.  The wavelength grids
  (one per redrock "wavehash") are laid end to end; grid g owns padded
  pixels ``[pix_offset_g - 5, pix_offset_g + npix_pad_g + 5)``, its real
  pixels start at ``pix_offset_g``, and the 5-pixel margins and the tail up
  to ``npix_pad_g`` (a multiple of 16) are zero, so the banded resolution
  product never reads another grid's values.  ``stride`` is nbasis rounded
  up to even so every pixel row is 16-byte aligned for the bulk copies.
* packed targets: ``rw[block][npix_block][12][32]`` -- 32 targets per block,
  one per lane, the 11 band values of sqrt(w) R and sqrt(w) f for every
  pixel of every segment (one segment per (grid, spectrum slot)), lanes
  fastest so the scan's copies are contiguous.
"""

from __future__ import annotations

import ctypes
from collections import OrderedDict

import numpy as np
import torch

from . import _lib
from .device import StatusWord, device, ptr, stream_handle, struct_bytes, to_device


def round_up(n, m):
    return ((n + m - 1) // m) * m


def centers2edges(centers):
    """Bin edges from centres (redrock rebin.py:100-118)."""
    centers = np.asarray(centers)
    edges = np.zeros(len(centers) + 1)
    edges[1:-1] = (centers[0:-1] + centers[1:]) / 2.0
    edges[0] = centers[0] - (centers[1] - edges[1])
    edges[-1] = centers[-1] + (centers[-1] - edges[-2])
    return edges


# ---------------------------------------------------------------------------
# wavelength-grid layout
# ---------------------------------------------------------------------------
class GridLayout:
    """Ordered set of wavelength grids (wavehash -> wave) and their place in
    the padded basis layout."""

    def __init__(self, grids):
        # grids: iterable of (key, npix, wave-or-None)
        self.keys = []
        self.npix = []
        self.npix_pad = []
        self.pix_offset = []
        self.waves = []
        start = 0
        for key, npix, wave in grids:
            npix = int(npix)
            npad = round_up(npix, _lib.chunk())
            self.keys.append(key)
            self.npix.append(npix)
            self.npix_pad.append(npad)
            self.pix_offset.append(start + _lib.HALF_BAND)
            self.waves.append(None if wave is None else np.asarray(wave, dtype=np.float64))
            start += npad + 2 * _lib.HALF_BAND
        self.pix_stride = start
        self.index = {k: i for i, k in enumerate(self.keys)}
        self._dev = {}

    @classmethod
    def from_dwave(cls, dwave):
        return cls((k, len(w), w) for k, w in dwave.items())

    @property
    def signature(self):
        return tuple(zip(self.keys, self.npix))

    def device_arrays(self, i):
        """(edges, wave) device tensors of grid i, cached."""
        if i not in self._dev:
            w = self.waves[i]
            if w is None:
                raise ValueError(f"grid {self.keys[i]!r} has no wavelength array")
            e = centers2edges(w)
            self._dev[i] = (to_device(e), to_device(w), float(e[0]), float(e[-1]))
        return self._dev[i]


# ---------------------------------------------------------------------------
# template bases on the device
# ---------------------------------------------------------------------------
class TemplateSource:
    """A template's rest-frame arrays and redshift grid, uploaded once."""

    def __init__(self, wave, flux, redshifts, igm_model, oii=None, method=_lib.RR_SOLVE_PCA):
        wave = np.ascontiguousarray(wave, dtype=np.float64)
        flux = np.ascontiguousarray(np.atleast_2d(flux), dtype=np.float64)
        self.nbasis = flux.shape[0]
        if self.nbasis > _lib.MAX_NBASIS:
            raise NotImplementedError(f"nbasis {self.nbasis} > {_lib.MAX_NBASIS} is not supported")
        if igm_model not in _lib.IGM_CODES:
            raise ValueError(f"Unrecognized model {igm_model}")
        self.igm = _lib.IGM_CODES[igm_model]
        self.zhost = np.ascontiguousarray(redshifts, dtype=np.float64)
        self.nx = len(wave)
        self.x = to_device(wave)
        self.y = to_device(flux)
        self.z = to_device(self.zhost)
        self.oii = oii
        self.oii_dev = None if oii is None else to_device(np.asarray(oii, dtype=np.float64))
        self.method = method
        self.x_first = float(wave[0])
        self.x_last = float(wave[-1])
        if len(self.zhost):
            self.xmin = float(wave[0] * (1 + self.zhost.max()))
            self.xmax = float(wave[-1] * (1 + self.zhost.min()))
        self.nbytes = wave.nbytes + flux.nbytes + self.zhost.nbytes

    @classmethod
    def from_template(cls, template):
        from .templates import oii_sums, solve_code
        return cls(template.wave, template.flux, template.redshifts, template.igm_model,
                   oii=oii_sums(template), method=solve_code(template))


class DeviceBasis:
    """One template's redshifted, resolution-ready basis for all z."""

    def __init__(self, basis, layout, nbasis, redshifts, oii=None, method=_lib.RR_SOLVE_PCA,
                 prior=None):
        self.basis = basis
        self.layout = layout
        self.nbasis = int(nbasis)
        self.stride = int(basis.shape[2])
        self.redshifts = np.asarray(redshifts, dtype=np.float64)
        self.nz = len(self.redshifts)
        self.oii = None if oii is None else to_device(oii)
        self.method = method
        self.prior = None if prior is None else to_device(prior)

    @classmethod
    def build(cls, src, layout, stream=None, status=None, **kw):
        """Fused rebin + IGM for every z (rr_build_basis).

        ``src`` is a TemplateSource (device-resident template arrays).  With
        a caller-owned ``status`` word the call stays asynchronous; otherwise
        it synchronises and checks the kernel status.
        """
        L = _lib.lib()
        dev = device()
        nb = src.nbasis
        stride = round_up(nb, 2)
        z = src.zhost
        basis = torch.empty((len(z), layout.pix_stride, stride), dtype=torch.float64, device=dev)
        kw.setdefault("oii", src.oii_dev)
        kw.setdefault("method", src.method)
        if len(z) == 0:
            return cls(basis, layout, nb, z, **kw)
        descs = []
        for i in range(len(layout.keys)):
            e, w, emin, emax = layout.device_arrays(i)
            apply = 0
            if src.igm != _lib.RR_IGM_NONE:
                # redrock skips the IGM product when no redshift puts the
                # grid's bluest pixel below Lyman-alpha (igm.py:396-401)
                apply = int(not (np.min(layout.waves[i]) / (1. + np.max(z)) > 1215.67))
            descs.append(_lib.GridDesc(ptr(e), ptr(w), layout.npix[i], layout.npix_pad[i],
                                       layout.pix_offset[i], emin, emax, apply, 0))
        st = status or StatusWord(dev)
        arr = (_lib.GridDesc * len(descs))(*descs)
        rc = L.rr_build_basis(ptr(src.x), src.nx, ptr(src.y), nb, ptr(src.z), len(z), src.xmin,
                              src.xmax, arr, len(descs), src.igm, layout.pix_stride, stride,
                              ptr(basis), st.ptr, stream_handle(stream))
        _lib.check(rc, "rr_build_basis")
        if status is None:
            torch.cuda.current_stream().synchronize()
            st.check("rr_build_basis")
        return cls(basis, layout, nb, z, **kw)

    @classmethod
    def from_tdata(cls, tdata, layout, redshifts=None, **kw):
        """Device copy of redrock-layout bases dict[wavehash] -> (nz, npix, nb)
        (numpy or CUDA tensors) into the padded layout."""
        dev = device()
        first = next(iter(tdata.values()))
        nz, _, nb = first.shape
        if nb > _lib.MAX_NBASIS:
            raise NotImplementedError(f"nbasis {nb} > {_lib.MAX_NBASIS} is not supported")
        stride = round_up(nb, 2)
        basis = torch.zeros((nz, layout.pix_stride, stride), dtype=torch.float64, device=dev)
        for i, k in enumerate(layout.keys):
            a = tdata[k]
            off, n = layout.pix_offset[i], layout.npix[i]
            if tuple(a.shape) != (nz, n, nb):
                raise ValueError(f"template data for {k!r} has shape {tuple(a.shape)}, "
                                 f"expected {(nz, n, nb)}")
            basis[:, off:off + n, :nb].copy_(to_device(a))
        z = np.zeros(nz) if redshifts is None else redshifts
        return cls(basis, layout, nb, z, **kw)

    def i8_digits(self, kpad, stream=None, variant=_lib.RR_YGEMM_INT8X7):
        """(digit planes, column exponents) of this basis for the exact
        tensor-core y of an INT8 scheme (rr_basis_col_exp +
        rr_slice_basis_i8), cached per scheme."""
        cache = self.__dict__.setdefault("_i8", {})
        cached = cache.get(variant)
        if cached is not None and cached[0] == kpad:
            return cached[1], cached[2]
        L = _lib.lib()
        sh = stream_handle(stream)
        dev = self.basis.device
        ce = torch.empty(max(self.nz * self.nbasis, 1), dtype=torch.int32, device=dev)
        rc = L.rr_basis_col_exp(ptr(self.basis), self.nz, self.layout.pix_stride, self.nbasis,
                                self.stride, ptr(ce), sh)
        _lib.check(rc, "rr_basis_col_exp")
        nbytes = int(L.rr_ygemm_i8_basis_bytes(variant, self.nz, self.nbasis, kpad))
        digits = torch.empty(max(nbytes, 16), dtype=torch.uint8, device=dev)
        rc = L.rr_slice_basis_i8(variant, ptr(self.basis), self.nz, self.layout.pix_stride,
                                 self.nbasis, self.stride, kpad, ptr(ce), ptr(digits), sh)
        _lib.check(rc, "rr_slice_basis_i8")
        cache[variant] = (kpad, digits, ce)
        return digits, ce

    def data_dict(self, as_numpy=True):
        """redrock's DistTemplate.local.data view: dict[wavehash] -> (nz, npix, nb)."""
        out = {}
        for i, k in enumerate(self.layout.keys):
            off, n = self.layout.pix_offset[i], self.layout.npix[i]
            v = self.basis[:, off:off + n, :self.nbasis]
            out[k] = v.cpu().numpy().copy() if as_numpy else v
        return out


# ---------------------------------------------------------------------------
# targets on the device
# ---------------------------------------------------------------------------
def spectrum_dia(s):
    """(data[ndiag, npix], offsets[ndiag]) of a redrock Spectrum's R."""
    npix = len(s.wave)
    R = getattr(s, "R", None)
    if R is None and getattr(s, "_mpshared", False):
        return np.asarray(s.R_data)[:, :npix], np.asarray(s.R_offsets)
    if R is None:
        R = getattr(s, "_Rcsr", None)
    if R is None:
        raise ValueError("spectrum has no resolution matrix")
    if not hasattr(R, "offsets"):
        R = R.todia()
    return np.asarray(R.data)[:, :npix], np.asarray(R.offsets)


class TargetBatch:
    """Host side of a target batch: the descriptors and the concatenated raw
    arrays (DIA resolution data, offsets, ivar, flux) that rr_pack_targets
    reads.  Building it is plain host data preparation (no arithmetic)."""

    def __init__(self, targets, layout):
        self.layout = layout
        self.ntarget = len(targets)
        self.nblock = max(1, (self.ntarget + _lib.LANES - 1) // _lib.LANES)
        # segments: one per (grid, spectrum slot)
        slots = [0] * len(layout.keys)
        per_target = []
        for t in targets:
            count = [0] * len(layout.keys)
            assign = []
            for s in t.spectra:
                g = layout.index[s.wavehash]
                assign.append((g, count[g]))
                count[g] += 1
            slots = [max(a, b) for a, b in zip(slots, count)]
            per_target.append(assign)
        segs = []
        seg_index = {}
        rw_off = 0
        for g in range(len(layout.keys)):
            for sl in range(slots[g]):
                seg_index[(g, sl)] = len(segs)
                segs.append(_lib.SegmentDesc(layout.npix_pad[g], layout.pix_offset[g], rw_off))
                rw_off += layout.npix_pad[g]
        if len(segs) > 16:
            raise NotImplementedError(f"{len(segs)} spectrum slots per target > 16")
        self.segs = segs
        self.npix_block = max(rw_off, 1)
        descs, rdata, roffs, ivar, flux = [], [], [], [], []
        first = [0]
        data_off = pix_off = diag_off = 0
        for it, (t, assign) in enumerate(zip(targets, per_target)):
            blk, lane = divmod(it, _lib.LANES)
            for s, (g, sl) in zip(t.spectra, assign):
                d, o = spectrum_dia(s)
                npix = len(s.wave)
                if npix != layout.npix[g]:
                    raise ValueError("spectrum length does not match its wavelength grid")
                wide = np.abs(o) > _lib.HALF_BAND
                if np.any(wide) and np.any(d[wide] != 0):
                    raise NotImplementedError("resolution bandwidth > 5 pixels is not supported")
                descs.append(_lib.SpectrumDesc(npix, data_off, pix_off, d.shape[0], diag_off, blk,
                                               lane, seg_index[(g, sl)], 0))
                rdata.append(d)
                roffs.append(o)
                ivar.append(s.ivar)
                flux.append(s.flux)
                data_off += d.size
                pix_off += npix
                diag_off += d.shape[0]
            first.append(len(descs))
        self.nspec = len(descs)
        self.descs = struct_bytes(descs)
        self.segs_bytes = struct_bytes(segs)
        self.first = np.asarray(first, dtype=np.int64)
        self.rows = np.full(self.nblock * _lib.LANES, -1, dtype=np.int32)
        self.rows[:self.ntarget] = np.arange(self.ntarget, dtype=np.int32)
        # the large arrays are gathered straight into pinned host memory (when
        # a GPU is present), so their upload needs no second staging copy
        self._pinned = {}
        self.rdata = _concat([np.asarray(d, dtype=np.float64).ravel() for d in rdata], np.float64,
                             self._pinned, "rdata")
        self.roffs = _concat([np.asarray(o, dtype=np.int32) for o in roffs], np.int32)
        self.ivar = _concat([np.asarray(v, dtype=np.float64) for v in ivar], np.float64,
                            self._pinned, "ivar")
        self.flux = _concat([np.asarray(v, dtype=np.float64) for v in flux], np.float64,
                            self._pinned, "flux")

    def host_arrays(self):
        return (self.descs, self.segs_bytes, self.first, self.rows, self.rdata, self.roffs,
                self.ivar, self.flux)

    @property
    def nbytes(self):
        return sum(a.nbytes for a in self.host_arrays())

    def to_device(self):
        return DeviceTargetBatch(self)


def _concat(parts, dtype, pinned=None, name=None):
    """Concatenate 1-D arrays; into a pinned host tensor (kept in
    pinned[name]) when pinned is given, the result is >= 1 MB and a GPU is
    present."""
    n = sum(p.size for p in parts)
    if (pinned is not None and n * np.dtype(dtype).itemsize >= (1 << 20)
            and torch.cuda.is_available()):
        t = torch.empty(n, dtype=torch.from_numpy(np.empty(0, dtype=dtype)).dtype,
                        pin_memory=True)
        pinned[name] = t
        out = t.numpy()
    else:
        out = np.empty(n, dtype=dtype)
    i = 0
    for p in parts:
        out[i:i + p.size] = p
        i += p.size
    return out


class DeviceTargetBatch:
    """The raw arrays of a TargetBatch resident on the device."""

    def __init__(self, batch):
        self.batch = batch
        self.descs = to_device(batch.descs, torch.uint8)
        self.segs = to_device(batch.segs_bytes, torch.uint8)
        self.first = to_device(batch.first, torch.int64)
        self.rows = to_device(batch.rows, torch.int32)
        pinned = getattr(batch, "_pinned", {})
        dev = device()

        def up(name, arr, dtype=torch.float64):
            t = pinned.get(name)
            return t.to(dev, non_blocking=True) if t is not None else to_device(arr, dtype)
        self.rdata = up("rdata", batch.rdata)
        self.roffs = to_device(batch.roffs, torch.int32)
        self.ivar = up("ivar", batch.ivar)
        self.flux = up("flux", batch.flux)


class TargetPack:
    """Targets packed for the fused scan (rr_pack_targets)."""

    def __init__(self, dbatch, stream=None, status=None):
        L = _lib.lib()
        dev = device()
        b = dbatch.batch
        self.layout = b.layout
        self.ntarget = b.ntarget
        self.nblock = b.nblock
        self.segs = b.segs
        self.npix_block = b.npix_block
        self.rows = dbatch.rows
        self.rw = torch.zeros((b.nblock, b.npix_block, _lib.RW, _lib.LANES), dtype=torch.float64,
                              device=dev)
        self.fwf = torch.zeros(b.nblock * _lib.LANES, dtype=torch.float64, device=dev)
        self.wsum = torch.zeros(b.nblock * _lib.LANES, dtype=torch.float64, device=dev)
        self._status = status or StatusWord(dev)
        if b.nspec:
            rc = L.rr_pack_targets(ptr(dbatch.descs), b.nspec, ptr(dbatch.first), b.ntarget,
                                   ptr(dbatch.rdata), ptr(dbatch.roffs), ptr(dbatch.ivar),
                                   ptr(dbatch.flux), ptr(dbatch.segs), len(b.segs), b.npix_block,
                                   b.nblock, ptr(self.rw), ptr(self.fwf), ptr(self.wsum),
                                   self._status.ptr, stream_handle(stream))
            _lib.check(rc, "rr_pack_targets")

    @classmethod
    def from_targets(cls, targets, layout, stream=None):
        return cls(TargetBatch(targets, layout).to_device(), stream=stream)

    def check(self):
        self._status.check("rr_pack_targets")

    def scan_targets_struct(self):
        # one segment array per pack: every struct handed out points at it,
        # so it must outlive all of them
        if getattr(self, "_segarr", None) is None:
            self._segarr = (_lib.SegmentDesc * len(self.segs))(*self.segs)
        arr = self._segarr
        return _lib.ScanTargets(ptr(self.rw), ptr(self.fwf), ptr(self.wsum), ptr(self.rows),
                                ctypes.cast(arr, ctypes.c_void_p).value, self.nblock,
                                len(self.segs), self.npix_block)


class ScanResult:
    def __init__(self, ntarget, basis, dev):
        self.zchi2 = torch.empty((ntarget, basis.nz), dtype=torch.float64, device=dev)
        self.zcoeff = torch.empty((ntarget, basis.nz, basis.nbasis), dtype=torch.float64,
                                  device=dev)
        self.penalty = torch.zeros((ntarget, basis.nz), dtype=torch.float64, device=dev)


class YGemm:
    """y = Tb^T W f of every (target, z) on the tensor cores: G = R^T W f of
    a target pack (rr_pack_g) and, per template, Y = G^T . basis.
    variant: "int8x6" / "int8x7" (exact Ozaki schemes of six base-256 or
    seven base-128 digits; rr_slice_g_i8 once here, the basis digits cached
    on the DeviceBasis, rr_ygemm_i8), or the FP32-accumulated "bf16x3" /
    "tf32x3" (rr_ygemm)."""

    def __init__(self, pack, variant, stream=None, status=None):
        L = _lib.lib()
        dev = device()
        if variant not in _lib.YGEMM_VARIANTS or variant == "fp64":
            raise ValueError(f"unknown tensor-core y variant {variant!r}")
        self.variant = _lib.YGEMM_VARIANTS[variant]
        self.layout = pack.layout
        self.npos = round_up(pack.nblock * _lib.LANES, 128)
        self.kpad = int(L.rr_ygemm_kpad(pack.layout.pix_stride))
        self.g = torch.empty((self.kpad, self.npos), dtype=torch.float64, device=dev)
        exact = self.variant in _lib.I8_VARIANTS
        self.row_exp = torch.empty(self.npos, dtype=torch.int32, device=dev) if exact else None
        self._status = status or StatusWord(dev)
        tgs = pack.scan_targets_struct()
        sh = stream_handle(stream)
        rc = L.rr_pack_g(ctypes.byref(tgs), pack.layout.pix_stride, self.kpad, self.npos,
                         ptr(self.g), ptr(self.row_exp), self._status.ptr, sh)
        _lib.check(rc, "rr_pack_g")
        self.g_digits = None
        if exact:
            nbytes = int(L.rr_ygemm_i8_g_bytes(self.variant, self.npos, self.kpad))
            self.g_digits = torch.empty(nbytes, dtype=torch.uint8, device=dev)
            rc = L.rr_slice_g_i8(self.variant, ptr(self.g), ptr(self.row_exp), self.npos,
                                 self.kpad, ptr(self.g_digits), sh)
            _lib.check(rc, "rr_slice_g_i8")

    def y(self, basis, stream=None):
        """[npos][nz][nbasis] y of every packed target against one basis."""
        L = _lib.lib()
        sh = stream_handle(stream)
        y = torch.empty((self.npos, basis.nz, basis.nbasis), dtype=torch.float64,
                        device=self.g.device)
        if self.variant in _lib.I8_VARIANTS:
            digits, col = basis.i8_digits(self.kpad, stream, self.variant)
            rc = L.rr_ygemm_i8(self.variant, ptr(self.g_digits), ptr(self.row_exp), self.npos,
                               self.kpad, ptr(digits), ptr(col), basis.nz, basis.nbasis, ptr(y),
                               self._status.ptr, sh)
            _lib.check(rc, "rr_ygemm_i8")
        else:
            rc = L.rr_ygemm(self.variant, ptr(self.g), self.npos, self.kpad, ptr(basis.basis),
                            basis.nz, basis.layout.pix_stride, basis.nbasis, basis.stride,
                            ptr(y), self._status.ptr, sh)
            _lib.check(rc, "rr_ygemm")
        return y


# y = Tb^T W f of the fused scan: "int8x6" (tensor-core GEMM, exact integer
# accumulation of six base-256 digit planes; the fastest), "int8x7" (seven
# base-128 planes: one bit more, 1.6x the GEMM time), "fp64" (summed inside
# the scan), or the FP32-accumulated "bf16x3" / "tf32x3" (precision-study
# variants: they miss |dchi2| <= 1e-3 at DESI S/N)
DEFAULT_Y = "int8x6"


def resolve_y(ygemm, layout):
    """The y variant actually used: the default unless given; an INT8
    scheme beyond its exact int32 pixel limit falls back to int8x7 (K <=
    65536), then to fp64."""
    v = DEFAULT_Y if ygemm is None else ygemm
    L = _lib.lib()
    kpad = int(L.rr_ygemm_kpad(layout.pix_stride))
    if v == "int8x6" and kpad > int(L.rr_ygemm_i8_max_kpad(_lib.RR_YGEMM_INT8X6)):
        v = "int8x7"
    if v == "int8x7" and kpad > int(L.rr_ygemm_i8_max_kpad(_lib.RR_YGEMM_INT8X7)):
        v = "fp64"
    return v


def _record(ev, stream):
    if isinstance(stream, torch.cuda.Stream):
        ev.record(stream)
    else:
        ev.record()


def run_fused(pack, bases, stream=None, status=None, ygemm=None, kernel_events=None,
              tiles=None, external_events=False):
    """One persistent launch over every (target, template, z).  ygemm:
    None (DEFAULT_Y), "fp64", "int8x6", "int8x7", "bf16x3" or "tf32x3"; other than
    "fp64", y is computed on the tensor cores first (YGemm).  kernel_events:
    a list that gets a (start, end) CUDA event pair around the scan launches
    alone (timing).  tiles: redshifts per thread {nbasis: ZT} for the small
    bases (nbasis 4: 1-3, nbasis 5: 1-2; rr_scan_options) and optionally
    "block_group" (the tile order), else the defaults."""
    L = _lib.lib()
    dev = device()
    results = [ScanResult(pack.ntarget, b, dev) for b in bases]
    tgs = pack.scan_targets_struct()
    counter = torch.zeros(_lib.FUSED_COUNTERS, dtype=torch.int32, device=dev)
    st = status or StatusWord(dev)
    ygemm = resolve_y(ygemm, pack.layout)
    yg = None if ygemm == "fp64" else YGemm(pack, ygemm, stream=stream, status=st)
    for i0 in range(0, len(bases), _lib.MAX_TEMPLATES):
        chunk = list(range(i0, min(len(bases), i0 + _lib.MAX_TEMPLATES)))
        tms = []
        for i in chunk:
            b, r = bases[i], results[i]
            if b.layout.signature != pack.layout.signature:
                raise ValueError("template basis and targets use different wavelength grids")
            if yg is not None:
                # kept with the result so it outlives the launch
                r.y_ext = yg.y(b, stream=stream)
            tms.append(_lib.ScanTemplate(ptr(b.basis), b.layout.pix_stride, b.nz, b.nbasis,
                                         b.stride, b.method, ptr(b.prior), ptr(b.oii),
                                         ptr(r.zchi2), ptr(r.zcoeff),
                                         ptr(r.penalty) if b.oii is not None else None,
                                         ptr(r.y_ext) if yg is not None else None))
        arr = (_lib.ScanTemplate * len(tms))(*tms)
        if kernel_events is not None:
            # external events become event-record nodes when the launches
            # are captured in a CUDA graph, so each replay times them
            e0 = torch.cuda.Event(enable_timing=True, external=external_events)
            e1 = torch.cuda.Event(enable_timing=True, external=external_events)
            _record(e0, stream)
        if tiles:
            opt = _lib.ScanOptions(int(tiles.get(4, 0)), int(tiles.get(5, 0)),
                                   int(tiles.get("block_group", 0)))
            rc = L.rr_zscan_fused_opt(ctypes.byref(tgs), arr, len(tms), ptr(counter),
                                      ctypes.byref(opt), st.ptr, stream_handle(stream))
        else:
            rc = L.rr_zscan_fused(ctypes.byref(tgs), arr, len(tms), ptr(counter), st.ptr,
                                  stream_handle(stream))
        _lib.check(rc, "rr_zscan_fused")
        if kernel_events is not None:
            _record(e1, stream)
            kernel_events.append((e0, e1))
    run_fused.last_counter = counter
    return results, st


# ---------------------------------------------------------------------------
# pair scan: arbitrary (target, z) pairs, template rebinned on the fly
# ---------------------------------------------------------------------------
class RowPack:
    """Targets packed target-major for the pair scan (rr_pack_rows)."""

    def __init__(self, dbatch, stream=None, status=None):
        L = _lib.lib()
        dev = device()
        b = dbatch.batch
        self.batch = b
        self.layout = b.layout
        self.ntarget = b.ntarget
        self.npix_row = b.npix_block
        self.rows = torch.zeros((b.ntarget, b.npix_block, _lib.RW), dtype=torch.float64, device=dev)
        self.sw = torch.zeros((b.ntarget, b.npix_block), dtype=torch.float64, device=dev)
        self.fwf = torch.zeros(max(b.ntarget, 1), dtype=torch.float64, device=dev)
        self.wsum = torch.zeros(max(b.ntarget, 1), dtype=torch.float64, device=dev)
        self._status = status or StatusWord(dev)
        if b.nspec:
            rc = L.rr_pack_rows(ptr(dbatch.descs), b.nspec, ptr(dbatch.first), b.ntarget,
                                ptr(dbatch.rdata), ptr(dbatch.roffs), ptr(dbatch.ivar),
                                ptr(dbatch.flux), ptr(dbatch.segs), len(b.segs), b.npix_block,
                                ptr(self.rows), ptr(self.sw), ptr(self.fwf), ptr(self.wsum),
                                self._status.ptr, stream_handle(stream))
            _lib.check(rc, "rr_pack_rows")
        # pair segments: one per (grid, slot) segment, with its grid arrays
        self.segments = []
        for sd in b.segs:
            g = self.layout.pix_offset.index(sd.basis_offset)
            e, w, _, _ = self.layout.device_arrays(g)
            self.segments.append(_lib.PairSegment(ptr(e), ptr(w), self.layout.npix[g],
                                                  sd.rw_offset,
                                                  float(np.min(self.layout.waves[g]))))

    @classmethod
    def from_targets(cls, targets, layout, stream=None):
        return cls(TargetBatch(targets, layout).to_device(), stream=stream)

    def check(self):
        self._status.check("rr_pack_rows")


def pair_ranges_ok(src, layout, z):
    """Host check of redrock's rebin range rule (rebin.py:330-341) for each
    redshift: every grid's edges inside [x0 (1+z), x_end (1+z)]."""
    z = np.asarray(z, dtype=np.float64)
    x0 = float(src.x_first)
    x1 = float(src.x_last)
    ok = np.ones(len(z), dtype=bool)
    for i in range(len(layout.keys)):
        _, _, emin, emax = layout.device_arrays(i)
        ok &= ~((emin < x0 * (1 + z)) | (emax > x1 * (1 + z)))
    return ok


def run_pairs(rowpack, src, pair_target, pair_z, stream=None, status=None, bounds=None):
    """chi2 (n,), coeff (n, nbasis), penalty (n,) device tensors for the
    pairs (target index into the packed targets, redshift).  ``bounds``:
    (lower, upper) per basis for a BVLS template (redrock's
    solver_args['bounds']); None is unbounded."""
    L = _lib.lib()
    dev = device()
    n = len(pair_z)
    nb = src.nbasis
    chi2 = torch.empty(n, dtype=torch.float64, device=dev)
    coeff = torch.empty((n, nb), dtype=torch.float64, device=dev)
    pen = torch.zeros(n, dtype=torch.float64, device=dev)
    if n == 0:
        return chi2, coeff, pen
    dt = to_device(np.asarray(pair_target, dtype=np.int32), torch.int32)
    dz = to_device(np.asarray(pair_z, dtype=np.float64))
    oii = src.oii_dev
    prior = None if getattr(src, "prior", None) is None else to_device(src.prior)
    hb = None
    if bounds is not None:
        hb = np.ascontiguousarray(np.broadcast_to(np.asarray(bounds, dtype=np.float64), (2, nb)))
    tm = _lib.PairTemplate(ptr(src.x), src.nx, ptr(src.y), nb, src.igm, src.method, 0,
                           ptr(prior), ptr(oii),
                           None if hb is None else hb.ctypes.data_as(ctypes.c_void_p))
    segs = (_lib.PairSegment * len(rowpack.segments))(*rowpack.segments)
    st = status or StatusWord(dev)
    rc = L.rr_zscan_pairs(ctypes.byref(tm), segs, len(rowpack.segments), ptr(rowpack.rows),
                          ptr(rowpack.fwf), ptr(rowpack.wsum), rowpack.npix_row, ptr(dt), ptr(dz),
                          n, ptr(chi2), ptr(coeff), ptr(pen), st.ptr, stream_handle(stream))
    _lib.check(rc, "rr_zscan_pairs")
    if status is None:
        torch.cuda.current_stream().synchronize()
        st.check("rr_zscan_pairs")
    return chi2, coeff, pen


def run_pairs_device(rowpack, src, pair_target, pair_z, status, stream=None):
    """run_pairs for pairs already on the device (int32 target indices and
    float64 redshifts, both CUDA tensors); stays asynchronous (the caller's
    status word reports kernel errors), so it can be captured in a graph."""
    L = _lib.lib()
    dev = device()
    n = int(pair_z.numel())
    nb = src.nbasis
    chi2 = torch.empty(n, dtype=torch.float64, device=dev)
    coeff = torch.empty((n, nb), dtype=torch.float64, device=dev)
    pen = torch.zeros(n, dtype=torch.float64, device=dev)
    if n == 0:
        return chi2, coeff, pen
    prior = getattr(src, "prior_dev", None)
    tm = _lib.PairTemplate(ptr(src.x), src.nx, ptr(src.y), nb, src.igm, src.method, 0,
                           ptr(prior), ptr(src.oii_dev))
    segs = (_lib.PairSegment * len(rowpack.segments))(*rowpack.segments)
    rc = L.rr_zscan_pairs(ctypes.byref(tm), segs, len(rowpack.segments), ptr(rowpack.rows),
                          ptr(rowpack.fwf), ptr(rowpack.wsum), rowpack.npix_row, ptr(pair_target),
                          ptr(pair_z), n, ptr(chi2), ptr(coeff), ptr(pen), status.ptr,
                          stream_handle(stream))
    _lib.check(rc, "rr_zscan_pairs")
    return chi2, coeff, pen


class FitzCandidates:
    """The K lowest local minima of every target's coarse chi2 (plus
    penalty) and their fine redshift grids, found on the device
    (rr_fitz_candidates): cand [T][K] (-1 past count), count [T], tie [T]
    (rows whose order must come from a host sort), and the pairs
    pair_t / pair_z [T * K * nfine] of every candidate's fine grid."""

    def __init__(self, zchi2, penalty, redshifts, K, nfine, stream=None):
        L = _lib.lib()
        dev = zchi2.device
        T, nz = zchi2.shape
        self.K, self.nfine = K, nfine
        self.cand = torch.empty((T, K), dtype=torch.int32, device=dev)
        self.count = torch.empty(T, dtype=torch.int32, device=dev)
        self.tie = torch.empty(T, dtype=torch.int8, device=dev)
        self.pair_z = torch.empty(T * K * nfine, dtype=torch.float64, device=dev)
        self.pair_t = torch.empty(T * K * nfine, dtype=torch.int32, device=dev)
        rc = L.rr_fitz_candidates(ptr(zchi2), ptr(penalty), T, nz, ptr(redshifts), K, nfine,
                                  ptr(self.cand), ptr(self.count), ptr(self.tie),
                                  ptr(self.pair_z), ptr(self.pair_t), stream_handle(stream))
        _lib.check(rc, "rr_fitz_candidates")


def run_pairs_grad(rowpack, src, pair_target, pair_z, want_dflux=False, stream=None, status=None,
                   dpen=None):
    """chi2, coeff, penalty, dchi2/dz, d2chi2/dz2 (and dchi2/dflux
    [n][npix_row] in the packed pixel order) device tensors for the pairs.
    dpen: a list that receives the d penalty / dz tensor (the [OII]
    penalty's derivative, zero where the penalty is inactive)."""
    L = _lib.lib()
    dev = device()
    n = len(pair_z)
    nb = src.nbasis
    chi2 = torch.empty(n, dtype=torch.float64, device=dev)
    coeff = torch.empty((n, nb), dtype=torch.float64, device=dev)
    pen = torch.zeros(n, dtype=torch.float64, device=dev)
    g = torch.empty(n, dtype=torch.float64, device=dev)
    h = torch.empty(n, dtype=torch.float64, device=dev)
    df = torch.zeros((n, rowpack.npix_row), dtype=torch.float64, device=dev) if want_dflux else None
    dp = torch.zeros(n, dtype=torch.float64, device=dev) if dpen is not None else None
    if dpen is not None:
        dpen.append(dp)
    if n == 0:
        return chi2, coeff, pen, g, h, df
    dt = to_device(np.asarray(pair_target, dtype=np.int32), torch.int32)
    dz = to_device(np.asarray(pair_z, dtype=np.float64))
    oii = src.oii_dev
    tm = _lib.PairTemplate(ptr(src.x), src.nx, ptr(src.y), nb, src.igm, src.method, 0, None,
                           ptr(oii))
    segs = (_lib.PairSegment * len(rowpack.segments))(*rowpack.segments)
    st = status or StatusWord(dev)
    rc = L.rr_zscan_pairs_grad(ctypes.byref(tm), segs, len(rowpack.segments), ptr(rowpack.rows),
                               ptr(rowpack.sw), ptr(rowpack.fwf), ptr(rowpack.wsum),
                               rowpack.npix_row, ptr(dt), ptr(dz), n, ptr(chi2), ptr(coeff),
                               ptr(pen), ptr(g), ptr(h), ptr(df), ptr(dp), st.ptr,
                               stream_handle(stream))
    _lib.check(rc, "rr_zscan_pairs_grad")
    if status is None:
        torch.cuda.current_stream().synchronize()
        st.check("rr_zscan_pairs_grad")
    return chi2, coeff, pen, g, h, df


# ---------------------------------------------------------------------------
# plain per-target path
# ---------------------------------------------------------------------------
class PlainTarget:
    """One target's spectra as band rows for the plain path."""

    def __init__(self, spectra, layout, weights=None, flux=None, wflux=None, stream=None):
        L = _lib.lib()
        dev = device()
        descs, rdata, roffs, pix_basis = [], [], [], []
        data_off = pix_off = diag_off = 0
        for s in spectra:
            g = layout.index[s.wavehash]
            d, o = spectrum_dia(s)
            npix = len(s.wave)
            if np.any(np.abs(o) > _lib.HALF_BAND) and np.any(d[np.abs(o) > _lib.HALF_BAND] != 0):
                raise NotImplementedError("resolution bandwidth > 5 pixels is not supported")
            d = np.ascontiguousarray(d, dtype=np.float64)
            descs.append(_lib.SpectrumDesc(npix, data_off, pix_off, d.shape[0], diag_off, 0, 0, 0,
                                           0))
            rdata.append(d.ravel())
            roffs.append(np.asarray(o, dtype=np.int32))
            pix_basis.append(layout.pix_offset[g] + np.arange(npix, dtype=np.int64))
            data_off += d.size
            pix_off += npix
            diag_off += d.shape[0]
        self.npix = pix_off
        if weights is None:
            weights = np.concatenate([s.ivar for s in spectra])
            flux = np.concatenate([s.flux for s in spectra])
            wflux = weights * flux
        self.w = to_device(weights)
        self.flux = to_device(flux)
        self.wflux = to_device(wflux)
        self.pix_basis = to_device(np.concatenate(pix_basis), torch.int64)
        self.band = torch.empty((self.npix, 2 * _lib.HALF_BAND + 1), dtype=torch.float64,
                                device=dev)
        dspecs = to_device(struct_bytes(descs), torch.uint8)
        # gathered once, straight into pinned memory, for the upload
        pinned = {}
        hrdata = _concat(rdata, np.float64, pinned, "rdata")
        t = pinned.get("rdata")
        drdata = t.to(dev, non_blocking=True) if t is not None else to_device(hrdata)
        droff = to_device(np.concatenate(roffs), torch.int32)
        st = StatusWord(dev)
        rc = L.rr_pack_band_rows(ptr(dspecs), len(descs), ptr(drdata), ptr(droff), self.npix,
                                 ptr(self.band), st.ptr, stream_handle(stream))
        _lib.check(rc, "rr_pack_band_rows")
        self._keep = (dspecs, drdata, droff, pinned)
        self._status = st


_plain_ws = {}


def run_plain(pt, basis, prior=None, method=_lib.RR_SOLVE_PCA, stream=None, bounds=None):
    """zchi2 (nz,), zcoeff (nz, nb) device tensors for one target.  bounds:
    (lower, upper) of RR_SOLVE_BVLS (scalars or nbasis arrays), else
    (-inf, inf)."""
    L = _lib.lib()
    dev = device()
    nz, nb = basis.nz, basis.nbasis
    zchi2 = torch.empty(nz, dtype=torch.float64, device=dev)
    zcoeff = torch.empty((nz, nb), dtype=torch.float64, device=dev)
    need = int(L.rr_zchi2_batch_plain_workspace_bytes(pt.npix, nz, nb))
    ws = _plain_ws.get(dev.index)
    if ws is None or ws.numel() < need:
        ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)
        _plain_ws[dev.index] = ws
    dprior = None if prior is None else to_device(prior)
    hb = None
    if bounds is not None:
        hb = np.ascontiguousarray(np.stack([np.broadcast_to(np.asarray(bounds[0], np.float64), (nb,)),
                                            np.broadcast_to(np.asarray(bounds[1], np.float64), (nb,))]))
    rc = L.rr_zchi2_batch_plain_ex(ptr(pt.band), ptr(pt.w), ptr(pt.wflux), ptr(pt.flux),
                                   ptr(pt.pix_basis), pt.npix, ptr(basis.basis),
                                   basis.layout.pix_stride, nz, nb, basis.stride, ptr(dprior),
                                   method, None if hb is None else hb.ctypes.data, ptr(zchi2),
                                   ptr(zcoeff), ptr(ws), ws.numel(), pt._status.ptr,
                                   stream_handle(stream))
    _lib.check(rc, "rr_zchi2_batch_plain_ex")
    return zchi2, zcoeff


# ---------------------------------------------------------------------------
# small LRU caches keyed by object identity
# ---------------------------------------------------------------------------
class IdCache:
    """LRU cache whose entries are valid while the same objects (by
    identity) are passed again.  Identity says nothing about contents: a
    caller that changes a cached object's arrays in place (a target's flux
    or ivar, say) must clear the cache (``redrock_b200.zscan.clear_caches``)
    before the next call, or it gets the results of the old contents."""

    def __init__(self, size=8):
        self.size = size
        self.d = OrderedDict()

    def get(self, key, objs, make):
        hit = self.d.get(key)
        if hit is not None and all(a is b for a, b in zip(hit[0], objs)) and len(hit[0]) == len(objs):
            self.d.move_to_end(key)
            return hit[1]
        val = make()
        self.d[key] = (list(objs), val)
        self.d.move_to_end(key)
        while len(self.d) > self.size:
            self.d.popitem(last=False)
        return val

    def clear(self):
        self.d.clear()
