"""ctypes binding of the C ABI in include/redrock_b200.h.

The shared library is built in-tree (redrock_b200/librr_b200.so) by
``make -C redrock_b200/csrc`` (``__graft_entry__.build()`` runs it).  There is no fallback: if the library or a
CUDA device is missing, the calls raise.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "librr_b200.so")

RR_OK, RR_EINVAL, RR_ERANGE, RR_ECUDA, RR_ETIMEOUT, RR_ENOTSUP, RR_ESCRATCH = range(7)
RR_IGM_NONE, RR_IGM_CALURA12, RR_IGM_KAMBLE20, RR_IGM_INOUE14 = range(4)
RR_SOLVE_PCA, RR_SOLVE_UNSUPPORTED, RR_SOLVE_NNLS, RR_SOLVE_BVLS = 0, 1, 2, 3
RR_YGEMM_NONE, RR_YGEMM_BF16X3, RR_YGEMM_TF32X3, RR_YGEMM_INT8X7, RR_YGEMM_INT8X6 = range(5)
YGEMM_VARIANTS = {"fp64": RR_YGEMM_NONE, "bf16x3": RR_YGEMM_BF16X3, "tf32x3": RR_YGEMM_TF32X3,
                  "int8x7": RR_YGEMM_INT8X7, "int8x6": RR_YGEMM_INT8X6}
I8_VARIANTS = (RR_YGEMM_INT8X7, RR_YGEMM_INT8X6)
HALF_BAND = 5
LANES = 32
RW = 12
CHUNK = 24   # default; chunk() returns the loaded library's value
MAX_TEMPLATES = 16
MAX_NBASIS = 10
FUSED_COUNTERS = 12   # RR_FUSED_COUNTERS: tile_counter ints of rr_zscan_fused

IGM_CODES = {None: RR_IGM_NONE, "None": RR_IGM_NONE, "Calura12": RR_IGM_CALURA12,
             "Kamble20": RR_IGM_KAMBLE20, "Inoue14": RR_IGM_INOUE14}

c_void_p = ctypes.c_void_p
c_int64 = ctypes.c_int64
c_int32 = ctypes.c_int32
c_int = ctypes.c_int
c_double = ctypes.c_double
c_size_t = ctypes.c_size_t


class GridDesc(ctypes.Structure):
    _fields_ = [("edges", c_void_p), ("wave", c_void_p), ("npix", c_int64),
                ("npix_pad", c_int64), ("pix_offset", c_int64), ("edge_min", c_double),
                ("edge_max", c_double), ("apply_igm", c_int), ("pad_", c_int)]


class SpectrumDesc(ctypes.Structure):
    _fields_ = [("npix", c_int64), ("data_offset", c_int64), ("pix_offset", c_int64),
                ("ndiag", c_int32), ("diag_offset", c_int32), ("block", c_int32),
                ("lane", c_int32), ("segment", c_int32), ("pad_", c_int32)]


class SegmentDesc(ctypes.Structure):
    _fields_ = [("npix_pad", c_int64), ("basis_offset", c_int64), ("rw_offset", c_int64)]


class ScanTemplate(ctypes.Structure):
    _fields_ = [("basis", c_void_p), ("pix_stride", c_int64), ("nz", c_int32),
                ("nbasis", c_int32), ("basis_stride", c_int32), ("method", c_int32),
                ("prior", c_void_p), ("oii", c_void_p), ("zchi2", c_void_p),
                ("zcoeff", c_void_p), ("penalty", c_void_p), ("y_ext", c_void_p)]


class ArchPair(ctypes.Structure):
    _fields_ = [("pix_off", c_int64), ("npix", c_int64), ("arch_off", c_int64),
                ("leg_off", c_int64)]


class CoaddGroup(ctypes.Structure):
    _fields_ = [("npix", c_int64), ("ndiag", c_int32), ("nspec", c_int32), ("first", c_int64),
                ("out_pix", c_int64), ("out_data", c_int64)]


class ScanOptions(ctypes.Structure):
    _fields_ = [("zt_nbasis4", c_int32), ("zt_nbasis5", c_int32), ("block_group", c_int32)]


class ScanTargets(ctypes.Structure):
    _fields_ = [("rw", c_void_p), ("fwf", c_void_p), ("wsum", c_void_p), ("rows", c_void_p),
                ("segs", c_void_p), ("nblock", c_int32), ("nseg", c_int32),
                ("npix_block", c_int64)]


class PairTemplate(ctypes.Structure):
    _fields_ = [("x", c_void_p), ("nx", c_int64), ("y", c_void_p), ("nbasis", c_int32),
                ("igm_model", c_int32), ("method", c_int32), ("pad_", c_int32),
                ("prior", c_void_p), ("oii", c_void_p), ("bounds", c_void_p)]


class PairSegment(ctypes.Structure):
    _fields_ = [("edges", c_void_p), ("wave", c_void_p), ("npix", c_int64),
                ("row_offset", c_int64), ("wave_min", c_double)]


class RRError(RuntimeError):
    def __init__(self, code, what):
        self.code = code
        super().__init__(f"{what}: {status_string(code)} (rr_status {code})")


_lib = None

_SIGNATURES = {
    "rr_version": (c_int, []),
    "rr_scan_chunk": (c_int, []),
    "rr_status_string": (ctypes.c_char_p, [c_int]),
    "rr_last_cuda_error": (c_int, []),
    "rr_trapz_rebin": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                               c_int64, c_double, c_double, c_double, c_double, c_void_p,
                               c_void_p, c_void_p]),
    "rr_igm_transmission": (c_int, [c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                    c_void_p]),
    "rr_build_basis": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64, c_double,
                               c_double, ctypes.POINTER(GridDesc), c_int, c_int, c_int64, c_int,
                               c_void_p, c_void_p, c_void_p]),
    "rr_pack_targets": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_int, c_int64, c_int, c_void_p,
                                c_void_p, c_void_p, c_void_p, c_void_p]),
    "rr_zscan_fused": (c_int, [ctypes.POINTER(ScanTargets), ctypes.POINTER(ScanTemplate), c_int,
                               c_void_p, c_void_p, c_void_p]),
    "rr_zscan_fused_opt": (c_int, [ctypes.POINTER(ScanTargets), ctypes.POINTER(ScanTemplate),
                                   c_int, c_void_p, ctypes.POINTER(ScanOptions), c_void_p,
                                   c_void_p]),
    "rr_pack_rows": (c_int, [c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                             c_void_p, c_void_p, c_int, c_int64, c_void_p, c_void_p, c_void_p,
                             c_void_p, c_void_p, c_void_p]),
    "rr_zscan_pairs_grad": (c_int, [ctypes.POINTER(PairTemplate), ctypes.POINTER(PairSegment),
                                    c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                    c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                    c_void_p]),
    "rr_zscan_pairs": (c_int, [ctypes.POINTER(PairTemplate), ctypes.POINTER(PairSegment), c_int,
                               c_void_p, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_int64,
                               c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "rr_fitz_candidates": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_int32,
                                   c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                   c_void_p]),
    "rr_pack_band_rows": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_int64, c_void_p,
                                  c_void_p, c_void_p]),
    "rr_zchi2_batch_plain_workspace_bytes": (c_size_t, [c_int64, c_int32, c_int32]),
    "rr_zchi2_batch_plain": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                     c_void_p, c_int64, c_int32, c_int32, c_int32, c_void_p,
                                     c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
                                     c_void_p]),
    "rr_zchi2_batch_plain_ex": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                        c_void_p, c_int64, c_int32, c_int32, c_int32, c_void_p,
                                        c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                                        c_void_p, c_void_p]),
    "rr_zchi2_batch_plain_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                             c_int64, c_void_p, c_int64, c_int32, c_int32,
                                             c_int32, c_void_p, c_int32, c_void_p, c_void_p,
                                             c_void_p, c_void_p]),
    "rr_negoii_penalty": (c_int, [c_void_p, c_int64, c_int32, c_void_p, c_void_p, c_void_p]),
    "rr_fma_peak": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p]),
    "rr_coadd": (c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                         c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "rr_coadd_ex": (c_int, [c_void_p, c_int64, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "rr_coadd_cosmics": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_double, c_void_p, c_void_p, c_int64, c_void_p, c_void_p]),
    "rr_archetype_fit_work_bytes": (c_size_t, [c_int64, c_int32, c_int32, c_int32, c_int64]),
    "rr_archetype_fit": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p, c_int64, c_void_p, c_int32, c_void_p, c_int64,
                                 c_void_p, c_int32, c_int32, c_int32, c_void_p, c_int32,
                                 c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "rr_ygemm_kpad": (c_int64, [c_int64]),
    "rr_pack_g": (c_int, [ctypes.POINTER(ScanTargets), c_int64, c_int64, c_int64, c_void_p,
                          c_void_p, c_void_p, c_void_p]),
    "rr_basis_col_exp": (c_int, [c_void_p, c_int64, c_int64, c_int, c_int, c_void_p, c_void_p]),
    "rr_ygemm": (c_int, [c_int, c_void_p, c_int64, c_int64, c_void_p, c_int64, c_int64, c_int,
                         c_int, c_void_p, c_void_p, c_void_p]),
    "rr_ygemm_i8_g_bytes": (c_int64, [c_int, c_int64, c_int64]),
    "rr_ygemm_i8_basis_bytes": (c_int64, [c_int, c_int64, c_int, c_int64]),
    "rr_ygemm_i8_max_kpad": (c_int64, [c_int]),
    "rr_slice_g_i8": (c_int, [c_int, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p]),
    "rr_slice_basis_i8": (c_int, [c_int, c_void_p, c_int64, c_int64, c_int, c_int, c_int64,
                                  c_void_p, c_void_p, c_void_p]),
    "rr_ygemm_i8": (c_int, [c_int, c_void_p, c_void_p, c_int64, c_int64, c_void_p, c_void_p,
                            c_int64, c_int, c_void_p, c_void_p, c_void_p]),
}


def exported_names():
    return list(_SIGNATURES)


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: build it with "
                               "`python -c 'import __graft_entry__ as g; g.build()'` "
                               "or `make -C redrock_b200/csrc`")
        L = ctypes.CDLL(LIBPATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def chunk():
    """Pixels per scan stage of the loaded library (npix_pad granularity)."""
    return int(lib().rr_scan_chunk())


def status_string(code):
    try:
        return lib().rr_status_string(code).decode()
    except Exception:
        return {0: "ok", 1: "invalid argument", 2: "edges must be within input x range",
                3: "CUDA runtime error", 4: "bounded device wait timed out",
                5: "unsupported input",
                6: "request exceeds the fixed scratch of the no-allocation entry point"
                }.get(code, "unknown")


def check(code, what):
    if code == RR_OK:
        return
    if code == RR_ERANGE:
        raise ValueError("edges must be within input x range")
    if code == RR_ECUDA:
        raise RRError(code, f"{what} (cudaError {lib().rr_last_cuda_error()})")
    raise RRError(code, what)
