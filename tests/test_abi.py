"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from redrock_b200 import _lib

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(rr_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_header():
    L = ctypes.CDLL(_lib.LIBPATH)
    decl = declared_functions()
    assert len(decl) >= 12
    missing = [n for n in decl if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers exactly the declared set
    assert set(_lib.exported_names()) == decl


def test_status_strings_without_gpu():
    L = _lib.lib()
    assert L.rr_version() >= 1
    assert L.rr_status_string(2).decode().startswith("edges must be within")
    assert L.rr_status_string(99).decode() == "unknown status"


def test_argument_errors_without_gpu():
    # validation happens before any CUDA call, so these run on a CPU host
    L = _lib.lib()
    assert L.rr_trapz_rebin(None, 1, None, 1, None, 1, None, 1, 0., 0., 0., 0., None, None,
                            None) == _lib.RR_EINVAL
    # range check: edges outside the redshifted range -> RR_ERANGE (ValueError)
    x = (ctypes.c_double * 2)(1.0, 2.0)
    assert L.rr_trapz_rebin(x, 2, x, 1, x, 1, x, 1, 1.5, 1.8, 1.0, 2.0, x, None,
                            None) == _lib.RR_ERANGE
    assert L.rr_igm_transmission(7, None, 1, None, 1, None, None) == _lib.RR_EINVAL
    assert L.rr_zscan_fused(None, None, 0, None, None, None) == _lib.RR_EINVAL
    assert L.rr_zchi2_batch_plain_workspace_bytes(100, 10, 4) > 100 * 10 * 4 * 8
    # a byte count that overflows (or a negative size) reads as SIZE_MAX, so
    # no workspace or scratch size check can pass it
    size_max = 2 ** (8 * ctypes.sizeof(ctypes.c_size_t)) - 1
    assert L.rr_zchi2_batch_plain_workspace_bytes(2 ** 62, 2 ** 30, 10) == size_max
    assert L.rr_zchi2_batch_plain_workspace_bytes(-1, 10, 4) == size_max
    assert L.rr_zchi2_batch_plain_noalloc(None, None, None, None, None, 2 ** 62, None, 8000,
                                          2 ** 30, 10, 10, None, 0, None, None, None,
                                          None) == _lib.RR_ESCRATCH


def test_header_constants_match_binding():
    src = open(os.path.join(ROOT, "include", "redrock_b200.h")).read()
    consts = dict(re.findall(r"#define\s+(RR_[A-Z0-9_]+)\s+(\d+)\b", src))
    assert int(consts["RR_FUSED_COUNTERS"]) == _lib.FUSED_COUNTERS
    assert int(consts["RR_CHUNK"]) == _lib.CHUNK
