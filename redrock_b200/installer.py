"""Rebind redrock's hot-path names to the GPU drop-ins.

redrock imports several of these functions by name (templates.py:23-24,
fitz.py:15-22, archetypes.py:17-23, zfind.py:32), so replacing the attribute
in its defining module alone would not reach those callers; every module
that holds a reference gets rebound.
"""

from __future__ import annotations

import importlib

# (redrock submodule, attribute) -> (our module, attribute)
PATCHES = {
    ("zscan", "calc_zchi2"): ("zscan", "calc_zchi2"),
    ("zscan", "calc_zchi2_batch"): ("zscan", "calc_zchi2_batch"),
    ("zscan", "calc_zchi2_one"): ("zscan", "calc_zchi2_one"),
    ("rebin", "trapz_rebin"): ("rebin", "trapz_rebin"),
    ("rebin", "rebin_template"): ("rebin", "rebin_template"),
    ("igm", "transmission_Lyman"): ("igm", "transmission_Lyman"),
    ("templates", "rebin_template"): ("rebin", "rebin_template"),
    ("templates", "trapz_rebin"): ("rebin", "trapz_rebin"),
    ("templates", "transmission_Lyman"): ("igm", "transmission_Lyman"),
    ("templates", "DistTemplate"): ("templates", "DistTemplate"),
    ("fitz", "rebin_template"): ("rebin", "rebin_template"),
    ("fitz", "calc_zchi2_one"): ("zscan", "calc_zchi2_one"),
    ("fitz", "calc_zchi2_batch"): ("zscan", "calc_zchi2_batch"),
    ("fitz", "transmission_Lyman"): ("igm", "transmission_Lyman"),
    ("fitz", "fitz"): ("fitz", "fitz"),
    ("zfind", "fitz"): ("fitz", "fitz"),
    ("archetypes", "trapz_rebin"): ("rebin", "trapz_rebin"),
    ("archetypes", "transmission_Lyman"): ("igm", "transmission_Lyman"),
    ("archetypes", "calc_zchi2_batch"): ("zscan", "calc_zchi2_batch"),
    ("archetypes", "per_camera_coeff_with_least_square_batch"):
        ("zscan", "per_camera_coeff_with_least_square_batch"),
    ("zscan", "per_camera_coeff_with_least_square_batch"):
        ("zscan", "per_camera_coeff_with_least_square_batch"),
    ("results", "write_zscan"): ("results", "write_zscan"),
    ("results", "read_zscan"): ("results", "read_zscan"),
    ("results", "read_zfit"): ("results", "read_zfit"),
    ("results", "read_zscan_redrock"): ("results", "read_zscan_redrock"),
    ("zfind", "read_zscan_redrock"): ("results", "read_zscan_redrock"),
}
# methods of redrock classes: (module, class, method) -> (our module, function)
METHOD_PATCHES = {
    ("targets", "Target", "compute_coadd"): ("coadd", "compute_coadd"),
}
FUSED_TARGETS = {
    ("zscan", "calc_zchi2_targets"): ("zscan", "calc_zchi2_targets"),
    ("zfind", "calc_zchi2_targets"): ("zscan", "calc_zchi2_targets"),
}


def install(redrock_pkg=None, fused_targets=True, modules=None):
    """Patch an imported redrock package; returns the list of patched names.

    ``modules`` may map submodule names to module objects (used by tests to
    patch stand-ins); otherwise ``redrock_pkg.<name>`` is imported.
    """
    if redrock_pkg is None and modules is None:
        redrock_pkg = importlib.import_module("redrock")
    table = dict(PATCHES)
    if fused_targets:
        table.update(FUSED_TARGETS)
    done = []
    for (sub, attr), (ours, oattr) in table.items():
        if modules is not None:
            mod = modules.get(sub)
        else:
            try:
                mod = importlib.import_module(f"{redrock_pkg.__name__}.{sub}")
            except Exception:
                mod = None
        if mod is None or not hasattr(mod, attr):
            continue
        src = importlib.import_module(f"redrock_b200.{ours}")
        setattr(mod, attr, getattr(src, oattr))
        done.append(f"{sub}.{attr}")
    for (sub, cls, meth), (ours, oattr) in METHOD_PATCHES.items():
        if modules is not None:
            mod = modules.get(sub)
        else:
            try:
                mod = importlib.import_module(f"{redrock_pkg.__name__}.{sub}")
            except Exception:
                mod = None
        klass = getattr(mod, cls, None) if mod is not None else None
        if klass is None or not hasattr(klass, meth):
            continue
        src = importlib.import_module(f"redrock_b200.{ours}")
        setattr(klass, meth, getattr(src, oattr))
        done.append(f"{sub}.{cls}.{meth}")
    return done
