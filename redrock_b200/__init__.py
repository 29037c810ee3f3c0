"""redrock-b200: B200-native redshift-scan engine for redrock.

Drop-in replacements (same signatures and outputs as redrock 0.22):

  redrock_b200.zscan.calc_zchi2, calc_zchi2_targets, calc_zchi2_batch,
      calc_zchi2_one, calc_negOII_penalty, spectral_data
  redrock_b200.rebin.trapz_rebin, rebin_template, centers2edges
  redrock_b200.igm.transmission_Lyman
  redrock_b200.templates.Template, DistTemplate
  redrock_b200.targets.Spectrum, Target, DistTargetsCopy

``redrock_b200.install(redrock)`` rebinds these names inside an imported
redrock package so zfind / fitz use them unchanged.  The compute runs in
librr_b200.so (hand-written sm_100a CUDA behind a C ABI,
include/redrock_b200.h); there is no CPU fallback.
"""

__version__ = "0.1.0"


def install(redrock_pkg=None, **kw):
    from .installer import install as _install
    return _install(redrock_pkg, **kw)
