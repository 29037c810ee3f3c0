"""Drop-in ``transmission_Lyman`` running on the GPU (redrock igm.py:369-439).

Same return conventions: ``None`` when no absorption can occur and
``always_return_array`` is false, a float for scalar z and wavelength, a 1-D
array when one of them is scalar, else a (nz, nwave) array; ValueError for
an unknown model.  numpy results for ``use_gpu=False``, CUDA tensors for
``use_gpu=True``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .device import device, ptr, stream_handle, to_device, to_numpy

LyA_wavelength = 1215.67
igm_models = ('Calura12', 'Kamble20', 'Inoue14', 'None', None)


def transmission_Lyman(zObj, lObs, use_gpu=False, model='Calura12', always_return_array=True):
    if model not in igm_models:
        raise ValueError(f'Unrecognized model {model}; should be one of {igm_models}')
    if (model == 'None' or model is None) and not always_return_array:
        return None
    zh = to_numpy(zObj)
    lh = to_numpy(lObs)
    min_wave = np.min(lh) / (1. + np.max(zh))
    if min_wave > LyA_wavelength and not always_return_array:
        return None
    scalar_z = np.isscalar(zObj) or (np.ndim(zh) == 0)
    scalar_l = np.isscalar(lObs) or (np.ndim(lh) == 0)
    z = np.atleast_1d(np.asarray(zh, dtype=np.float64))
    lo = np.atleast_1d(np.asarray(lh, dtype=np.float64))
    nz, nw = len(z), len(lo)
    dev = device()
    if always_return_array and (min_wave > LyA_wavelength or model is None or model == 'None'):
        T = torch.ones((nz, nw), dtype=torch.float64, device=dev)
    else:
        T = torch.empty((nz, nw), dtype=torch.float64, device=dev)
        dz = to_device(z)
        dl = to_device(lo)
        rc = _lib.lib().rr_igm_transmission(_lib.IGM_CODES[model], ptr(dz), nz, ptr(dl), nw,
                                            ptr(T), stream_handle())
        _lib.check(rc, "rr_igm_transmission")
    if scalar_z and scalar_l:
        return float(T[0, 0].item())
    if scalar_z:
        T = T[0]
    elif scalar_l:
        T = T[:, 0]
    return T if use_gpu else T.cpu().numpy()
