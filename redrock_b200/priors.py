"""Redshift priors (redrock 0.22 priors.py).

A prior adds a function of (z - z0) / sigma to each target's coarse chi2(z)
of every template before the fine-grid refinement (zfind.py:318-322).  The
per-target (z0, sigma) and the function name come from redrock's prior file
(a FITS table PRIORS with TARGETID, Z, SIGMA, FUNCTION, read with astropy
or, without it, with ``redrock_b200.fits``); they can also be given as
arrays.
"""

from __future__ import annotations

import os

import numpy as np


class Priors:
    """Priors keyed by TARGETID (priors.py:12-60)."""

    def __init__(self, filename=None, targetid=None, z=None, sigma=None, function='gaussian'):
        if filename is not None:
            filename = os.path.expandvars(filename)
            try:
                from astropy.io import fits
                with fits.open(filename, memmap=False) as h:
                    rows = h['PRIORS'].data
                    targetid, z, sigma = rows['TARGETID'], rows['Z'], rows['SIGMA']
                    function = rows['FUNCTION'][0]
            except ImportError:
                from .fits import read_table
                _, rows = read_table(filename, 'PRIORS')
                targetid, z, sigma = rows['TARGETID'], rows['Z'], rows['SIGMA']
                function = rows['FUNCTION'][0]
            if isinstance(function, bytes):
                function = function.decode()
            function = str(function).strip()
        z = np.asarray(z)
        self._param = {targetid[i]: {'Z': z[i], 'SIGMA': sigma[i]} for i in range(z.size)}
        self._type = function
        self._func = getattr(self, self._type)

    def eval(self, targetid, z):
        """Prior term of the chi2 on the redshift grid z (0 for a target
        without a prior)."""
        try:
            z0 = self._param[targetid]['Z']
            s0 = self._param[targetid]['SIGMA']
            return self._func(z, z0, s0)
        except KeyError:
            print(f'targetid {targetid} not in priors')
            return 0.

    @staticmethod
    def gaussian(z, z0, s0):
        return ((z - z0) / s0) ** 2

    @staticmethod
    def lorentzien(z, z0, s0):
        return -2 * np.log(1 / (1. + ((z - z0) / s0) ** 2))

    @staticmethod
    def tophat(z, z0, s0):
        """0 inside |z - z0| < s0/2, NaN outside, and +inf on the grid points
        just beyond either end (or on the end points themselves) so that the
        minima finder never selects a point outside (priors.py:90-130)."""
        prior = np.where(np.abs(z - z0) < s0 / 2, 0., np.nan)
        if np.all(np.isnan(prior)):
            return prior
        inside = np.argwhere(prior >= 0.0)
        left, right = inside[0], inside[-1]
        prior[left if left == 0 else left - 1] = np.inf
        prior[right if right == prior.size - 1 else right + 1] = np.inf
        return prior
