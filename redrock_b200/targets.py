"""Target containers with redrock's interface (redrock 0.22 targets.py).

These mirror the attribute names and behaviour the scan reads from
redrock's own ``Spectrum`` / ``Target`` / ``DistTargetsCopy`` (so the drop-in
functions accept either), for use where redrock itself is not installed.

  Spectrum          targets.py:18-142  (ivar masking by R row integral
                                        :33-35, wavehash :44-53, Rcsr :85-89)
  Target            targets.py:145-265 (gpu_spectral_data :256-263),
                    compute_coadd targets.py:267-373 (redrock_b200.coadd)
  DistTargets       targets.py:390-489 (wavegrids :468-489)
  DistTargetsCopy   targets.py:521-577
  distribute_targets targets.py:492-518, utils.distribute_work utils.py:185-227
"""

from __future__ import annotations

import numpy as np
import scipy.sparse

MIN_RESOLUTION_INTEGRAL = 0.99


class Spectrum:
    def __init__(self, wave, flux, ivar, R, Rcsr=None, band=None):
        if R is not None:
            w = np.asarray(R.sum(axis=1))[:, 0] < MIN_RESOLUTION_INTEGRAL
            ivar[w] = 0.
        self.nwave = wave.size
        self.wave = wave
        self.flux = flux
        self.ivar = ivar
        self.R = R
        self._Rcsr = Rcsr
        self._mpshared = False
        self.band = band
        if band is not None:
            self.wavehash = band
        elif hasattr(R, 'data'):
            self.wavehash = hash((len(wave), wave[0], wave[1], wave[-2], wave[-1],
                                  R.data.shape[0]))
        else:
            self.wavehash = hash((len(wave), wave[0], wave[1], wave[-2], wave[-1]))

    @property
    def Rcsr(self):
        if self._Rcsr is None:
            self._Rcsr = self.R.tocsr()
        return self._Rcsr


class Target:
    def __init__(self, targetid, spectra, coadd=False, cosmics_nsig=0., meta=None):
        self.id = targetid
        self.spectra = spectra
        self.meta = {} if meta is None else meta
        if coadd:
            self.compute_coadd(cache_Rcsr=False, cosmics_nsig=cosmics_nsig)
        self.gpuweights = None
        self.gpuflux = None
        self.gpuwflux = None
        # redrock takes the bands of the spectra given, before any coadd
        self.bands = [s.band for s in spectra]
        self.nleg = 0
        self._legendre = None
        self._gpulegendre = None

    def compute_coadd(self, cache_Rcsr=False, cosmics_nsig=0.):
        """Per-grid coadd of the exposures on the GPU (targets.py:267-373)."""
        from .coadd import coadd_targets
        coadd_targets([self], cache_Rcsr=cache_Rcsr, cosmics_nsig=cosmics_nsig)

    def legendre(self, nleg, use_gpu=False):
        """Legendre polynomials P_0..P_{nleg-1} of each grid's reduced
        wavelength, dict[wavehash] -> (nleg, npix), cached per nleg
        (targets.py:237-254); CUDA tensors when use_gpu."""
        if self._legendre is None or self.nleg != nleg:
            import scipy.special
            dwave = {s.wavehash: s.wave for s in self.spectra}
            self._legendre = {hs: np.array([scipy.special.legendre(i)(reduced_wavelength(w))
                                            for i in range(nleg)]).reshape(nleg, len(w))
                              for hs, w in dwave.items()}
            self._gpulegendre = None
            self.nleg = nleg
        if use_gpu:
            if self._gpulegendre is None:
                from .device import to_device
                self._gpulegendre = {hs: to_device(a) for hs, a in self._legendre.items()}
            return self._gpulegendre
        return self._legendre

    def gpu_spectral_data(self):
        """Concatenated (weights, flux, wflux) as CUDA tensors, cached."""
        if self.gpuweights is None:
            from .device import to_device
            self.gpuweights = to_device(np.concatenate([s.ivar for s in self.spectra]))
            self.gpuflux = to_device(np.concatenate([s.flux for s in self.spectra]))
            self.gpuwflux = self.gpuweights * self.gpuflux
        return (self.gpuweights, self.gpuflux, self.gpuwflux)


def reduced_wavelength(wave):
    """Wavelengths mapped linearly onto [-1, 1] (utils.py:260-271)."""
    wave = np.asarray(wave)
    wavemax = wave.max()
    wavemin = wave.min()
    return 2 * (wave - wavemin) / (wavemax - wavemin) - 1


def distribute_work(nproc, ids, weights=None, capacities=None):
    """Greedy weighted distribution (same assignment rule as redrock's)."""
    if weights is None:
        weights = {x: 1 for x in ids}
    sids = list(sorted(ids, key=lambda x: weights[x], reverse=True))
    if capacities is None:
        capacities = [1] * nproc
    dist = [list() for _ in range(nproc)]
    procs = [dict(id=i, capacity=c, load=0) for i, c in enumerate(capacities)]
    for i_d in sids:
        w = weights[i_d]
        best = min(procs, key=lambda p: ((p['load'] + w) / p['capacity'], 1 / p['capacity'],
                                         p['id']))
        best['load'] += w
        dist[procs.index(best)].append(i_d)
    return dist


def distribute_targets(targets, nproc):
    ids = [t.id for t in targets]
    return distribute_work(nproc, ids, weights={t.id: len(t.spectra) for t in targets})


class DistTargets:
    def __init__(self, targetids, comm=None):
        self._comm = comm
        self._targetids = targetids
        self._dwave = None

    @property
    def comm(self):
        return self._comm

    @property
    def all_target_ids(self):
        return self._targetids

    def local_target_ids(self):
        return self._local_target_ids()

    def local(self):
        return self._local_data()

    def wavegrids(self):
        if self._dwave is None:
            my = {}
            for t in self.local():
                for s in t.spectra:
                    if s.wavehash not in my:
                        my[s.wavehash] = s.wave.copy()
            if self._comm is None:
                self._dwave = my
            else:
                self._dwave = {}
                for part in self._comm.allgather(my):
                    for k, v in part.items():
                        self._dwave.setdefault(k, v.copy())
        return self._dwave


class DistTargetsCopy(DistTargets):
    def __init__(self, targets, comm=None, root=0):
        size = 1 if comm is None else comm.size
        rank = 0 if comm is None else comm.rank
        ids = [t.id for t in targets] if rank == root else []
        if comm is not None:
            ids = comm.bcast(ids, root=root)
        proc = distribute_targets(targets, size)
        self._my_targets = proc[rank]
        if comm is None:
            self._my_data = targets
        else:
            mine = set(self._my_targets)
            buf = {}
            for t in targets:
                r = comm.bcast(t, root=root)
                if r.id in mine:
                    buf[r.id] = r
            self._my_data = [buf[x] for x in self._my_targets]
        super().__init__(ids, comm=comm)

    def _local_target_ids(self):
        return self._my_targets

    def _local_data(self):
        return self._my_data


def from_synth(specs):
    """redrock_b200.synth target specs -> Target objects."""
    out = []
    for t in specs:
        spectra = []
        for s in t.spectra:
            npix = len(s.wave)
            R = scipy.sparse.dia_matrix((s.rdata, s.roffsets), shape=(npix, npix))
            spectra.append(Spectrum(s.wave, s.flux.copy(), s.ivar.copy(), R, band=s.band))
        out.append(Target(t.targetid, spectra))
    return out
