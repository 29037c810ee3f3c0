"""Details-file I/O (redrock results.py) through redrock_b200.hdf5: the
reader against a file that redrock itself wrote with h5py (when redrock's
test data is present: its install at baseline/_ref, or $REDROCK_PY), and write -> read round trips."""
import os

import numpy as np
import pytest

from tests.conftest import redrock_test_data

REF_H5 = redrock_test_data("rrdetails-test.h5")


@pytest.mark.skipif(REF_H5 is None, reason="redrock's test data not present")
def test_read_redrock_written_details_file():
    from redrock_b200 import hdf5
    from redrock_b200.results import read_zfit, read_zscan, read_zscan_redrock
    f = hdf5.File(REF_H5)
    assert f.keys() == ['targetids', 'zfit', 'zscan']
    assert f['zscan'].keys() == ['GALAXY', 'QSO:::HIZ']
    tids = f['targetids']
    assert tids.dtype == np.int64 and len(tids) == 3
    z = f['zscan/GALAXY/zchi2']
    assert z.shape == (3, 1446) and np.all(np.isfinite(z))
    assert f['zscan/QSO:::HIZ/zcoeff'].shape == (3, 1046, 4)
    t = f[f'zfit/{tids[1]}/zfit']
    assert t.dtype.names[:3] == ('targetid', 'z', 'zerr')
    assert t['coeff'].shape == (6, 10) and t['zz'].shape == (6, 15)
    assert np.all(t['targetid'] == tids[1])
    res = read_zscan_redrock(REF_H5)
    assert set(res) == set(tids.tolist())
    assert np.array_equal(res[tids[2]]['GALAXY']['zchi2'], z[2])
    zs, zfit = read_zscan(REF_H5)
    assert zfit['spectype'].dtype.kind == 'U'
    assert len(zfit['z']) == 18
    sel = read_zfit(REF_H5, select_targetids=tids[0], upper=True)
    assert np.all(sel['TARGETID'] == tids[0])
    for ft in ('GALAXY', 'QSO:::HIZ'):
        assert 'zfit' in zs[tids[0]][ft]


def _fake_results(rng, nt=3):
    zscan = {}
    rows = []
    for i in range(nt):
        tid = 1000 + i
        zscan[tid] = {}
        for ft, nz, nb in (("GALAXY", 40, 10), ("STAR:::K", 7, 5)):
            zscan[tid][ft] = dict(redshifts=np.linspace(0, 1, nz), zchi2=rng.uniform(size=nz),
                                  penalty=rng.uniform(size=nz), zcoeff=rng.normal(size=(nz, nb)))
        for k in range(3):
            rows.append((tid, k))
    n = len(rows)
    zfit = {
        'targetid': np.array([r[0] for r in rows]), 'z': rng.uniform(size=n),
        'zerr': rng.uniform(size=n), 'zwarn': np.zeros(n, dtype=np.int64),
        'chi2': rng.uniform(size=n), 'zz': rng.uniform(size=(n, 15)),
        'zzchi2': rng.uniform(size=(n, 15)), 'coeff': rng.normal(size=(n, 10)),
        'fitmethod': np.array(['PCA'] * n), 'npixels': np.full(n, 7000),
        'spectype': np.array(['GALAXY', 'STAR', 'GALAXY'] * nt, dtype='<U6'),
        'subtype': np.array(['', 'K', ''] * nt, dtype='<U20'),
        'ncoeff': np.array([10, 5, 10] * nt), 'znum': np.array([r[1] for r in rows]),
        'deltachi2': rng.uniform(size=n)}
    return zscan, zfit


def test_write_read_roundtrip(tmp_path):
    from redrock_b200 import hdf5
    from redrock_b200.results import read_zfit, read_zscan, read_zscan_redrock, write_zscan
    rng = np.random.default_rng(3)
    zscan, zfit = _fake_results(rng)
    fn = str(tmp_path / "sub" / "details.h5")
    write_zscan(fn, zscan, zfit)
    f = hdf5.File(fn)
    assert f.keys() == ['targetids', 'zbest', 'zfit', 'zscan']
    zb = f['zbest']
    assert len(zb) == 3 and 'znum' not in zb.dtype.names
    assert zb['chi2'].dtype == np.float32 and zb['zwarn'].dtype == np.int32
    assert zb['spectype'].dtype.kind == 'S'
    res = read_zscan_redrock(fn)
    for tid in zscan:
        for ft in zscan[tid]:
            np.testing.assert_array_equal(res[tid][ft]['zchi2'],
                                          zscan[tid][ft]['zchi2'].astype(np.float32))
            np.testing.assert_array_equal(res[tid][ft]['zcoeff'],
                                          zscan[tid][ft]['zcoeff'].astype(np.float32))
            np.testing.assert_array_equal(res[tid][ft]['redshifts'], zscan[tid][ft]['redshifts'])
    back = read_zfit(fn)
    np.testing.assert_array_equal(back['targetid'], zfit['targetid'])
    np.testing.assert_array_equal(back['z'], zfit['z'])
    np.testing.assert_array_equal(back['coeff'], zfit['coeff'].astype(np.float32))
    assert list(back['spectype']) == list(zfit['spectype'])
    zs, _ = read_zscan(fn, select_targetids=1001)
    assert list(zs) == [1001]
    assert len(zs[1001]['STAR:::K']['zfit']['z']) == 1
    with pytest.raises(FileExistsError):
        open(fn, 'x')
    write_zscan(fn, zscan, zfit, clobber=True)


def test_hdf5_large_group_and_empty(tmp_path):
    from redrock_b200 import hdf5
    tree = {'g': {str(i): np.arange(i % 5) for i in range(600)}, 's': np.float64(2.5),
            'e': np.zeros((0, 3))}
    fn = str(tmp_path / "x.h5")
    hdf5.write_file(fn, tree)
    f = hdf5.File(fn)
    assert len(f['g'].keys()) == 600
    assert f['g'].keys() == sorted(str(i) for i in range(600))
    np.testing.assert_array_equal(f['g/599'], np.arange(4))
    assert f['s'] == 2.5 and f['e'].shape == (0, 3)
    assert 'g/600' not in f


REF_ARCH = redrock_test_data("rrarchetype-galaxy-test.fits")


@pytest.mark.skipif(REF_ARCH is None, reason="redrock's test data not present")
def test_archetype_file_as_redrock_reads_it():
    """Archetype(filename) without astropy gives the arrays redrock's own
    Archetype builds from the same file (redrock run here with
    astropy.io.fits.open served by the FITS reader)."""
    import sys
    from redrock_b200 import fits as F
    from redrock_b200.archetypes import Archetype
    a = Archetype(REF_ARCH)
    assert a._narch == 2 and a.flux.shape == (2, 48860)
    assert a._rrtype == 'GALAXY' and a.version == 'v3.0'
    assert list(a._subtype) == ['LRG_0', 'ELG_1']
    assert list(a.full_type) == ['GALAXY:::LRG_0', 'GALAXY:::ELG_1']
    np.testing.assert_allclose(a.wave[:2], [1228.0701754386, 1228.2701754386])
    before = set(sys.modules)
    from tests.redrock_ref import import_redrock

    class _H:
        def __init__(self, fn):
            self.h = {h.header.get('EXTNAME', ''): h for h in F.read_hdus(fn)}

        def __getitem__(self, k):
            return self.h[k]

        def close(self):
            pass

    from tests.conftest import redrock_dir
    rr = import_redrock(redrock_dir())
    import redrock.archetypes as ra
    old = sys.modules["astropy.io.fits"].open
    ra.fits.open = lambda fn, memmap=False: _H(fn)
    try:
        ref = ra.Archetype(REF_ARCH)
    finally:
        ra.fits.open = old
        # drop redrock and the astropy stand-ins again
        for name in set(sys.modules) - before:
            if name.split(".")[0] in ("redrock", "astropy", "fitsio"):
                del sys.modules[name]
    np.testing.assert_array_equal(a.flux, ref.flux)
    np.testing.assert_array_equal(a.wave, ref.wave)
    assert list(a._subtype) == list(ref._subtype)
    assert list(a._full_type) == list(ref._full_type)
    assert a._rrtype == ref._rrtype and a.version == ref._version
