"""Host-side logic that needs no GPU: layouts, packing descriptors, the
installer, work distribution."""
import types

import numpy as np
import pytest

from redrock_b200 import _lib, synth
from redrock_b200.engine import GridLayout, TargetBatch, centers2edges, round_up
from redrock_b200.installer import PATCHES, install
from redrock_b200.targets import DistTargetsCopy, distribute_work, from_synth


def test_centers2edges_known():
    assert np.allclose(centers2edges([1, 2, 3]), [0.5, 1.5, 2.5, 3.5])
    assert np.allclose(centers2edges([1, 3, 5]), [0, 2, 4, 6])
    assert np.allclose(centers2edges([1, 3, 4]), [0, 2, 3.5, 4.5])


def test_grid_layout_padding():
    lay = GridLayout.from_dwave(synth.camera_grids())
    assert lay.npix == [2751, 2326, 2881]
    ch = _lib.chunk()
    assert lay.npix_pad == [round_up(n, ch) for n in (2751, 2326, 2881)]
    assert lay.pix_offset[0] == 5
    # each grid owns [offset - 5, offset + npix_pad + 5), end to end
    for i in range(1, 3):
        assert lay.pix_offset[i] - 5 == lay.pix_offset[i - 1] + lay.npix_pad[i - 1] + 5
    assert lay.pix_stride == lay.pix_offset[-1] + lay.npix_pad[-1] + 5
    assert all(p % ch == 0 for p in lay.npix_pad)


def test_target_batch_descriptors():
    tg = from_synth(synth.make_targets(35, seed=1, drop_camera_frac=0.2))
    lay = GridLayout.from_dwave(synth.camera_grids())
    b = TargetBatch(tg, lay)
    assert b.nblock == 2
    assert len(b.segs) == 3
    assert b.npix_block == sum(lay.npix_pad)
    descs = np.frombuffer(b.descs.tobytes(), dtype=np.dtype([
        ("npix", "i8"), ("data_offset", "i8"), ("pix_offset", "i8"), ("ndiag", "i4"),
        ("diag_offset", "i4"), ("block", "i4"), ("lane", "i4"), ("segment", "i4"),
        ("pad", "i4")]))
    assert len(descs) == b.nspec == sum(len(t.spectra) for t in tg)
    assert b.first[-1] == b.nspec and np.all(np.diff(b.first) >= 2)
    assert np.all(descs["ndiag"] == 11)
    assert b.ivar.size == descs["npix"].sum()
    # target i -> (block, lane) = divmod(i, 32)
    tid = np.repeat(np.arange(len(tg)), np.diff(b.first))
    assert np.all(descs["block"] == tid // 32) and np.all(descs["lane"] == tid % 32)
    assert list(b.rows[:35]) == list(range(35)) and np.all(b.rows[35:] == -1)


def test_multi_exposure_segments():
    ut = from_synth([synth.util_target(0.2, 1, 111), synth.util_target(0.3, 2, 222)])
    dw = {s.wavehash: s.wave for t in ut for s in t.spectra}
    lay = GridLayout.from_dwave(dw)
    b = TargetBatch(ut, lay)
    # two exposures per camera -> two slots per grid
    assert len(b.segs) == 4


def test_wide_band_rejected():
    tg = from_synth(synth.make_targets(1, seed=1))
    s = tg[0].spectra[0]
    import scipy.sparse
    n = len(s.wave)
    data = np.ones((13, n)) / 13
    s.R = scipy.sparse.dia_matrix((data, np.arange(-6, 7)), shape=(n, n))
    lay = GridLayout.from_dwave(synth.camera_grids())
    with pytest.raises(NotImplementedError):
        TargetBatch(tg, lay)


def test_spectrum_masks_low_resolution_rows():
    # redrock targets.py:33-35: rows whose R integral < 0.99 get ivar 0
    from redrock_b200.targets import Spectrum
    import scipy.sparse
    n = 20
    d, o = synth.util_R(n)     # not normalised at the edges
    ivar = np.ones(n)
    s = Spectrum(np.arange(n, dtype=float), np.zeros(n), ivar,
                 scipy.sparse.dia_matrix((d, o), shape=(n, n)))
    assert s.ivar[0] == 0 and s.ivar[n // 2] == 1


def test_distribute_work_matches_rule():
    ids = list(range(10))
    w = {i: (i % 3) + 1 for i in ids}
    dist = distribute_work(3, ids, weights=w)
    loads = [sum(w[i] for i in d) for d in dist]
    assert sorted(sum(dist, [])) == ids
    assert max(loads) - min(loads) <= 1
    # capacities: a process with 3x capacity takes ~3x the load
    dist = distribute_work(2, list(range(40)), capacities=[3, 1])
    assert len(dist[0]) == 30 and len(dist[1]) == 10


def test_dist_targets_copy_and_wavegrids():
    tg = from_synth(synth.make_targets(3, seed=2))
    d = DistTargetsCopy(tg)
    assert sorted(d.local_target_ids()) == [t.id for t in tg]
    assert set(d.wavegrids()) == {"b", "r", "z"}


def test_installer_rebinds_every_import_site():
    mods = {}
    for sub, attr in PATCHES:
        mods.setdefault(sub, types.SimpleNamespace())
        setattr(mods[sub], attr, "original")
    mods.setdefault("zfind", types.SimpleNamespace())
    mods["zfind"].calc_zchi2_targets = "original"
    mods["zscan"].calc_zchi2_targets = "original"

    class Target:
        compute_coadd = "original"
    mods["targets"] = types.SimpleNamespace(Target=Target)
    done = install(modules=mods)
    assert len(done) == len(PATCHES) + 3
    assert Target.compute_coadd.__module__ == "redrock_b200.coadd"
    for sub, attr in PATCHES:
        assert callable(getattr(mods[sub], attr))
    assert mods["fitz"].calc_zchi2_batch.__module__ == "redrock_b200.zscan"
    assert mods["templates"].DistTemplate.__module__ == "redrock_b200.templates"


def test_installer_on_unmodified_redrock():
    """install() on the real redrock package (its install at baseline/_ref,
    or $REDROCK_PY) rebinds every listed name in redrock's own modules."""
    import sys
    from tests.conftest import redrock_dir
    from redrock_b200.installer import FUSED_TARGETS, METHOD_PATCHES
    d = redrock_dir()
    if d is None:
        pytest.skip("redrock not installed at baseline/_ref and REDROCK_PY unset")
    before = set(sys.modules)
    path0 = list(sys.path)
    try:
        from tests.redrock_ref import import_redrock, install_table_stubs
        rr = import_redrock(d)
        install_table_stubs()
        import redrock.zfind  # noqa: F401
        own_batch = rr.fitz.calc_zchi2_batch
        done = install(rr)
        assert len(done) == len(PATCHES) + len(FUSED_TARGETS) + len(METHOD_PATCHES)
        assert rr.fitz.calc_zchi2_batch is not own_batch
        assert rr.fitz.calc_zchi2_batch.__module__ == "redrock_b200.zscan"
        assert rr.templates.rebin_template.__module__ == "redrock_b200.rebin"
        assert rr.zfind.calc_zchi2_targets.__module__ == "redrock_b200.zscan"
        assert rr.targets.Target.compute_coadd.__module__ == "redrock_b200.coadd"
    finally:
        for name in set(sys.modules) - before:
            if name.split(".")[0] in ("redrock", "astropy", "fitsio"):
                del sys.modules[name]
        sys.path[:] = path0


def test_flop_model():
    import bench
    # the per-eval flop model at P = 7958 px (GALAXY, QSO, STAR)
    assert round(bench.flops_per_eval(10, 7958)) == 2785853
    assert round(bench.flops_per_eval(4, 7958)) == 923189
    assert round(bench.flops_per_eval(5, 7958)) == 1193802


def test_calc_deltachi2_known_answers():
    # redrock test_zscan.py:101-111 / test_zfind.py
    from redrock_b200.zfind import calc_deltachi2
    chi2 = np.array([1.0, 2.0, 4.0, 8.0])
    z = np.array([3.0, 3.1, 3.2, 3.3])
    zwarn = np.array([0, 0, 0, 0])
    dchi2, _ = calc_deltachi2(chi2, z, zwarn)
    assert np.all(dchi2 == np.array([1, 2, 4, 0.0]))
    z = np.array([3.0, 3.0, 4.0, 4.0])
    dchi2, _ = calc_deltachi2(chi2, z, zwarn)
    assert np.all(dchi2 == np.array([3, 2, 0.0, 0.0]))


def test_deltachi2_fast_path_matches_numpy_loop():
    """calc_deltachi2's float64 path (Python floats) gives the numpy loop's
    bits on random fit sets with close pairs, bad fits and both limits."""
    from redrock_b200 import zfind as Z
    rng = np.random.default_rng(3)
    for it in range(500):
        n = int(rng.integers(1, 12))
        chi2 = rng.uniform(0, 30, n)
        z = rng.uniform(0, 3, n) if it % 2 else np.round(rng.uniform(0, 0.01, n), 4)
        zw = rng.choice([0, 0, 0, 4, 1024, 32], n)
        dl = rng.choice([100.0, 1000.0], n)
        ok = (zw & Z.BADFIT_MASK) == 0
        d2 = np.zeros(n)
        for i in range(n - 1):
            dv = Z._fitz.get_dv(z[i + 1:], z[i])
            ii = (np.abs(dv) > np.minimum(dl[i], dl[i + 1:])) & ok[i + 1:]
            if np.any(ii):
                d2[i] = np.min((chi2[i + 1:] - chi2[i])[ii])
        sz = np.zeros(n, dtype=bool)
        for i in range(n):
            m = np.arange(n) != i
            sz[i] = np.any(ok[m] & (np.abs(chi2[m] - chi2[i]) < Z.MIN_DELTACHI2)
                           & (np.abs(Z._fitz.get_dv(z[m], z[i])) >= np.minimum(dl[i], dl[m])))
        got = Z.calc_deltachi2(chi2, z, zw, dvlimit=dl)
        np.testing.assert_array_equal(got[0], d2)
        np.testing.assert_array_equal(got[1], sz)


def test_find_minima_and_minfit():
    from redrock_b200.fitz import find_minima, minfit
    assert list(find_minima([1, 1, 1, 2, 2, 2])) == [0, 1, 2, 4, 5]
    assert list(find_minima([3, 1, 2, 0, 5])) == [3, 1]
    x = np.array([0.1, 0.2, 0.3])
    x0, xerr, y0, zw = minfit(x, 2.0 + ((x - 0.21) / 0.05) ** 2)
    assert abs(x0 - 0.21) < 1e-12 and abs(xerr - 0.05) < 1e-12 and abs(y0 - 2.0) < 1e-9
    assert zw == 0
    assert minfit(x[:2], x[:2])[3] == 2 ** 10


def test_minfit_batch_matches_minfit():
    """The batched parabola agrees with redrock's polyfit-based minfit on
    fine-grid triples (vertex within 1e-9 in z, same ZWARN bits; chi2 at the
    vertex within polyfit's own cancellation error), and
    degenerate triples (flat, constant HUGE_CHI2, NaN, repeated x) give
    exactly minfit's answer."""
    from redrock_b200.fitz import minfit, minfit_batch
    rng = np.random.default_rng(11)
    xs, ys = [], []
    for it in range(400):
        # fine-grid spacings of the z grids: 2 coarse steps over 14 intervals
        # (STAR: linspace(-0.002, 0.002, 100); GALAXY / QSO: 3e-4 / 5e-4 in ln(1 + z))
        if it % 5 == 0:
            z1 = rng.uniform(-0.002, 0.002)
            h = 2 * 0.004 / 99 / 14
        else:
            z1 = rng.uniform(0.0, 6.0)
            h = 2 * (1 + z1) * rng.uniform(3e-4, 5e-4) / 14
        x = np.array([z1 - h, z1, z1 + h])
        a = rng.uniform(1e5, 1e11) * rng.choice([1, 1, 1, -1])
        zt = z1 + rng.uniform(-1.5, 1.5) * h
        xs.append(x)
        ys.append(rng.uniform(-50, 2e4) + a * (x - zt) ** 2)
    x = np.array([0.5, 0.5 + 4e-5, 0.5 + 8e-5])
    deg = [(x, np.full(3, 9999999.0)), (x, np.array([5.0, 5.0, 5.0])),
           (x, np.array([1.0, np.nan, 2.0])), (np.array([0.5, 0.5, 0.6]), np.array([3.0, 2.0, 4.0])),
           (x, 1.0 + 1e3 * (x - x[0]))]
    for xx, yy in deg:
        xs.append(xx)
        ys.append(yy)
    x0, xerr, y0, zw = minfit_batch(np.array(xs), np.array(ys))
    for i, (xx, yy) in enumerate(zip(xs, ys)):
        r = minfit(xx, yy)
        if i >= 400:
            np.testing.assert_array_equal([x0[i], xerr[i], y0[i], zw[i]], r, err_msg=str(i))
            continue
        assert zw[i] == r[3], i
        assert abs(x0[i] - r[0]) <= 1e-9 * max(1.0, abs(r[0])), i
        assert abs(xerr[i] - r[1]) <= 1e-5 * r[1], i
        # polyfit's y0 = c - b^2/4a cancels terms of size a x0^2
        assert abs(y0[i] - r[2]) <= 1e-14 * x0[i] ** 2 / xerr[i] ** 2 + 1e-9 * abs(r[2]), i
    assert all(len(v) == 0 for v in minfit_batch(np.zeros((0, 3)), np.zeros((0, 3))))


def test_prior_functions():
    """priors.py:62-130: Gaussian and Lorentzian terms; the top-hat is 0
    inside |z - z0| < width/2, NaN outside, +inf one point beyond each end
    (or on the end point itself); a target without a prior adds 0."""
    from redrock_b200.priors import Priors
    z = np.linspace(0.0, 1.0, 11)
    p = Priors(targetid=np.array([7]), z=np.array([0.5]), sigma=np.array([0.25]),
               function='gaussian')
    np.testing.assert_allclose(p.eval(7, z), ((z - 0.5) / 0.25) ** 2)
    assert p.eval(8, z) == 0.0
    np.testing.assert_allclose(Priors.lorentzien(z, 0.5, 0.25),
                               -2 * np.log(1 / (1 + ((z - 0.5) / 0.25) ** 2)))
    t = Priors.tophat(z, 0.5, 0.25)
    assert np.isnan(t[:3]).all() and np.isnan(t[8:]).all()
    assert t[3] == np.inf and t[7] == np.inf and (t[4:7] == 0).all()
    t = Priors.tophat(z, 0.0, 0.25)
    assert t[0] == 0 and t[1] == np.inf or t[0] == np.inf
    assert np.isnan(Priors.tophat(z, 5.0, 0.1)).all()


def test_fitz_stack_matches_vstack():
    """fitz's result stacking gives np.vstack's arrays (shape and dtype)."""
    from redrock_b200.fitz import _vstack
    cases = [[1.5, np.float64(2.0)], [1, 2, np.int64(3)], ['PCA', 'PCA'], [np.float64(1)],
             [np.array([1.0, 2.0]), np.array([3.0, 4.0])], [np.zeros((1, 3)), np.ones((1, 3))],
             ['GALAXY:::ELG_0', 'GALAXY:::BGS_12'], [[np.zeros((3, 2))], [np.ones((3, 2))]]]
    for c in cases:
        a, b = _vstack(c), np.vstack(c)
        assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b)


def test_newton_refinement_logic_on_a_model_function(monkeypatch):
    """refine_newton's bracketed Newton/secant iteration, with the pair
    evaluation replaced by an analytic chi2(z) (a quadratic with a cubic
    term, exact gradient, useless kernel curvature): every pair converges to
    its minimum within 1e-4 of its width and the returned curvature is the
    true one."""
    import torch
    import redrock_b200.adjoint as A
    rng = np.random.default_rng(0)
    nt = 200
    zmin = rng.uniform(0.1, 1.0, nt)
    sig = rng.uniform(1e-6, 1e-4, nt)

    def fake(ctx, t, z, want_dflux=False):
        t = np.asarray(t)
        x = (np.asarray(z) - zmin[t]) / sig[t]
        c = x * x + 0.01 * np.abs(x) ** 3
        g = (2 * x + 0.03 * np.abs(x) * x) / sig[t]
        n = len(x)
        return (torch.tensor(c), torch.zeros((n, 3), dtype=torch.float64),
                torch.zeros(n, dtype=torch.float64), torch.tensor(g),
                torch.full((n,), 1e30, dtype=torch.float64), None)

    monkeypatch.setattr(A, "run_pairs_grad",
                        lambda rows, src, t, z, want_dflux=False, dpen=None: fake(None, t, z))
    monkeypatch.setattr(A, "pair_ranges_ok", lambda src, layout, z: np.ones(len(z), bool))
    ctx = types.SimpleNamespace(src=types.SimpleNamespace(nbasis=3), rows=None, layout=None)
    step = 4e-5
    z0 = zmin + rng.uniform(-0.5, 0.5, nt) * step
    z, c, co, g, h, it = A.refine_newton(ctx, np.arange(nt), z0, z0 - step, z0 + step)
    assert it < 24
    assert np.all(np.abs(z - zmin) <= 1e-4 * sig)
    np.testing.assert_allclose(h * sig ** 2 / 2, 1.0, rtol=1e-3)


def test_fitz_column_stacking_matches_per_target_vstack():
    """fitz_targets stacks each result column once over all targets' minima
    and slices it per target: the slices equal a per-target np.vstack
    (values, dtype, shape); a column of mixed types or shapes is left to
    the per-target path."""
    import numpy as np
    from redrock_b200.fitz import _stack_rows, _vstack
    rng = np.random.default_rng(0)
    rows, spans = [], []
    for j in range(40):
        a = len(rows)
        for _ in range(int(rng.integers(1, 4))):
            rows.append(dict(z=float(rng.random()), zerr=float(rng.random()),
                             zwarn=int(rng.integers(0, 5)), chi2=float(rng.random()),
                             zz=rng.random(15), zzchi2=rng.random(15), coeff=rng.random((1, 10)),
                             fitmethod='PCA', npixels=np.int64(7000 + j)))
        spans.append((a, len(rows)))
    cols = {k: _stack_rows([r[k] for r in rows]) for k in rows[0]}
    for a, b in spans:
        for k in rows[0]:
            ref = _vstack([r[k] for r in rows[a:b]])
            got = cols[k][a:b]
            assert got.dtype == ref.dtype and got.shape == ref.shape
            assert np.array_equal(got, ref), k
    assert _stack_rows([np.zeros(10), np.zeros((1, 10))]) is None
    assert _stack_rows([1, 2.0]) is None
    assert _stack_rows(['PCA', 'NMF3']) is None


def test_resolve_y_falls_back_by_pixel_count(monkeypatch):
    """The default tensor-core y scheme (INT8X6) gives way to INT8X7 when the
    padded pixel count is beyond its exact int32 range, and INT8X7 to the
    FP64 sum inside the scan beyond its own; explicit choices are kept."""
    from redrock_b200 import _lib, engine

    class FakeLib:
        kpad = 8064

        def rr_ygemm_kpad(self, pix_stride):
            return self.kpad

        def rr_ygemm_i8_max_kpad(self, variant):
            return {_lib.RR_YGEMM_INT8X6: 21824, _lib.RR_YGEMM_INT8X7: 65536}.get(variant, -1)

    fake = FakeLib()
    monkeypatch.setattr(_lib, "lib", lambda: fake)

    class Layout:
        pix_stride = 0

    assert engine.DEFAULT_Y == "int8x6"
    assert engine.resolve_y(None, Layout) == "int8x6"
    fake.kpad = 21824 + 64
    assert engine.resolve_y(None, Layout) == "int8x7"
    assert engine.resolve_y("int8x6", Layout) == "int8x7"
    fake.kpad = 65536 + 64
    assert engine.resolve_y(None, Layout) == "fp64"
    assert engine.resolve_y("bf16x3", Layout) == "bf16x3"


def test_int8_digit_schemes_reconstruct_exactly():
    """The digit decompositions the INT8 y GEMM slices its operands into
    (restated in numpy): X = rint(x 2^(mant - e)) with e the exponent of
    128/127 max |x| splits into balanced digits that all fit int8 -- seven
    base-128 digits (|digit| <= 64) or six base-256 digits (the leading
    one within +-127 thanks to the margin) -- and the digits sum back to X
    exactly, including values just below the margin and at +-max."""
    import numpy as np
    rng = np.random.default_rng(3)

    def digits(X, nd, bits):
        half, mask = 1 << (bits - 1), (1 << bits) - 1
        out, x = [], X.copy()
        for _ in range(nd - 1):
            a = ((x + half) & mask) - half
            x = (x - a) >> bits
            out.append(a)
        out.append(x)
        return out[::-1]

    for nd, bits, mant, lim in ((7, 7, 48, 64), (6, 8, 47, 127)):
        for trial in range(50):
            x = rng.uniform(-1, 1, 4096) * 10.0 ** rng.uniform(-30, 30)
            m = np.abs(x).max()
            x[:4] = [m, -m, m * (1 - 2.0 ** -40), -m * 127 / 128]
            e = np.frexp(np.abs(x).max() * (128.0 / 127.0))[1]
            X = np.rint(np.ldexp(x, mant - e)).astype(np.int64)
            d = digits(X, nd, bits)
            half = 1 << (bits - 1)
            for di in d[1:]:      # low digits: balanced, [-base/2, base/2)
                assert int(di.min()) >= -half and int(di.max()) < half
            assert int(np.abs(d[0]).max()) <= lim
            assert all(int(di.min()) >= -128 and int(di.max()) <= 127 for di in d)
            rec = sum(di * (1 << (bits * (nd - 1 - k))) for k, di in enumerate(d))
            assert np.array_equal(rec, X)


def _zfit_rows(rng, nmin, nz_fine, nb, npix, tie_chi2=None):
    """One template's fitz result for one target (the columns fitz returns)."""
    import numpy as np
    from redrock_b200 import zfind as ZF
    chi2 = rng.uniform(9000, 9100, nmin)
    if tie_chi2 is not None:
        chi2[:] = tie_chi2
    z = rng.uniform(0, 2, nmin)
    if nmin > 1 and rng.random() < 0.3:
        z[1] = z[0] * (1 + 1e-5)          # within max_velo_diff
        chi2[1] = chi2[0] + 1.0            # and within MIN_DELTACHI2
    zwarn = np.where(rng.random(nmin) < 0.2, ZF.BAD_MINFIT, 0).astype(np.int64)
    return dict(z=z[:, None], zerr=rng.random((nmin, 1)), zwarn=zwarn[:, None],
                chi2=chi2[:, None], zz=rng.random((nmin, nz_fine)),
                zzchi2=rng.random((nmin, nz_fine)), coeff=rng.random((nmin, nb)),
                fitmethod=np.full((nmin, 1), 'PCA'), npixels=np.full((nmin, 1), npix))


def test_batched_zfind_finalisation_matches_per_target():
    """zfind's batched finalisation gives the concatenation of the
    per-target tables (redrock's per-target logic) column for column:
    values, order (stable chi2 order, the nminima-per-spectype cut and the
    re-sort of targets that lose fits, ties included), znum, deltachi2 and
    every ZWARN bit, with NODATA / LITTLE_COVERAGE targets in the batch."""
    import numpy as np
    from redrock_b200 import zfind as ZF
    rng = np.random.default_rng(11)
    fts = ['GALAXY', 'QSO', 'STAR:::A', 'STAR:::F', 'STAR:::K']
    nbs = [10, 4, 5, 5, 5]
    for trial in range(6):
        nminima = 3
        tids = list(range(1000, 1000 + 60))
        fits_list = []
        for i, tid in enumerate(tids):
            npix = 0 if i % 17 == 3 else (30 if i % 13 == 5 else 7000)
            tie = 9050.0 if i % 11 == 2 else None
            fits = []
            for ft, nb in zip(fts, nbs):
                nmin = int(rng.integers(1, 4))
                fits.append((ft, _zfit_rows(rng, nmin, 15, nb, npix, tie)))
            fits_list.append(fits)
        copies = [[(ft, {k: v.copy() for k, v in z.items()}) for ft, z in fits]
                  for fits in fits_list]
        rows = [ZF._finalise_target(tid, fits, nminima) for tid, fits in zip(tids, copies)]
        ref = {k: np.concatenate([r[k] for r in rows], axis=0) for k in rows[0]}
        got = ZF._finalise_batch(tids, fits_list, nminima)
        assert got is not None
        assert list(got) == list(rows[0])
        for k in ref:
            assert got[k].shape == ref[k].shape, k
            assert got[k].dtype.kind == ref[k].dtype.kind, k
            assert np.array_equal(got[k], ref[k]), k
        assert np.any(ref['zwarn'] & ZF.SMALL_DELTA_CHI2)
        assert np.any(ref['zwarn'] & ZF.NODATA) and np.any(ref['zwarn'] & ZF.LITTLE_COVERAGE)
    # a target without minima for a template goes the per-target way
    fits_list[0][1] = (fts[1], _zfit_rows(rng, 0, 15, 4, 7000))
    assert ZF._finalise_batch(tids, fits_list, 3) is None


def test_batched_deltachi2_matches_per_target_loop():
    """The padded all-targets deltachi2 gives the per-target loop's values
    and flags, NaN chi2, bad fits and velocity-limit edges included."""
    import numpy as np
    from redrock_b200 import zfind as ZF
    rng = np.random.default_rng(5)
    n = rng.integers(1, 10, 300)
    first = np.r_[0, np.cumsum(n)[:-1]]
    tot = int(n.sum())
    chi2 = rng.uniform(100, 130, tot)
    chi2[rng.random(tot) < 0.02] = np.nan
    z = rng.uniform(0, 3, tot)
    # pairs at and near the velocity limit
    for a in first[:100]:
        if a + 1 < tot:
            z[a + 1] = z[a] + 1000.0 / ZF._fitz.C_KMS * (1 + z[a]) * rng.choice([0.5, 1.0, 2.0])
    okfit = rng.random(tot) < 0.85
    dl = np.where(rng.random(tot) < 0.5, ZF.MAX_VELO_DIFF, ZF.MAX_VELO_DIFF_STAR).astype(float)
    d_b, s_b = ZF._deltachi2_batch(chi2, z, okfit, dl, first, n)
    for i in range(len(n)):
        a, b = first[i], first[i] + n[i]
        d, sz = ZF._deltachi2_f64(chi2[a:b], z[a:b], okfit[a:b], dl[a:b])
        np.testing.assert_array_equal(d_b[a:b], d)
        np.testing.assert_array_equal(s_b[a:b], sz)


def test_find_minima_definition():
    """fitz's candidate minima: every index whose value is <= both
    neighbours (edges against their one neighbour), ordered by np.argsort
    of the values -- checked against that definition written out directly,
    on rows with plateaus, ties and NaN."""
    import numpy as np
    from redrock_b200.fitz import find_minima
    rng = np.random.default_rng(9)
    assert list(find_minima([1, 1, 1, 2, 2, 2])) == [0, 1, 2, 4, 5]
    assert list(find_minima([3.0])) == [0]
    for _ in range(200):
        x = np.round(rng.normal(size=int(rng.integers(2, 60))), 1)
        if rng.random() < 0.2:
            x[rng.integers(0, len(x))] = np.nan
        n = len(x)
        idx = [i for i in range(n)
               if (i == 0 or x[i] <= x[i - 1]) and (i == n - 1 or x[i] <= x[i + 1])]
        idx = np.array(idx, dtype=np.int64)
        np.testing.assert_array_equal(find_minima(x), idx[np.argsort(x[idx])])


def test_fitz_post_fit_checks_batched(monkeypatch):
    """fitz_targets applies redrock's checks after each parabola fit
    (fitz.py:263-280) to whole batches of candidates: every reported
    minimum equals the scalar sequence -- the parabola through the three
    fine-grid points around the lowest one, BAD_MINFIT and the grid's
    first lowest point when the vertex leaves the fine grid, Z_FITLIMIT
    outside redshifts[1:-1] -- on monotone, constant and regular fine
    grids (a stand-in for the pair scan, no GPU)."""
    import numpy as np
    from redrock_b200 import fitz as F

    class FakeRef:
        def __init__(self, targets, template, layout=None, rowpack=None):
            self.oii = None
            self.src = type("S", (), {"nbasis": template.nbasis})()

        def scan(self, tidx, z):
            z = np.asarray(z, dtype=np.float64)
            t = np.asarray(tidx)
            c = 100 + 1e6 * (z - 0.5 - 0.01 * (t % 7)) ** 2 + 3 * np.sin(z * 3000 + t)
            c = np.where(t % 13 == 4, 100 + 50 * z, c)
            return c, np.ones((len(z), self.src.nbasis)), np.zeros(len(z)), np.ones(len(z), bool)

    monkeypatch.setattr(F, "_Refiner", FakeRef)

    class Tg:
        def __init__(self):
            self.spectra = [type("Sp", (), {"ivar": np.ones(4)})()]

    class Tm:
        nbasis, method, igm_model, solve_matrices_algorithm = 10, 'PCA', None, 'PCA'
        template_type = 'GALAXY'

    zg = np.linspace(-0.005, 1.5, 3311)
    n = 300
    chi2 = [100 + 1e3 * (zg - 0.7 - 0.01 * (i % 7)) ** 2 + 50 * np.sin(zg * (200 + i) + i)
            for i in range(n)]
    chi2[5][:] = 1e10
    out = F.fitz_targets(chi2, zg, [Tg() for _ in range(n)], Tm(), nminima=3)
    checked = 0
    for res in out:
        for m in range(len(res['z'])):
            zz, c2 = res['zz'][m], res['zzchi2'][m]
            i = min(max(int(np.argmin(c2)), 1), len(zz) - 2)
            x0, xerr, y0, zw = (float(v[0]) for v in F.minfit_batch(zz[None, i - 1:i + 2],
                                                                     c2[None, i - 1:i + 2]))
            zw = int(zw)
            zbest, chi2min = x0, y0
            if zbest < zz[0] or zbest > zz[-1]:
                zw |= F.BAD_MINFIT
                k = int(np.where(c2 == np.min(c2))[0][0])
                zbest, chi2min = zz[k], c2[k]
            if zbest < zg[1] or zbest > zg[-2] or x0 < zg[1] or x0 > zg[-2]:
                zw |= F.Z_FITLIMIT
            assert res['z'][m, 0] == zbest and res['chi2'][m, 0] == chi2min
            assert res['zerr'][m, 0] == xerr and res['zwarn'][m, 0] == zw
            checked += 1
    assert checked > 3 * n - 10
    assert any(res['zwarn'][:, 0].any() for res in out)


def test_pipelined_chunk_bounds():
    """The pipelined scan's target chunks: one launch for small batches, else
    a small first chunk and then chunks of the chosen size, covering every
    target exactly once in order."""
    from redrock_b200 import zscan
    assert zscan._chunk_bounds(300, 224) == [(0, 300)]
    for n, chunk in ((500, 224), (5000, 448), (20000, 448), (449, 224), (4097, 448)):
        b = zscan._chunk_bounds(n, chunk)
        assert b[0] == (0, min(zscan.FIRST_CHUNK, chunk))
        assert b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))
        assert all(0 < j - i <= chunk for i, j in b)
