"""GPU covariance post-processing (lya_covariance, lya_covariance_smooth)
against the oracle's restatement of post_processing.py:30-91, itself pinned to
the reference's own functions (test_postproc_oracle.py).  Tolerance: 1e-12 of
the largest entry (the Gram matrix sums the pixels in another order)."""
import os

import numpy as np
import pytest

from lya2pcf_b200 import covariance as LC
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import postproc as P

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'cov_golden.npz'))


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_golden_cases():
    c, m = LC.cov(G['a_xi'], G['a_we'])
    assert rel(c, G['a_cov']) < 1e-12 and rel(m, G['a_mean']) < 1e-12
    rp, rt = LC.bin_coordinates(5, 5)
    assert rel(LC.cov_smooth(G['a_xi'], G['a_we'], rp, rt, c), G['a_cov_smooth']) < 1e-12
    c, m = LC.cov(G['b_xi'], G['b_we'])
    rp, rt = LC.bin_coordinates(4, 4)
    cs = LC.cov_smooth(G['b_xi'], G['b_we'], rp, rt, c)
    assert rel(c, G['b_cov']) < 1e-12
    assert np.array_equal(cs, c)          # a zero variance: the unsmoothed covariance
    with pytest.raises(ZeroDivisionError):
        LC.cov(G['d_xi'], G['d_we'], numpix=(3, 3))


def test_full_size_matches_oracle():
    """676 owner pixels x 2500 bins, the size of the 150,000-forest run."""
    rng = np.random.default_rng(3)
    we = rng.uniform(0.0, 5.0, (676, 2500)) * (rng.uniform(size=(676, 2500)) > 0.05)
    xi = rng.normal(0.0, 0.1, (676, 2500)) * (we > 0)
    c, m = LC.cov(xi, we)
    co, mo = P.cov(xi, we)
    assert rel(c, co) < 1e-12 and rel(m, mo) < 1e-12
    rp, rt = LC.bin_coordinates(50, 50)
    assert rel(LC.cov_smooth(xi, we, rp, rt, c), P.cov_smooth(xi, we, rp, rt, co)) < 1e-12


def test_from_correlation_run_on_device():
    """The rows taken on the device from the last run's per-slot histograms
    equal the reading loop of post_processing.py applied to the same
    histograms."""
    fs = synthetic.make(0)
    with PairEngine(np_=10, nt=10) as eng:      # 20 Mpc/h bins: every bin has pairs
        eng.upload(fs)
        eng.build_pairs(synthetic.angmax_for(fs))
        eng.run()
        h, c = eng.histograms()
        mean, cov, cs, smoothed = eng.covariance()
    W, DW = h[:, 0], h[:, 1]
    assert (W.sum(axis=0) > 0).all()
    xi = np.divide(DW, W, out=np.zeros_like(DW), where=W != 0)
    co, mo = P.cov(xi, W)
    assert rel(cov, co) < 1e-12 and rel(mean, mo) < 1e-12
    rp, rt = P.bin_coordinates(10, 10)
    assert smoothed
    assert rel(cs, P.cov_smooth(xi, W, rp, rt, co)) < 1e-12


def test_empty_bin_of_a_run_is_an_error():
    """With 4 Mpc/h bins a 2,000-forest patch leaves some small-r_perp bins
    empty: like the reference's cov, the library refuses (ZeroDivisionError
    there, LYA_ERR_DATA here) unless every bin has weight."""
    from lya2pcf_b200 import _native as N
    fs = synthetic.make(0, scale=0.2)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(synthetic.angmax_for(fs))
        eng.run()
        h, c = eng.histograms()
        empty = (h[:, 0].sum(axis=0) == 0).any()
        if empty:
            with pytest.raises(N.LyaError) as e:
                eng.covariance()
            assert e.value.code == 5
        else:
            eng.covariance()


def test_dropin_post_processing_writes_reference_outputs(tmp_path):
    from lya2pcf_b200.dropin_path import ensure_on_path
    ensure_on_path()
    import importlib
    pp = importlib.import_module('post_processing')
    rng = np.random.default_rng(5)
    for pix in range(30):
        w = rng.uniform(0.5, 3.0, (50, 50))
        dw = w * rng.normal(0, 0.2, (50, 50))
        np.save(str(tmp_path / f'2d_histogram_pixel_{pix}.npy'), np.array([w, dw]))
    cdir = str(tmp_path) + '/'
    with pytest.warns(UserWarning):
        pp.main(['--corr-dir', cdir])     # no distortion.npy: no FITS table
    da, we = pp.read_histograms(cdir, (50, 50))
    co, mo = P.cov(da, we)
    rp, rt = P.bin_coordinates(50, 50)
    so = P.cov_smooth(da, we, rp, rt, co)
    assert rel(np.load(cdir + 'covariance_not_smooth.npy'), co) < 1e-12
    assert rel(np.load(cdir + 'covariance.npy'), so) < 1e-12
    assert rel(np.load(cdir + 'correlation_2d.npy').ravel(), mo) < 1e-12
    assert rel(np.load(cdir + 'error_2d.npy').ravel(), np.sqrt(np.diagonal(so))) < 1e-12
