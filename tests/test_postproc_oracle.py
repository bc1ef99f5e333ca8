"""The covariance oracle (oracle/postproc.py) against golden vectors made by
running the reference's own cov / cov_smooth / diag_error / bin_coordinates
(tests/golden/make_cov_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from lya2pcf_b200 import covariance as LC
from oracle import postproc as P

G = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'cov_golden.npz'))


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_bin_coordinates():
    rp, rt = P.bin_coordinates(5, 5)
    assert np.array_equal(rp, G['a_rp']) and np.array_equal(rt, G['a_rt'])
    rp2, rt2 = LC.bin_coordinates(5, 5)
    assert np.array_equal(rp2, rp) and np.array_equal(rt2, rt)


def test_cov_and_smooth_match_reference():
    c, m = P.cov(G['a_xi'], G['a_we'])
    assert rel(c, G['a_cov']) < 1e-12 and rel(m, G['a_mean']) < 1e-12
    rp, rt = P.bin_coordinates(5, 5)
    assert rel(P.cov_smooth(G['a_xi'], G['a_we'], rp, rt, c), G['a_cov_smooth']) < 1e-12


def test_zero_variance_returns_unsmoothed():
    c, m = P.cov(G['b_xi'], G['b_we'])
    rp, rt = P.bin_coordinates(4, 4)
    out = P.cov_smooth(G['b_xi'], G['b_we'], rp, rt, c)
    assert np.array_equal(G['b_cov_smooth'], G['b_cov'])
    assert rel(out, G['b_cov_smooth']) < 1e-12


def test_diag_error_and_zero_weight():
    e, m = P.diag_error(G['c_xi'], G['c_we'])
    assert rel(e, G['c_error']) < 1e-12 and rel(m, G['c_mean']) < 1e-12
    e2, m2 = LC.diag_error(G['c_xi'].copy(), G['c_we'])
    assert rel(e2, G['c_error']) < 1e-12
    assert bool(G['d_raises'])
    with pytest.raises(ZeroDivisionError):
        P.cov(G['d_xi'], G['d_we'])
