"""CPU restatement of the reference's covariance post-processing -- test
infrastructure (the checker of the library's lya_covariance), never part of
the product path.

Follows lya2pcf ``post_processing.py``:
  bin_coordinates  post_processing.py:13-28   bin labels 1..np, 1..nt (rp-major)
  cov              post_processing.py:30-52   weighted means and covariance
  cov_smooth       post_processing.py:54-91   correlation averaged over (|drp|, |drt|) steps
  diag_error       post_processing.py:93-109  diagonal errors only

Pinned against golden vectors made by running the reference's own functions
(tests/golden/make_cov_golden.py -> tests/golden/cov_golden.npz).  The sums
run in numpy's order, so results agree with the reference to rounding (the
tests use 1e-12 of the largest entry).
"""
import numpy as np


def bin_coordinates(numpix_r_p, numpix_r_t):
    """post_processing.py:13-28: bin b = (p, t) gets labels (p + 1, t + 1)."""
    rp = np.repeat(np.arange(1, numpix_r_p + 1), numpix_r_t)
    rt = np.tile(np.arange(1, numpix_r_t + 1), numpix_r_p)
    return rp, rt


def cov(xi, weight):
    """post_processing.py:30-52.  xi, weight: [n_pixels, n_bins].  Returns
    (covariance [n_bins, n_bins], means [n_bins]); a bin whose weights sum to
    0 raises ZeroDivisionError, as the reference's numba code does."""
    xi = np.asarray(xi, dtype=np.float64)
    weight = np.asarray(weight, dtype=np.float64)
    W = weight.sum(axis=0)
    if np.any(W == 0.0):
        raise ZeroDivisionError('a bin has zero total weight')
    means = (xi * weight).sum(axis=0) / W
    y = weight * (xi - means)
    c = (y.T @ y) / np.outer(W, W)
    return c, means


def cov_smooth(xi, weight, r_p, r_t, covariance_matrix):
    """post_processing.py:54-91: the correlation matrix averaged over pairs of
    bins with the same (|r_p step|, |r_t step|); the unsmoothed covariance when
    a variance is 0."""
    c = np.asarray(covariance_matrix, dtype=np.float64)
    var = np.diagonal(c)
    if np.any(var == 0.0):
        return c
    norm = np.sqrt(np.outer(var, var))
    corr = c / norm
    n = var.shape[0]
    nbin = int(np.sqrt(len(xi[0])))
    a, b = np.triu_indices(n, 1)
    sp = np.rint(np.abs(np.asarray(r_p)[b] - np.asarray(r_p)[a])).astype(np.int64)
    st = np.rint(np.abs(np.asarray(r_t)[b] - np.asarray(r_t)[a])).astype(np.int64)
    s = np.zeros((nbin, nbin))
    k = np.zeros((nbin, nbin))
    np.add.at(s, (sp, st), corr[a, b])
    np.add.at(k, (sp, st), 1.0)
    sm = np.zeros((n, n))
    sm[a, b] = s[sp, st] / k[sp, st]
    sm[b, a] = sm[a, b]
    sm[np.arange(n), np.arange(n)] = np.diagonal(corr)
    return sm * norm


def diag_error(da, we):
    """post_processing.py:93-109."""
    mda = (da * we).sum(axis=0)
    swe = we.sum(axis=0)
    w = swe > 0.
    mda[w] /= swe[w]
    wda = we * (da - mda)
    error = np.sqrt((wda ** 2).sum(axis=0))
    error[w] /= swe[w]
    return error, mda
