"""Covariance post-processing on the GPU, with the reference's functions.

Same names, arguments and results as lya2pcf ``post_processing.py``:

    bin_coordinates(numpix_r_p, numpix_r_t) -> (r_p, r_t)      post_processing.py:13-28
    cov(xi, weight) -> (covariance_matrix, means)               post_processing.py:30-52
    cov_smooth(xi, weight, r_p, r_t, covariance_matrix)         post_processing.py:54-91
    diag_error(da, we) -> (error, mda)                          post_processing.py:93-109

``cov`` and ``cov_smooth`` run in the native library (``lya_covariance``,
``lya_covariance_smooth``: the weighted Gram matrix on the FP64 tensor cores);
a bin whose weights sum to 0 raises ZeroDivisionError like the reference's
numba code.  ``diag_error`` is a few column sums and stays in numpy.  The bin
layout is the reference's (``bin_coordinates``): ``cov_smooth`` takes r_p, r_t
for the same signature and checks that they are that layout.
"""
import ctypes as C

import numpy as np

from . import _native as N


def bin_coordinates(numpix_r_p, numpix_r_t):
    """Bin labels 1..numpix_r_p and 1..numpix_r_t of every flat bin p*nt + t."""
    rp = np.repeat(np.arange(1, numpix_r_p + 1), numpix_r_t)
    rt = np.tile(np.arange(1, numpix_r_t + 1), numpix_r_p)
    return rp, rt


class _Ctx:
    """A library context with the bin shape of a covariance call."""

    def __init__(self, device, np_, nt):
        self.lib = N.load()
        self.ctx = C.c_void_p()
        N.check(self.lib.lya_ctx_create(int(device), C.byref(self.ctx)))
        N.check(self.lib.lya_set_bins(self.ctx, 200.0, 200.0, int(np_), int(nt)), self.ctx)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.lib.lya_ctx_destroy(self.ctx)


def _shape(n_bins, numpix=None):
    if numpix is not None:
        return int(numpix[0]), int(numpix[1])
    side = int(round(np.sqrt(n_bins)))
    if side * side != n_bins:
        raise ValueError(f'{n_bins} bins are not a square grid: give numpix=(np, nt)')
    return side, side


def cov(xi, weight, device=0, numpix=None):
    """Covariance matrix and weighted means of the per-pixel correlations."""
    xi = np.ascontiguousarray(xi, dtype=np.float64)
    weight = np.ascontiguousarray(weight, dtype=np.float64)
    if xi.shape != weight.shape or xi.ndim != 2:
        raise ValueError('xi and weight must be 2-d arrays of the same shape')
    n, nb = xi.shape
    np_, nt = _shape(nb, numpix)
    mean = np.zeros(nb)
    c = np.zeros((nb, nb))
    with _Ctx(device, np_, nt) as k:
        rc = k.lib.lya_covariance(k.ctx, n, N.ptr(xi), N.ptr(weight), N.ptr(mean), N.ptr(c))
        if rc == 5:   # LYA_ERR_DATA: a bin with zero total weight
            raise ZeroDivisionError(k.lib.lya_last_error(k.ctx).decode())
        N.check(rc, k.ctx)
    return c, mean


def cov_smooth(xi, weight, r_p, r_t, covariance_matrix, device=0, numpix=None):
    """Smoothed covariance: the correlation averaged over equal bin steps."""
    c = np.ascontiguousarray(covariance_matrix, dtype=np.float64)
    nb = c.shape[0]
    np_, nt = _shape(nb, numpix)
    rp0, rt0 = bin_coordinates(np_, nt)
    if not (np.array_equal(np.asarray(r_p), rp0) and np.array_equal(np.asarray(r_t), rt0)):
        raise ValueError('r_p, r_t must be bin_coordinates(numpix_rp, numpix_rt)')
    out = np.zeros_like(c)
    sm = C.c_int32(0)
    with _Ctx(device, np_, nt) as k:
        N.check(k.lib.lya_covariance_smooth(k.ctx, N.ptr(c), N.ptr(out), C.byref(sm)), k.ctx)
    if not sm.value:
        print('WARNING: Data has some empty bins. Returning the unsmoothed covariance')
    return out


def diag_error(da, we):
    """Diagonal errors without the full covariance (post_processing.py:93-109)."""
    mda = (da * we).sum(axis=0)
    swe = we.sum(axis=0)
    w = swe > 0.
    mda[w] /= swe[w]
    wda = we * (da - mda)
    print("Computing errors...")
    error2 = (wda ** 2).sum(axis=0)
    error = np.sqrt(error2)
    error[w] /= swe[w]
    return error, mda
