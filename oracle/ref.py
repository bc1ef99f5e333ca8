"""ctypes front end of the reference's own CUDA kernels (``oracle/_ref``).
TEST INFRASTRUCTURE ONLY.

``libref_kernels.so`` is ``cuda_kernels.cpp`` from the reference tree compiled
by ``oracle/Makefile`` (target ``ref``) behind ``ref_launch.cu``; it exists only
where the reference tree was available at build time and the file travels with
the repository to the GPU machine.  :func:`corr_pixel` drives
``pair_correlation`` like ``correlation_procedures_pycuda.two_point_per_pixel``.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_ref', 'libref_kernels.so')
_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.ref_corr_pixel.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, C.c_int, P, P, P, C.c_double,
                                     C.c_double, C.c_int, C.c_int, P, P]
        L.ref_corr_pixel.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def padded(fs, max_len=None):
    """The reference's padded ``[n_forest x max_lenght]`` arrays
    (``correlation_procedures_pycuda.py:63-87``)."""
    L = fs.lengths
    max_len = int(max_len or max(1, L.max() if len(L) else 1))
    dc = np.zeros((fs.n, max_len)); we = np.zeros((fs.n, max_len)); dw = np.zeros((fs.n, max_len))
    for f in range(fs.n):
        a, b = fs.start[f], fs.start[f + 1]
        dc[f, :b - a] = fs.dc[a:b]; we[f, :b - a] = fs.w[a:b]; dw[f, :b - a] = fs.dw[a:b]
    return max_len, dc, we, dw


def corr_pixel(fs, f1_list, nbr_lists, rpmax=200.0, rtmax=200.0, np_=50, nt=50, weights=True):
    """(w_hist, dw_hist) [np, nt] of the reference kernel for first forests
    ``f1_list`` with neighbour lists ``nbr_lists``.  ``weights=False`` runs it with
    w = dw = 1, which makes w_hist the exact pair count."""
    max_len, dc, we, dw = padded(fs)
    if not weights:
        we = np.where(np.arange(max_len)[None, :] < fs.lengths[:, None], 1.0, 0.0)
        dw = we.copy()
    f1 = np.ascontiguousarray(f1_list, dtype=np.int32)
    off = np.zeros(len(f1) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(x) for x in nbr_lists])
    nbr = np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.int32) for x in nbr_lists])
                               if len(nbr_lists) else np.zeros(0, np.int32), dtype=np.int32)
    if nbr.size == 0:
        nbr = np.zeros(1, dtype=np.int32)
    lens = np.ascontiguousarray(fs.lengths, dtype=np.int32)
    x = np.ascontiguousarray(fs.ux); y = np.ascontiguousarray(fs.uy); z = np.ascontiguousarray(fs.uz)
    w_hist = np.zeros((np_, nt)); dw_hist = np.zeros((np_, nt))
    dc = np.ascontiguousarray(dc); we = np.ascontiguousarray(we); dw = np.ascontiguousarray(dw)
    rc = lib().ref_corr_pixel(fs.n, max_len, _p(dc), _p(we), _p(dw), _p(lens), _p(x), _p(y), _p(z), len(f1), _p(f1),
                              _p(off), _p(nbr), float(rpmax), float(rtmax), int(np_), int(nt), _p(w_hist),
                              _p(dw_hist))
    if rc != 0:
        raise RuntimeError(f'reference kernel launcher returned {rc} (1 = unsafe input, 2 = CUDA error)')
    return w_hist, dw_hist
