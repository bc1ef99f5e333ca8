"""ctypes front end of the reference's own CUDA kernels (``oracle/_ref``).
TEST INFRASTRUCTURE ONLY.

``libref_kernels.so`` is ``cuda_kernels.cpp`` from the reference tree compiled
by ``oracle/Makefile`` (target ``ref``) behind ``ref_launch.cu``; it exists only
where the reference tree was available at build time and the file travels with
the repository to the GPU machine.  :func:`corr_pixel` drives
``pair_correlation`` like ``correlation_procedures_pycuda.two_point_per_pixel``;
:func:`dist_pixel` drives ``precompute_distances``, ``compute_etas``,
``order_active`` and ``compute_d`` like
``distortion_procedures_pycuda.distortion_per_pixel``, and :func:`dist_bins`
returns the bins ``precompute_distances`` writes.
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
        L.ref_corr_timed.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, C.c_int, P, P, P, C.c_double,
                                     C.c_double, C.c_int, C.c_int, P, P, P]
        L.ref_corr_timed.restype = C.c_int
        L.ref_dist_pixel.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, C.c_int, P, P, P, C.c_float,
                                     C.c_float, C.c_int, C.c_int, P, P]
        L.ref_dist_pixel.restype = C.c_int
        L.ref_dist_bins.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_int, C.c_int, P, C.c_float, C.c_float,
                                    P, P]
        L.ref_dist_bins.restype = C.c_int
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


def corr_timed(fs, f1_list, nbr_lists, rpmax=200.0, rtmax=200.0, np_=50, nt=50):
    """Device milliseconds of the reference kernel's per-forest launch loop
    (three small copies, a launch and a synchronize per first forest, as
    ``two_point_per_pixel``), the padded catalogue uploaded beforehand.
    Returns ``(ms, w_hist, dw_hist)``."""
    max_len, dc, we, dw = padded(fs)
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
    ms = C.c_double(0.0)
    rc = lib().ref_corr_timed(fs.n, max_len, _p(dc), _p(we), _p(dw), _p(lens), _p(x), _p(y), _p(z), len(f1), _p(f1),
                              _p(off), _p(nbr), float(rpmax), float(rtmax), int(np_), int(nt), _p(w_hist),
                              _p(dw_hist), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f'reference kernel launcher returned {rc} (1 = unsafe input, 2 = CUDA error)')
    return ms.value, w_hist, dw_hist


# parameters.py:59 -- the distortion path pads every forest to this many pixels
DIST_MAX_LENGHT = 208


def _padded32(fs, max_len):
    """FP32 ``[n_forest x max_len]`` dc, we, delta_lambda and per-forest x, y, z,
    omega, omega_delta_lambda2: the gran_* arrays of
    ``distortion_procedures_pycuda.init`` (``:71-100``)."""
    L = fs.lengths
    if len(L) and L.max() > max_len:
        raise ValueError(f'forest longer than max_lenght={max_len}')
    dc = np.zeros((fs.n, max_len), np.float32); we = np.zeros_like(dc); dl = np.zeros_like(dc)
    for f in range(fs.n):
        a, b = fs.start[f], fs.start[f + 1]
        dc[f, :b - a] = fs.dc[a:b]; we[f, :b - a] = fs.w[a:b]; dl[f, :b - a] = fs.dl[a:b]
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    return (dc, we, dl, np.ascontiguousarray(L, dtype=np.int32), f32(fs.ux), f32(fs.uy), f32(fs.uz),
            f32(fs.omega), f32(fs.odl2))


def _binners(rpmax, rtmax, np_, nt):
    # distortion_procedures_pycuda.py:167 -- float32([numpix_rp / rmax, numpix_rt / rmax])
    return float(np.float32(np_ / rpmax)), float(np.float32(nt / rtmax))


def dist_pixel(fs, f1_list, nbr_lists, rpmax=200.0, rtmax=200.0, np_=50, nt=50, max_len=DIST_MAX_LENGHT):
    """``(D[nb, nb] float32, W_B[nb] float32)`` of the reference kernels for
    first forests ``f1_list`` with (already subsampled) neighbour lists."""
    dc, we, dl, lens, x, y, z, om, o2 = _padded32(fs, max_len)
    f1 = np.ascontiguousarray(f1_list, dtype=np.int32)
    off = np.zeros(len(f1) + 1, dtype=np.int64)
    off[1:] = np.cumsum([len(x_) for x_ in nbr_lists])
    nbr = np.ascontiguousarray(np.concatenate([np.asarray(x_, dtype=np.int32) for x_ in nbr_lists])
                               if len(nbr_lists) else np.zeros(0, np.int32), dtype=np.int32)
    if nbr.size == 0:
        nbr = np.zeros(1, dtype=np.int32)
    nb = np_ * nt
    D = np.zeros((nb, nb), dtype=np.float32)
    WB = np.zeros(nb, dtype=np.float32)
    brp, brt = _binners(rpmax, rtmax, np_, nt)
    rc = lib().ref_dist_pixel(fs.n, max_len, _p(dc), _p(we), _p(dl), _p(lens), _p(x), _p(y), _p(z), _p(om), _p(o2),
                              len(f1), _p(f1), _p(off), _p(nbr), brp, brt, int(np_), int(nt), _p(D), _p(WB))
    if rc != 0:
        raise RuntimeError(f'reference distortion launcher returned {rc} (1 = unsafe input, 2 = CUDA error)')
    return D, WB


def dist_bins(fs, f1, nbr_list, rpmax=200.0, rtmax=200.0, np_=50, nt=50, max_len=DIST_MAX_LENGHT):
    """``(bin_rp, bin_rt)`` int32 ``[len1, nn, max_len]`` written by the
    reference's ``precompute_distances`` for one first forest (entries
    ``j >= len(f2)`` are -1)."""
    dc, we, dl, lens, x, y, z, om, o2 = _padded32(fs, max_len)
    nbr = np.ascontiguousarray(nbr_list, dtype=np.int32)
    l1 = int(lens[f1])
    bp = np.zeros((l1, len(nbr), max_len), dtype=np.int32)
    bt = np.zeros_like(bp)
    brp, brt = _binners(rpmax, rtmax, np_, nt)
    rc = lib().ref_dist_bins(fs.n, max_len, _p(dc), _p(lens), _p(x), _p(y), _p(z), int(f1), len(nbr), _p(nbr),
                             brp, brt, _p(bp), _p(bt))
    if rc != 0:
        raise RuntimeError(f'reference distortion launcher returned {rc} (1 = unsafe input, 2 = CUDA error)')
    return bp, bt
