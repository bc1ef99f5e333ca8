"""ctypes front end of the CPU oracle (``oracle.c``).  TEST INFRASTRUCTURE ONLY.

Used by the tests, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py`` as the checker of the CUDA path; the product never imports it.
Each function names the reference routine it restates (see ``oracle.c``).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_build', 'liboracle.so')

NQ = 6
Q_W, Q_DW, Q_RP, Q_RT, Q_Z, Q_DWABS = range(NQ)
GPU_FORMULA, CPU_FORMULA = 0, 1
BIN_FP64, BIN_FP32 = 0, 1

_lib = None


def build(force=False):
    if force or not os.path.exists(LIB_PATH) or \
            os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, 'oracle.c')):
        subprocess.run(['make', '-s', '-C', HERE, 'all'], check=True)
    return LIB_PATH


class _Forests(C.Structure):
    _fields_ = [('n', C.c_int64), ('start', C.c_void_p)] + \
               [(k, C.c_void_p) for k in ('dc', 'w', 'dw', 'z', 'dl', 'ux', 'uy', 'uz', 'ra', 'dec', 'omega', 'odl2')]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_neighbours.argtypes = [P, P, P, C.c_double, C.c_double, P, P, P, C.c_int]
        L.orc_corr.argtypes = [P, C.c_int64, P, P, P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_double, P, P, C.c_int]
        L.orc_corr_wdw.argtypes = [P, C.c_int64, P, P, P, C.c_double, C.c_double, C.c_int, C.c_int, P, C.c_int]
        L.orc_adjoint.argtypes = [P, C.c_int64, P, P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, P, P, P, P]
        L.orc_distortion.argtypes = [P, C.c_int64, P, P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, P, P]
        L.orc_distortion_mode.argtypes = [P, C.c_int64, P, P, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                          C.c_int, P, P]
        L.orc_dist_bins.argtypes = [P, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                    C.c_int, P, P]
        L.orc_cos12.argtypes = [C.c_double] * 6 + [C.c_int]
        L.orc_cos12.restype = C.c_double
        for f in ('orc_neighbours', 'orc_corr', 'orc_corr_wdw', 'orc_adjoint', 'orc_distortion', 'orc_distortion_mode',
                  'orc_dist_bins'):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Catalog:
    """Keeps contiguous copies of a ForestSet's arrays alive for the C side."""

    def __init__(self, fs):
        self.fs = fs
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        self.arrays = dict(start=np.ascontiguousarray(fs.start, dtype=np.int64),
                           dc=f64(fs.dc), w=f64(fs.w), dw=f64(fs.dw), z=f64(fs.z), dl=f64(fs.dl),
                           ux=f64(fs.ux), uy=f64(fs.uy), uz=f64(fs.uz), ra=f64(fs.ra), dec=f64(fs.dec),
                           omega=f64(fs.omega), odl2=f64(fs.odl2))
        self.name = np.ascontiguousarray(fs.name, dtype=np.int64)
        self.struct = _Forests(fs.n, *[_ptr(self.arrays[k]) for k in
                                        ('start', 'dc', 'w', 'dw', 'z', 'dl', 'ux', 'uy', 'uz', 'ra', 'dec',
                                         'omega', 'odl2')])

    @property
    def ref(self):
        return C.byref(self.struct)


def cos12(u1, u2, variant):
    return lib().orc_cos12(*map(float, u1), *map(float, u2), int(variant))


def reference_order_key(fs):
    """Order in which the reference visits candidate neighbours: ascending
    healpix pixel, then the forest's position inside its pixel's list."""
    local = np.zeros(fs.n, dtype=np.int64)
    seen = {}
    for f, p in enumerate(fs.pix.tolist()):
        local[f] = seen.get(p, 0)
        seen[p] = local[f] + 1
    return fs.pix.astype(np.int64) * (1 << 32) + local


def neighbours(fs, angmax, nthreads=None, key=None, cat=None):
    """CSR neighbour lists ``(offsets[n+1], nbr)`` of ``quasar.neighborhood``."""
    cat = cat or Catalog(fs)
    nthreads = nthreads or os.cpu_count() or 1
    key = np.ascontiguousarray(reference_order_key(fs) if key is None else key, dtype=np.int64)
    mumin = float(np.cos(angmax))
    counts = np.zeros(fs.n, dtype=np.int64)
    rc = lib().orc_neighbours(cat.ref, _ptr(cat.name), _ptr(key), float(angmax), mumin, _ptr(counts), None, None,
                              int(nthreads))
    assert rc == 0
    off = np.zeros(fs.n + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    nbr = np.zeros(max(1, int(off[-1])), dtype=np.int32)
    rc = lib().orc_neighbours(cat.ref, _ptr(cat.name), _ptr(key), float(angmax), mumin, _ptr(counts), _ptr(off),
                              _ptr(nbr), int(nthreads))
    assert rc == 0
    return off, nbr[:int(off[-1])]


def owner_slots(fs):
    """Output slot of every forest's pairs: index of its healpix pixel among the
    sorted distinct pixels.  Returns (slot_of_forest, slot_pixels)."""
    pixels, slot = np.unique(fs.pix, return_inverse=True)
    return slot.astype(np.int64), pixels


def items_from_csr(fs, off, nbr):
    """Forest-pair list grouped by owner slot: (f1, f2, slot_item_start, slot_pixels)."""
    slot, pixels = owner_slots(fs)
    f1 = np.repeat(np.arange(fs.n, dtype=np.int32), np.diff(off))
    f2 = np.asarray(nbr, dtype=np.int32)
    order = np.argsort(slot[f1], kind='stable')
    f1, f2 = f1[order], f2[order]
    counts = np.bincount(slot[f1], minlength=len(pixels)) if len(f1) else np.zeros(len(pixels), dtype=np.int64)
    sis = np.zeros(len(pixels) + 1, dtype=np.int64)
    np.cumsum(counts, out=sis[1:])
    return np.ascontiguousarray(f1), np.ascontiguousarray(f2), sis, pixels


def corr(fs, f1, f2, slot_item_start, rpmax=200.0, rtmax=200.0, np_=50, nt=50, mode=GPU_FORMULA,
         cos_variant=0, angmax=0.0, nthreads=None, cat=None):
    """Per-slot histograms ``out[nslot, 6, np*nt]`` (W, DW, RP, RT, Z, DWABS) and
    pair counts ``cnt[nslot, np*nt]``."""
    cat = cat or Catalog(fs)
    nthreads = nthreads or os.cpu_count() or 1
    nslot = len(slot_item_start) - 1
    nb = np_ * nt
    out = np.zeros((nslot, NQ, nb), dtype=np.float64)
    cnt = np.zeros((nslot, nb), dtype=np.uint64)
    f1 = np.ascontiguousarray(f1, dtype=np.int32)
    f2 = np.ascontiguousarray(f2, dtype=np.int32)
    sis = np.ascontiguousarray(slot_item_start, dtype=np.int64)
    rc = lib().orc_corr(cat.ref, nslot, _ptr(sis), _ptr(f1), _ptr(f2), float(rpmax), float(rtmax), int(np_), int(nt),
                        int(mode), int(cos_variant), float(angmax), _ptr(out), _ptr(cnt), int(nthreads))
    assert rc == 0
    return out, cnt


def corr_wdw(fs, f1, f2, slot_item_start, rpmax=200.0, rtmax=200.0, np_=50, nt=50, nthreads=None, cat=None):
    """W and DW only (the reference kernel's outputs), ``out[nslot, 2, np*nt]``:
    the work the CPU baseline times."""
    cat = cat or Catalog(fs)
    nthreads = nthreads or os.cpu_count() or 1
    nslot = len(slot_item_start) - 1
    out = np.zeros((nslot, 2, np_ * nt), dtype=np.float64)
    f1 = np.ascontiguousarray(f1, dtype=np.int32)
    f2 = np.ascontiguousarray(f2, dtype=np.int32)
    sis = np.ascontiguousarray(slot_item_start, dtype=np.int64)
    rc = lib().orc_corr_wdw(cat.ref, nslot, _ptr(sis), _ptr(f1), _ptr(f2), float(rpmax), float(rtmax), int(np_),
                            int(nt), _ptr(out), int(nthreads))
    assert rc == 0
    return out


def adjoint(fs, f1, f2, coef_dw, coef_w, rpmax=200.0, rtmax=200.0, np_=50, nt=50, cos_variant=0, cat=None):
    cat = cat or Catalog(fs)
    g_dw = np.zeros(fs.npix_total, dtype=np.float64)
    g_w = np.zeros(fs.npix_total, dtype=np.float64)
    f1 = np.ascontiguousarray(f1, dtype=np.int32)
    f2 = np.ascontiguousarray(f2, dtype=np.int32)
    cdw = np.ascontiguousarray(coef_dw, dtype=np.float64)
    cw = np.ascontiguousarray(coef_w, dtype=np.float64)
    rc = lib().orc_adjoint(cat.ref, len(f1), _ptr(f1), _ptr(f2), float(rpmax), float(rtmax), int(np_), int(nt),
                           int(cos_variant), _ptr(cdw), _ptr(cw), _ptr(g_dw), _ptr(g_w))
    assert rc == 0
    return g_dw, g_w


def distortion(fs, f1, f2, rpmax=200.0, rtmax=200.0, np_=50, nt=50, cos_variant=0, bin_mode=BIN_FP64, cat=None):
    """Unnormalised distortion numerator D[nb, nb] and bin weights W_B[nb].
    ``bin_mode`` BIN_FP64 bins pairs with the correlation's FP64 formula,
    BIN_FP32 with the reference distortion's FP32 precompute_distances."""
    cat = cat or Catalog(fs)
    nb = np_ * nt
    D = np.zeros((nb, nb), dtype=np.float64)
    WB = np.zeros(nb, dtype=np.float64)
    f1 = np.ascontiguousarray(f1, dtype=np.int32)
    f2 = np.ascontiguousarray(f2, dtype=np.int32)
    rc = lib().orc_distortion_mode(cat.ref, len(f1), _ptr(f1), _ptr(f2), float(rpmax), float(rtmax), int(np_),
                                   int(nt), int(cos_variant), int(bin_mode), _ptr(D), _ptr(WB))
    assert rc == 0
    return D, WB


def dist_bins(fs, a, b, rpmax=200.0, rtmax=200.0, np_=50, nt=50, cos_variant=0, bin_mode=BIN_FP32, cat=None):
    """(bin_rp, bin_rt) int32 [len_a, len_b] of forest pair (a, b)."""
    cat = cat or Catalog(fs)
    la, lb = int(fs.start[a + 1] - fs.start[a]), int(fs.start[b + 1] - fs.start[b])
    bp = np.zeros((la, lb), dtype=np.int32)
    bt = np.zeros((la, lb), dtype=np.int32)
    if la and lb:
        rc = lib().orc_dist_bins(cat.ref, int(a), int(b), float(rpmax), float(rtmax), int(np_), int(nt),
                                 int(cos_variant), int(bin_mode), _ptr(bp), _ptr(bt))
        assert rc == 0
    return bp, bt


def pair_count_total(fs, f1, f2):
    """Reference pair count of a forest-pair list: sum of len1 * len2."""
    L = fs.lengths
    return int(np.sum(L[np.asarray(f1)] * L[np.asarray(f2)]))
