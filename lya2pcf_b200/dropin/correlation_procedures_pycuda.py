"""Drop-in replacement of lya2pcf's ``correlation_procedures_pycuda`` module.

Same module API as the reference (``correlation_procedures_pycuda.py:16-171``):

    init(data, log_file, shape_hist, angmax, pixel_list=None)
    two_point_per_pixel(pixel, **kargs) -> (w_hist, dw_hist)   # float64, shape_hist

``init`` packs the pixel dict into the library's CSR catalogue (setting
``forest.index`` like the reference), uploads it once and builds every
forest's neighbour list on the device.  The first ``two_point_per_pixel``
call bins the whole work queue (or the pixels passed to
:func:`restrict_pixels`) in one persistent launch; each call then returns one
pixel's histograms.  :func:`pixel_extras` gives the outputs the reference does
not have (pair counts and w1w2-weighted mean r_par, r_perp, z).

Device: ``CUDA_DEVICE`` (set per MPI rank by the reference drivers,
``2pla.py:21-22``) modulo the visible device count.
"""
import os
import sys

import numpy as np

_here = os.path.dirname(os.path.abspath(__file__))
_root = os.path.dirname(os.path.dirname(_here))
for _p in (_here, _root):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from parameters import *   # noqa: E402,F401,F403
from parameters import rpmax, rtmax   # noqa: E402
from lya2pcf_b200 import _native as N   # noqa: E402
from lya2pcf_b200.engine import PairEngine   # noqa: E402
from lya2pcf_b200.forests import from_quasar_dict   # noqa: E402

KERNEL = N.KERNEL_FP32_GUARDED
GUARD = 1e-4            # Mpc/h
myfloat = np.float64

data = None
log_file = None
shape_hist = None
angmax = None
_engine = None
_slot_of_pixel = {}
_computed = False
_restrict = None            # owner slots of this rank's share (None: every pixel)
_queue_restricted = False   # the device work queue holds only a share's pairs


def _device():
    want = int(os.environ.get('CUDA_DEVICE', '0'))
    try:
        import torch
        n = torch.cuda.device_count()
    except Exception:
        n = 0
    return want % n if n > 0 else want


def init(data_aux, log_file_aux, shape_hist_aux, angmax_aux, pixel_list=None):
    """Upload the forests of ``pixel_list`` (default: every pixel) and build the
    neighbour lists (``correlation_procedures_pycuda.py:16-111`` + the per-forest
    ``neighborhood`` calls of ``:144``)."""
    global data, log_file, shape_hist, angmax, _engine, _slot_of_pixel, _computed, _restrict, _queue_restricted
    data = data_aux
    log_file = log_file_aux
    shape_hist = tuple(int(x) for x in shape_hist_aux)
    angmax = float(angmax_aux)
    fs, forests = from_quasar_dict(data, pixel_list)
    for k, q in enumerate(forests):
        q.index = k
    if _engine is not None:
        _engine.close()
    _engine = PairEngine(device=_device(), rpmax=rpmax, rtmax=rtmax, np_=shape_hist[0], nt=shape_hist[1])
    _engine.upload(fs)
    n_pairs = _engine.build_pairs(angmax)
    _slot_of_pixel = {int(p): s for s, p in enumerate(_engine.slot_pixels.tolist())}
    _computed = False
    _restrict = None
    _queue_restricted = False
    if log_file is not None:
        log_file.write(f'\nUploaded {fs.n} forests ({fs.npix_total} pixels); {n_pairs} neighbouring forest pairs')
        log_file.flush()


def restrict_pixels(pixels):
    """Bin only the pairs owned by ``pixels`` (any subset of the pixel dict,
    e.g. one rank's cost-balanced share) on the next computation."""
    global _restrict, _computed
    _restrict = frozenset(_slot_of_pixel[int(p)] for p in pixels if int(p) in _slot_of_pixel)
    _computed = False


def _compute():
    global _computed, _queue_restricted
    if not _computed:
        if _restrict is None:
            if _queue_restricted:   # an earlier share compacted the queue: rebuild it
                _engine.build_pairs(angmax)
                _queue_restricted = False
            _engine.run(kernel=KERNEL, guard=GUARD)
        elif _restrict:
            if _queue_restricted:
                _engine.build_pairs(angmax)
            _engine.select_slots(sorted(_restrict))
            _queue_restricted = True
            _engine.run(kernel=KERNEL, guard=GUARD)
        _computed = True


def _slot_hist(pixel):
    _compute()
    s = _slot_of_pixel.get(int(pixel))
    if s is None or (_restrict is not None and s not in _restrict):
        return None, None
    hist, cnt = _engine.histograms(s, 1)
    return hist[0], cnt[0]


def two_point_per_pixel(pixel, **kargs):
    """(w_hist, dw_hist): sum w1 w2 and sum dw1 dw2 over pixel pairs whose first
    forest lies in healpix ``pixel`` (``correlation_procedures_pycuda.py:114-171``)."""
    h, _ = _slot_hist(pixel)
    if h is None:
        return (np.zeros(shape_hist, dtype=myfloat), np.zeros(shape_hist, dtype=myfloat))
    return (h[N.Q_W].reshape(shape_hist).copy(), h[N.Q_DW].reshape(shape_hist).copy())


def pixel_extras(pixel):
    """New outputs of one pixel: pair counts and the w1w2-weighted means of
    r_par, r_perp and z = (z1+z2)/2 per bin (0 where a bin is empty)."""
    h, c = _slot_hist(pixel)
    if h is None:
        z = np.zeros(shape_hist)
        return dict(npairs=np.zeros(shape_hist, dtype=np.uint64), rp=z, rt=z.copy(), z=z.copy())
    W = h[N.Q_W]
    mean = lambda q: np.divide(h[q], W, out=np.zeros_like(W), where=W != 0).reshape(shape_hist)  # noqa: E731
    return dict(npairs=c.reshape(shape_hist).copy(), rp=mean(N.Q_RP), rt=mean(N.Q_RT), z=mean(N.Q_Z))
