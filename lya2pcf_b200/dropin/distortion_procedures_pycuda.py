"""Drop-in replacement of lya2pcf's ``distortion_procedures_pycuda`` module.

Same module API as the reference (``distortion_procedures_pycuda.py:19-279``):

    init(data, log_file, shape_hist, angmax, reject, pixel_list=None)
    distortion_per_pixel(forest_list, **kargs) -> (dist_hist[nb, nb], weight_B[nb])

Subsampling is the reference's: the module seeds Python's ``random`` with 1 at
import (``:11``); for every first forest, in list order, the neighbour list in
the reference's visiting order (ascending healpix pixel, then list position,
as ``query_disc`` + ``neighborhood`` give it) is shuffled with
``random.shuffle`` and its first ``ceil(n (1 - reject))`` entries are kept
(``:220-225``).  The selected forest pairs are binned on the GPU
(``lya_dist_run``); the returned arrays are float64 (the reference returns
float32 and its driver sums them in float64, ``distortion.py:107-108``).
"""
import os
import random
import sys

import numpy as np

_here = os.path.dirname(os.path.abspath(__file__))
_root = os.path.dirname(os.path.dirname(_here))
for _p in (_here, _root):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from parameters import *   # noqa: E402,F401,F403
from parameters import rpmax, rtmax   # noqa: E402
from lya2pcf_b200.engine import PairEngine   # noqa: E402
from lya2pcf_b200.forests import from_quasar_dict   # noqa: E402

random.seed(1)

data = None
log_file = None
shape_hist = None
angmax = None
reject_fraction = None
total_bins = None
_engine = None
_nbr_off = None
_nbr = None


def _device():
    want = int(os.environ.get('CUDA_DEVICE', '0'))
    try:
        import torch
        n = torch.cuda.device_count()
    except Exception:
        n = 0
    return want % n if n > 0 else want


def init(data_aux, log_file_aux, shape_hist_aux, angmax_aux, reject_aux, pixel_list=None):
    """Upload the forests and build every forest's neighbour list in the
    reference's order (``distortion_procedures_pycuda.py:19-194``)."""
    global data, log_file, shape_hist, angmax, reject_fraction, total_bins, _engine, _nbr_off, _nbr
    data = data_aux
    log_file = log_file_aux
    shape_hist = tuple(int(x) for x in shape_hist_aux)
    angmax = float(angmax_aux)
    reject_fraction = float(reject_aux)
    total_bins = int(np.prod(shape_hist))
    fs, forests = from_quasar_dict(data, pixel_list)
    for k, q in enumerate(forests):
        q.index = k
    if _engine is not None:
        _engine.close()
    _engine = PairEngine(device=_device(), rpmax=rpmax, rtmax=rtmax, np_=shape_hist[0], nt=shape_hist[1])
    _engine.upload(fs)
    _engine.build_pairs(angmax)
    f1, f2 = _engine.get_pairs()
    # reference visiting order of the candidates: ascending pixel, then list position
    local = np.zeros(fs.n, dtype=np.int64)
    seen = {}
    for f, p in enumerate(fs.pix.tolist()):
        local[f] = seen.get(p, 0)
        seen[p] = local[f] + 1
    key = fs.pix.astype(np.int64) * (1 << 32) + local
    order = np.lexsort((key[f2], f1))
    _nbr = f2[order]
    _nbr_off = np.zeros(fs.n + 1, dtype=np.int64)
    np.cumsum(np.bincount(f1, minlength=fs.n), out=_nbr_off[1:])
    if log_file is not None:
        log_file.write(f'\nUploaded {fs.n} forests; {len(f1)} neighbouring forest pairs')
        log_file.flush()


def selected_pairs(forest_list):
    """(f1, f2) of the subsample the reference keeps for these first forests;
    consumes Python's random stream exactly as the reference does."""
    f1, f2 = [], []
    for forest1 in forest_list:
        i = forest1.index
        nbrs = _nbr[_nbr_off[i]:_nbr_off[i + 1]].tolist()
        keep = int(np.ceil(len(nbrs) * (1. - reject_fraction)))
        random.shuffle(nbrs)
        f1.extend([i] * keep)
        f2.extend(nbrs[:keep])
    return np.asarray(f1, dtype=np.int32), np.asarray(f2, dtype=np.int32)


def distortion_per_pixel(forest_list, **kargs):
    """(dist_hist[nb, nb], weight_B[nb]) summed over the kept pairs of the
    forests in ``forest_list`` (``distortion_procedures_pycuda.py:195-279``)."""
    f1, f2 = selected_pairs(forest_list)
    order = np.argsort(f1, kind='stable')
    _engine.set_pairs(f1[order], f2[order])
    return _engine.distortion()
