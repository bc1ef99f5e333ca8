"""GPU distortion matrix against the oracle's restatement of the reference's
compute_etas / compute_d (FP64, same bins).  Tolerance: 1e-10 of the largest
|D| entry (the two sides add the same terms in different orders); W to 1e-12."""
import random

import numpy as np
import pytest

import edge_cases as E
from lya2pcf_b200 import synthetic
from lya2pcf_b200.dropin_path import ensure_on_path
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _check(D, W, Do, Wo):
    np.testing.assert_allclose(W, Wo, rtol=1e-12, atol=1e-12 * np.abs(Wo).max())
    assert np.abs(D - Do).max() <= 1e-10 * np.abs(Do).max()


def test_distortion_all_pairs_matches_oracle():
    fs = synthetic.make(3, n=90)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        D, W = eng.distortion()
    assert len(f1) > 100
    Do, Wo = O.distortion(fs, f1, f2)
    _check(D, W, Do, Wo)
    assert np.count_nonzero(Do) > 1000


def test_distortion_edge_catalogue():
    """Length-1 forest (sum w dl^2 = 0), empty and unsorted forests, twins."""
    fs = E.edge_catalog()
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(0.05)
        f1, f2 = eng.get_pairs()
        D, W = eng.distortion()
    Do, Wo = O.distortion(fs, f1, f2)
    assert np.all(np.isfinite(Do))
    _check(D, W, Do, Wo)


def test_dropin_subsample_matches_oracle():
    """The drop-in module keeps the reference's subsample (random.seed(1),
    reference neighbour order, shuffle per first forest) and bins it."""
    ensure_on_path()
    import distortion_procedures_pycuda as dp
    fs = synthetic.make(3, n=120)
    data = fs.to_quasar_dict()
    dmin = min(float(f.dc[0]) for p in data for f in data[p])
    am = 2 * np.arcsin(0.5 * 200 / dmin)
    dp.init(data, None, (50, 50), am, 0.5)
    pixel = list(data.keys())[len(data) // 2]
    state = random.getstate()
    f1, f2 = dp.selected_pairs(data[pixel])
    random.setstate(state)
    D, W = dp.distortion_per_pixel(data[pixel])
    # the subsample: ceil(n/2) of each forest's reference-ordered neighbours
    fsn = dp._engine.fs
    off, nbr = O.neighbours(fsn, am)
    for f in {q.index for q in data[pixel]}:
        mine = set(f2[f1 == f].tolist())
        full = set(nbr[off[f]:off[f + 1]].tolist())
        assert mine <= full and len(mine) == int(np.ceil(len(full) * 0.5))
    Do, Wo = O.distortion(fsn, f1, f2)
    _check(D, W, Do, Wo)
