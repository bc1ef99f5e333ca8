"""The projection oracle (oracle/ingest.py) against golden vectors from the
reference's own quasar.fill_dw (tests/golden/make_fill_dw_golden.py), and the
columnar catalogue cache.  CPU only."""
import os

import numpy as np

from lya2pcf_b200 import synthetic
from lya2pcf_b200.forests import ForestSet
from oracle import ingest as I

G = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'fill_dw_golden.npz'))


def test_fill_dw_matches_reference_bit_for_bit():
    dw, dl, om, o2 = I.fill_dw_all(G['start'], G['we'], G['delta'], G['loglam'])
    assert np.array_equal(np.isnan(dw), np.isnan(G['dw']))          # the one-pixel forest: 0/0
    ok = ~np.isnan(G['dw'])
    assert np.array_equal(dw[ok], G['dw'][ok])
    assert np.array_equal(dl, G['delta_lambda'])
    assert np.array_equal(om, G['omega']) and np.array_equal(o2, G['odl2'])
    dwn, _, _, _ = I.fill_dw_all(G['start'], G['we'], G['delta'], G['loglam'], project=False)
    assert np.array_equal(dwn, G['dw_noproject'])


def test_columnar_cache_round_trip(tmp_path):
    fs = synthetic.make(4, n=40)
    path = str(tmp_path / 'catalogue.npz')
    fs.save(path)
    back = ForestSet.load(path)
    for k in ForestSet._COLUMNS:
        assert np.array_equal(getattr(back, k), getattr(fs, k)), k
    assert back.n == fs.n and back.npix_total == fs.npix_total
