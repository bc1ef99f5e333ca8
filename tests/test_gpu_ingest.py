"""Device-side ingest (lya_upload_deltas): the projection of quasar.fill_dw on
the GPU against the reference's own values (golden vectors) and the oracle,
and the correlation of a catalogue ingested from its deltas against the same
catalogue projected on the host.  Tolerance: 1e-12 of the largest |w delta|
(the device sums in another order)."""
import os

import numpy as np
import pytest

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from lya2pcf_b200.forests import ForestSet
from oracle import ingest as I

pytestmark = pytest.mark.gpu
G = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'fill_dw_golden.npz'))


def _geometry(start, w, rng):
    """A ForestSet shell around CSR weights: positions on a small patch."""
    n = len(start) - 1
    npix = int(start[-1])
    ra = rng.uniform(0.5, 0.52, n)
    dec = rng.uniform(0.1, 0.12, n)
    dc = np.concatenate([3500.0 + 1.9 * np.arange(start[f + 1] - start[f]) for f in range(n)])
    return ForestSet(start=np.asarray(start, dtype=np.int64), dc=dc, w=np.asarray(w, dtype=np.float64),
                     dw=np.zeros(npix), z=np.full(npix, 2.3), dl=np.zeros(npix), ra=ra, dec=dec,
                     ux=np.cos(ra) * np.cos(dec), uy=np.sin(ra) * np.cos(dec), uz=np.sin(dec),
                     name=np.arange(n, dtype=np.int64), pix=np.zeros(n, dtype=np.int64), omega=np.zeros(n),
                     odl2=np.zeros(n))


def test_projection_matches_reference():
    fs = _geometry(G['start'], G['we'], np.random.default_rng(1))
    scale = np.abs(G['we'] * G['delta']).max()
    with PairEngine() as eng:
        eng.upload_deltas(fs, G['delta'], G['loglam'])
        dw, dl, om, o2 = eng.projection()
        assert np.array_equal(np.isnan(dw), np.isnan(G['dw']))
        ok = ~np.isnan(G['dw'])
        assert np.abs(dw[ok] - G['dw'][ok]).max() <= 1e-12 * scale
        assert np.abs(dl - G['delta_lambda']).max() <= 1e-12 * np.abs(G['delta_lambda']).max()
        np.testing.assert_allclose(om, G['omega'], rtol=1e-13)
        np.testing.assert_allclose(o2, G['odl2'], rtol=1e-12)
        eng.upload_deltas(fs, G['delta'], G['loglam'], project=False)
        dw0, dl0, om0, _ = eng.projection()
        assert np.array_equal(dw0, G['dw_noproject']) and not dl0.any() and not om0.any()


def test_zero_weight_forest_is_an_error():
    w = G['we'].copy()
    a, b = G['start'][3], G['start'][4]
    w[a:b] = 0.0
    fs = _geometry(G['start'], w, np.random.default_rng(2))
    with PairEngine() as eng:
        with pytest.raises(N.LyaError) as e:
            eng.upload_deltas(fs, G['delta'], G['loglam'])
        assert e.value.code == 5


def test_correlation_from_deltas_equals_host_projection():
    rng = np.random.default_rng(7)
    fs = synthetic.make(4, n=120)
    delta = rng.normal(0, 0.25, fs.npix_total)
    loglam = np.log10(1215.67 * (1.0 + fs.z))
    dw, dl, om, o2 = I.fill_dw_all(fs.start, fs.w, delta, loglam)
    fs.dw, fs.dl, fs.omega, fs.odl2 = dw, dl, om, o2
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
        h1, c1 = eng.histograms()
        eng.upload_deltas(fs, delta, loglam)
        dwd, dld, omd, o2d = eng.projection()
        eng.build_pairs(am)
        eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
        h2, c2 = eng.histograms()
    assert np.abs(dwd - dw).max() <= 1e-12 * np.abs(fs.w * delta).max()
    assert np.array_equal(c1, c2)
    np.testing.assert_allclose(h2[:, N.Q_W], h1[:, N.Q_W], rtol=1e-12, atol=0)
    assert np.abs(h2[:, N.Q_DW] - h1[:, N.Q_DW]).max() <= 1e-9 * np.abs(h1[:, N.Q_DW]).max()
