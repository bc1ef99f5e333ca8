"""The drop-in module API and the 2pla.py driver, end to end, against the oracle."""
import glob
import os
import subprocess
import sys

import numpy as np
import pytest

from lya2pcf_b200 import synthetic
from lya2pcf_b200.dropin_path import DROPIN_DIR, ensure_on_path
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _oracle_per_pixel(fs, angmax):
    off, nbr = O.neighbours(fs, angmax)
    f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
    ho, co = O.corr(fs, f1, f2, sis)
    return {int(p): (ho[k], co[k]) for k, p in enumerate(pixels)}


def test_module_api_matches_oracle():
    ensure_on_path()
    import correlation_procedures_pycuda as cp
    fs = synthetic.make(0, scale=0.2)
    data = fs.to_quasar_dict()
    dmin = min(float(f.dc[0]) for p in data for f in data[p])
    angmax = 2 * np.arcsin(0.5 * 200 / dmin)
    cp.init(data, None, (50, 50), angmax)
    idx = [q.index for p in data for q in data[p]]
    assert idx == list(range(fs.n))
    ref = _oracle_per_pixel(fs, angmax)
    for pixel in data:
        w, dw = cp.two_point_per_pixel(pixel)
        assert w.shape == (50, 50) and w.dtype == np.float64
        ho, co = ref[int(pixel)]
        np.testing.assert_allclose(w.ravel(), ho[O.Q_W], rtol=1e-6, atol=0)
        assert np.all(np.abs(dw.ravel() - ho[O.Q_DW]) <= 1e-6 * ho[O.Q_DWABS] + 1e-300)
        ex = cp.pixel_extras(pixel)
        assert np.array_equal(ex['npairs'].ravel(), co)
        W = ho[O.Q_W]
        rp = np.divide(ho[O.Q_RP], W, out=np.zeros_like(W), where=W != 0)
        np.testing.assert_allclose(ex['rp'].ravel(), rp, rtol=1e-6, atol=1e-9)


def test_2pla_driver_writes_reference_files(tmp_path):
    fs = synthetic.make(0, scale=0.2)
    data = fs.to_quasar_dict()
    ddir = tmp_path / 'deltas'
    cdir = tmp_path / 'out'
    ddir.mkdir()
    np.save(ddir / 'data1.npy', data, allow_pickle=True)
    r = subprocess.run([sys.executable, os.path.join(DROPIN_DIR, '2pla.py'), '--gpu', '--data-dir', str(ddir),
                        '--corr-dir', str(cdir)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    files = sorted(glob.glob(str(cdir / '2d_histogram_pixel_*')))
    assert len(files) == len(data)
    dmin = min(float(f.dc[0]) for p in data for f in data[p])
    ref = _oracle_per_pixel(fs, 2 * np.arcsin(0.5 * 200 / dmin))
    for f in files:
        pixel = int(os.path.basename(f)[len('2d_histogram_pixel_'):-4])
        w_hist, dw_hist = np.load(f)            # post_processing.py:139 unpacks exactly two arrays
        ho, co = ref[pixel]
        np.testing.assert_allclose(w_hist.ravel(), ho[O.Q_W], rtol=1e-6, atol=0)
        ex = np.load(cdir / f'pairs_2d_pixel_{pixel}.npz')
        assert np.array_equal(ex['npairs'].ravel(), co)


def test_multiple_data_driver_per_file_and_merged(tmp_path):
    """Two data files holding the two halves of the owner pixels.  With
    --per-file every file is binned alone (the reference's
    2pla_multiple_data.py): each pixel's histograms are those of its own file's
    catalogue.  Merged (the default): those of the whole catalogue, i.e. the
    pairs across the two files are counted too."""
    fs = synthetic.make(0, scale=0.2)
    data = fs.to_quasar_dict()
    pixels = sorted(data)
    half = {p: data[p] for p in pixels[:len(pixels) // 2]}, {p: data[p] for p in pixels[len(pixels) // 2:]}
    ddir = tmp_path / 'deltas'
    ddir.mkdir()
    for k, d in enumerate(half):
        np.save(ddir / f'data{k + 1}.npy', d, allow_pickle=True)
    script = os.path.join(DROPIN_DIR, '2pla_multiple_data.py')
    runs = {}
    for mode in ('per-file', 'merged'):
        cdir = tmp_path / mode
        cmd = [sys.executable, script, '--gpu', '--data-dir', str(ddir), '--corr-dir', str(cdir)]
        if mode == 'per-file':
            cmd.append('--per-file')
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        runs[mode] = {int(os.path.basename(f)[len('2d_histogram_pixel_'):-4]): np.load(f)
                      for f in glob.glob(str(cdir / '2d_histogram_pixel_*'))}
        assert len(runs[mode]) == len(data)
    from lya2pcf_b200.forests import from_quasar_dict
    ref = {}
    for d in half:
        fsd, _ = from_quasar_dict(d)
        dmin = min(float(f.dc[0]) for p in d for f in d[p])
        ref.update(_oracle_per_pixel(fsd, 2 * np.arcsin(0.5 * 200 / dmin)))
    dmin = min(float(f.dc[0]) for p in data for f in data[p])
    ref_all = _oracle_per_pixel(fs, 2 * np.arcsin(0.5 * 200 / dmin))
    more = 0
    for p in data:
        w_pf, _ = runs['per-file'][p]
        w_m, _ = runs['merged'][p]
        np.testing.assert_allclose(w_pf.ravel(), ref[p][0][O.Q_W], rtol=1e-6, atol=0)
        np.testing.assert_allclose(w_m.ravel(), ref_all[p][0][O.Q_W], rtol=1e-6, atol=0)
        more += int(ref_all[p][1].sum() > ref[p][1].sum())
    assert more > 0, 'the halves share neighbouring forests: merging adds pairs'
