"""GPU distortion matrix against the oracle's restatement of the reference's
compute_etas / compute_d (FP64, same bins).  Tolerance: 1e-10 of the largest
|D| entry (the two sides add the same terms in different orders); W to 1e-12."""
import random

import numpy as np
import pytest

import edge_cases as E
from lya2pcf_b200 import _native as N
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


@pytest.mark.parametrize('np_,nt', [(37, 23), (64, 16)])
def test_distortion_other_binnings(np_, nt):
    """An odd number of r_par bins (moments from the spare accumulator rows
    after an odd row length) and 64 r_par bins (no spare rows: the moment loop)."""
    fs = synthetic.make(3, n=90)
    am = synthetic.angmax_for(fs)
    with PairEngine(np_=np_, nt=nt) as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        D, W = eng.distortion()
    Do, Wo = O.distortion(fs, f1, f2, np_=np_, nt=nt)
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


def _oracle_all_pairs(data):
    """(D, W) of every neighbouring forest pair of ``data``, its own angmax."""
    from lya2pcf_b200.forests import from_quasar_dict
    fsd, _ = from_quasar_dict(data)
    dmin = min(float(f.dc[0]) for p in data for f in data[p])
    off, nbr = O.neighbours(fsd, 2 * np.arcsin(0.5 * 200 / dmin))
    f1 = np.repeat(np.arange(fsd.n, dtype=np.int32), np.diff(off)).astype(np.int32)
    return O.distortion(fsd, f1, nbr.astype(np.int32))


def _check_ratio(R, Do, Wo):
    """distortion.npy = D / W[:, None] against the oracle's (D, W): rows of
    zero weight are 0/0 on both sides; the others to 1e-9 of max |D| once
    multiplied back by the row weight."""
    empty = Wo == 0
    assert np.all(np.isnan(R[empty]))
    assert np.all(np.isfinite(R[~empty]))
    err = np.abs(R[~empty] - Do[~empty] / Wo[~empty, None]) * Wo[~empty, None]
    assert err.max() <= 1e-9 * np.abs(Do).max()


def test_multiple_data_driver_per_file_and_merged(tmp_path):
    """distortion_multiple_data.py over two files holding the two halves of
    the owner pixels.  --per-file (the reference's computation) sums each
    file's own matrix; merged (the default) is the whole catalogue's, with the
    pairs across the files.  --excluded 0 keeps every pair, so both are the
    oracle's all-pairs matrices; --excluded 0.5 --per-file must equal the
    module API driven file by file from random.seed(1)."""
    import glob as _glob
    import os
    import subprocess
    import sys
    from lya2pcf_b200.dropin_path import DROPIN_DIR
    fs = synthetic.make(3, n=120)
    data = fs.to_quasar_dict()
    pixels = sorted(data)
    half = {p: data[p] for p in pixels[:len(pixels) // 2]}, {p: data[p] for p in pixels[len(pixels) // 2:]}
    ddir = tmp_path / 'deltas'
    ddir.mkdir()
    for k, d in enumerate(half):
        np.save(ddir / f'data{k + 1}.npy', d, allow_pickle=True)
    script = os.path.join(DROPIN_DIR, 'distortion_multiple_data.py')
    out = {}
    for mode, extra in (('per-file', ['--per-file', '--excluded', '0']), ('merged', ['--excluded', '0']),
                        ('half', ['--per-file', '--excluded', '0.5'])):
        cdir = tmp_path / mode
        r = subprocess.run([sys.executable, script, '--data-dir', str(ddir), '--corr-dir', str(cdir)] + extra,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[mode] = np.load(cdir / 'distortion.npy')
        assert out[mode].shape == (2500, 2500)

    parts = [_oracle_all_pairs(d) for d in half]
    Dp, Wp = parts[0][0] + parts[1][0], parts[0][1] + parts[1][1]
    _check_ratio(out['per-file'], Dp, Wp)
    Dm, Wm = _oracle_all_pairs(data)
    _check_ratio(out['merged'], Dm, Wm)
    assert Wm.sum() > Wp.sum(), 'the halves share neighbouring forests: merging adds pairs'

    ensure_on_path()
    import distortion_procedures_pycuda as dp
    random.seed(1)
    Dh, Wh = np.zeros((2500, 2500)), np.zeros(2500)
    for f in sorted(_glob.glob(str(ddir / 'data*.npy'))):
        d = np.load(f, allow_pickle=True).item()
        dmin = min(float(q.dc[0]) for p in d for q in d[p])
        dp.init(d, None, (50, 50), 2 * np.arcsin(0.5 * 200 / dmin), 0.5)
        for p in d:
            D, W = dp.distortion_per_pixel(d[p])
            Dh += D
            Wh += W
    assert 0 < Wh.sum() < Wp.sum()
    _check_ratio(out['half'], Dh, Wh)


def test_every_launch_shape_and_the_item_limit():
    """Every launch shape of the distortion kernel (lya_dist_config) gives the
    oracle's D and W; a limit of n items bins exactly the first n forest pairs;
    the autotuner leaves a working shape selected."""
    fs = synthetic.make(3, n=70)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        Do, Wo = O.distortion(fs, f1, f2)
        for shape in range(len(PairEngine.DIST_SHAPES)):
            N.check(eng.lib.lya_dist_config(eng.ctx, shape, 0), eng.ctx)
            D, W = eng.distortion()
            _check(D, W, Do, Wo)
        n = len(f1) // 3
        N.check(eng.lib.lya_dist_config(eng.ctx, 0, n), eng.ctx)
        D, W = eng.distortion()
        Dn, Wn = O.distortion(fs, f1[:n], f2[:n])
        _check(D, W, Dn, Wn)
        tune = eng.autotune_distortion(fraction=0.5, min_items=10)
        assert 0 <= tune['best'] < len(PairEngine.DIST_SHAPES)
        D, W = eng.distortion()
        _check(D, W, Do, Wo)
