"""GPU parity of the pair-histogram kernels against the CPU oracle.

Counts are compared bit for bit; floating-point sums within the tolerances
stated per test (FP32 kernel: 1e-6 relative, normwise for DW against
sum |dw1 dw2|; FP64 kernels: 1e-12)."""
import numpy as np
import pytest

import edge_cases as E
from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KERNELS = [N.KERNEL_FP32_GUARDED, N.KERNEL_FP64_DIAGONAL, N.KERNEL_FP64_PLAIN]
TOL = {N.KERNEL_FP32_GUARDED: 1e-6, N.KERNEL_FP64_DIAGONAL: 1e-12, N.KERNEL_FP64_PLAIN: 1e-12}
# (kernel, walk variant): the FP32 kernel with its default walk (lean walk for
# eligible forest pairs) and with the two-diagonal walk for every pair, and the
# two FP64 kernels
CASES = [(N.KERNEL_FP32_GUARDED, 0), (N.KERNEL_FP32_GUARDED, N.VARIANT_TWO_DIAGONALS), (N.KERNEL_FP64_DIAGONAL, 0),
         (N.KERNEL_FP64_PLAIN, 0)]
CASE_IDS = ['fp32', 'fp32-diag2', 'fp64diag', 'fp64plain']


def check_hist(h, c, ho, co, kern, label=''):
    assert np.array_equal(c, co), f'{label}: pair counts differ ({int(np.abs(c.astype(np.int64) - co.astype(np.int64)).sum())} pairs)'
    tol = TOL[kern]
    W, Wo = h[:, N.Q_W], ho[:, O.Q_W]
    assert np.all(np.abs(W - Wo) <= tol * np.abs(Wo) + 1e-300), f'{label}: W'
    # DW has random signs: compare against its condition scale sum |dw1 dw2|
    assert np.all(np.abs(h[:, N.Q_DW] - ho[:, O.Q_DW]) <= tol * ho[:, O.Q_DWABS] + 1e-300), f'{label}: DW'
    for q, qo in ((N.Q_RP, O.Q_RP), (N.Q_RT, O.Q_RT), (N.Q_Z, O.Q_Z)):
        assert np.all(np.abs(h[:, q] - ho[:, qo]) <= tol * np.abs(ho[:, qo]) + 1e-9 * tol), f'{label}: q{q}'


@pytest.fixture(scope='module')
def cfg0():
    fs = synthetic.make(0)
    am = synthetic.angmax_for(fs)
    eng = PairEngine().upload(fs)
    eng.build_pairs(am)
    off, nbr = O.neighbours(fs, am)
    f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
    yield fs, am, eng, (off, nbr), (f1, f2, sis, pixels)
    eng.close()


def test_device_neighbours_equal_oracle(cfg0):
    fs, am, eng, (off, nbr), _ = cfg0
    d1, d2 = eng.get_pairs()
    assert len(d1) == off[-1]
    o1 = np.repeat(np.arange(fs.n), np.diff(off))
    assert set(zip(d1.tolist(), d2.tolist())) == set(zip(o1.tolist(), nbr.tolist()))
    assert np.all(np.diff(d1) >= 0)          # grouped by first forest
    st = eng.stats()
    assert st['ref_pairs'] == float(np.sum(fs.lengths[o1] * fs.lengths[nbr]))


@pytest.fixture(scope='module')
def cfg0_oracle(cfg0):
    """The oracle's histograms of every owner slot of the small configuration
    (7e10 pixel pairs, all host threads)."""
    fs, am, eng, _, (f1, f2, sis, pixels) = cfg0
    return O.corr(fs, f1, f2, sis)


@pytest.mark.parametrize('kern,var', CASES, ids=CASE_IDS)
def test_config0_all_slots_match_oracle(cfg0, cfg0_oracle, kern, var):
    """Every owner slot of the small configuration: counts bit-exact against
    the oracle, sums within the kernel's tolerance."""
    fs, am, eng, _, (f1, f2, sis, pixels) = cfg0
    ho, co = cfg0_oracle
    assert len(pixels) >= 15   # the 100 deg^2 patch covers 17 healpix pixels at nside 16
    eng.run(kernel=kern, variant=var)
    h, c = eng.histograms()
    check_hist(h, c, ho, co, kern, f'kernel {kern}')


def test_slot_restricted_run(cfg0):
    fs, am, eng, _, (f1, f2, sis, pixels) = cfg0
    st = eng.run(kernel=N.KERNEL_FP32_GUARDED, slots=(3, 5))
    h, c = eng.histograms()
    assert c[:3].sum() == 0 and c[5:].sum() == 0 and c[3:5].sum() > 0
    ho, co = O.corr(fs, f1[sis[3]:sis[5]], f2[sis[3]:sis[5]], sis[3:6] - sis[3])
    assert np.array_equal(c[3:5], co)
    assert st['run_ref_pairs'] == float(np.sum(fs.lengths[f1[sis[3]:sis[5]]] * fs.lengths[f2[sis[3]:sis[5]]]))


@pytest.mark.parametrize('var', [0, N.VARIANT_TWO_DIAGONALS], ids=['fp32', 'fp32-diag2'])
def test_fp32_counts_equal_fp64_all_slots(cfg0, var):
    fs, am, eng, _, _ = cfg0
    eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=var)
    h32, c32 = eng.histograms()
    eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
    h64, c64 = eng.histograms()
    assert np.array_equal(c32, c64)
    for q in (N.Q_W, N.Q_RP, N.Q_RT, N.Q_Z):
        np.testing.assert_allclose(h32[:, q], h64[:, q], rtol=1e-6, atol=0)


@pytest.mark.parametrize('kern,var', CASES, ids=CASE_IDS)
def test_edge_catalog(kern, var):
    fs = E.edge_catalog()
    am = 0.05
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        off, nbr = O.neighbours(fs, am)
        f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
        d1, d2 = eng.get_pairs()
        assert set(zip(d1.tolist(), d2.tolist())) == set(zip(f1.tolist(), f2.tolist()))
        ho, co = O.corr(fs, f1, f2, sis)
        eng.run(kernel=kern, variant=var)
        h, c = eng.histograms()
        check_hist(h, c, ho, co, kern, 'edge catalogue')
        assert c.sum() > 0


@pytest.mark.parametrize('kern,var', CASES, ids=CASE_IDS)
def test_whole_sky_sweep_pairs(kern, var):
    """The seeded whole-sky golden sweep (high declinations, pairs across
    ra = 0 / 2 pi; its CPU-formula histograms pin the oracle to the reference
    numba kernel): one owner slot per forest pair, counts bit-exact against the
    oracle's GPU formula, sums within the kernel's tolerance."""
    import os
    from helpers import forestset
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'numba_sweep.npz'))
    keys = ('ra', 'dec', 'dc', 'w', 'dw', 'z')
    n = int(g['n_cases'])
    fs = forestset([{k: g[f'c{c}_{t}_{k}'] for k in keys} for c in range(n) for t in ('a', 'b')],
                   pix=np.repeat(np.arange(n), 2))
    f1 = np.arange(0, 2 * n, 2, dtype=np.int32)
    f2 = f1 + 1
    ho, co = O.corr(fs, f1, f2, np.arange(n + 1))
    with PairEngine() as eng:
        eng.upload(fs)
        eng.set_pairs(f1, f2)
        eng.run(kernel=kern, variant=var)
        h, c = eng.histograms()
    check_hist(h, c, ho, co, kern, 'whole-sky sweep')
    assert c.sum() > 200000


@pytest.mark.parametrize('kern,var', CASES, ids=CASE_IDS)
def test_adversarial_bin_edges_bit_exact(kern, var):
    """Pairs within a few ulps of an rt edge: the FP32 kernel must fall back to
    the FP64 formula and land where the oracle does."""
    fs, f1, f2, vb = E.cos_variant_cases(192)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.set_pairs(f1, f2)
        st = eng.run(kernel=kern, variant=var)
        h, c = eng.histograms()
    got = np.array([int(np.nonzero(c[s])[0][0]) if c[s].sum() else -1 for s in range(len(f1))])
    assert np.array_equal(got, vb[:, 0])
    if kern == N.KERNEL_FP32_GUARDED:
        assert st['guard_rechecks'] >= len(f1) // 2


def test_guard_below_bound_is_rejected(cfg0):
    fs, am, eng, _, _ = cfg0
    with pytest.raises(N.LyaError) as e:
        eng.run(kernel=N.KERNEL_FP32_GUARDED, guard=1e-7)
    assert e.value.code == 6
    eng.run(kernel=N.KERNEL_FP32_GUARDED, guard=1e-4)   # context still usable


def test_errors_do_not_poison_context(cfg0):
    fs, am, eng, _, _ = cfg0
    with pytest.raises(N.LyaError):
        eng.run(kernel=7)
    with pytest.raises(N.LyaError):
        eng.run(slots=(5, 2))
    with pytest.raises(N.LyaError):
        eng.set_pairs(np.array([0, fs.n + 5]), np.array([1, 2]))
    eng.build_pairs(am)
    eng.run()


def test_unsorted_and_empty_forests_full_walk():
    """Forests with decreasing dc are walked over every diagonal (no band
    pruning) and still match the oracle."""
    rng = np.random.default_rng(2)
    fs = synthetic.make(4, n=60)
    # reverse a third of the forests
    for f in range(0, fs.n, 3):
        a, b = fs.start[f], fs.start[f + 1]
        for arr in (fs.dc, fs.w, fs.dw, fs.z, fs.dl):
            arr[a:b] = arr[a:b][::-1].copy()
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        off, nbr = O.neighbours(fs, am)
        f1, f2, sis, _ = O.items_from_csr(fs, off, nbr)
        ho, co = O.corr(fs, f1, f2, sis)
        for kern, var in CASES:
            eng.run(kernel=kern, variant=var)
            h, c = eng.histograms()
            check_hist(h, c, ho, co, kern, f'unsorted {kern}/{var}')


def test_lean_walk_mixed_with_ineligible_forests():
    """The FP32 kernel's lean walk takes pairs of sorted forests with
    0 <= dc < 1e6 only; forests with negative or very large dc, or a NaN pixel,
    fall back to the two-diagonal walk in the same launch.  Counts and sums
    match the oracle."""
    fs = synthetic.make(4, n=60)
    am = synthetic.angmax_for(fs)
    for f in range(0, fs.n, 5):          # shifted below zero (still sorted)
        a, b = fs.start[f], fs.start[f + 1]
        fs.dc[a:b] -= fs.dc[a] + 50.0
    for f in range(1, fs.n, 7):          # beyond the lean range
        a, b = fs.start[f], fs.start[f + 1]
        fs.dc[a:b] += 2.0e6
    for f in range(2, fs.n, 11):         # one NaN pixel
        a, b = fs.start[f], fs.start[f + 1]
        if b - a > 3:
            fs.dc[a + 2] = np.nan
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        off, nbr = O.neighbours(fs, am)
        f1, f2, sis, _ = O.items_from_csr(fs, off, nbr)
        ho, co = O.corr(fs, f1, f2, sis)
        eng.run(kernel=N.KERNEL_FP32_GUARDED)
        h, c = eng.histograms()
    check_hist(h, c, ho, co, N.KERNEL_FP32_GUARDED, 'lean walk with ineligible forests')
    assert c.sum() > 0


def test_graph_replay_and_recapture(cfg0):
    """A run is captured in a CUDA graph and replayed when called again with
    the same options: the replay reproduces the captured run's counts bit for
    bit; changing the walk or the run-length cap captures again and still
    gives the same counts."""
    fs, am, eng, _, _ = cfg0
    eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=0, run_cap=128)
    h1, c1 = eng.histograms()
    eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=0, run_cap=128)
    h2, c2 = eng.histograms()
    assert np.array_equal(c1, c2)
    np.testing.assert_allclose(h2, h1, rtol=1e-12, atol=0)
    for var, cap in ((N.VARIANT_TWO_DIAGONALS, 64), (0, 32), (1, 256)):
        eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=var, run_cap=cap)
        h3, c3 = eng.histograms()
        assert np.array_equal(c3, c1), f'walk {var}, cap {cap}'
        np.testing.assert_allclose(h3[:, N.Q_W], h1[:, N.Q_W], rtol=1e-6, atol=0)
    # a slot-restricted run captures its own graph; the full run after it is captured again
    eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=0, run_cap=128, slots=(3, 5))
    h4, c4 = eng.histograms()
    assert c4[:3].sum() == 0 and c4[5:].sum() == 0 and np.array_equal(c4[3:5], c1[3:5])
    eng.run(kernel=N.KERNEL_FP32_GUARDED, variant=0, run_cap=128)
    h5, c5 = eng.histograms()
    assert np.array_equal(c5, c1)
    with pytest.raises(N.LyaError):
        eng.run(kernel=N.KERNEL_FP32_GUARDED, run_cap=100)   # not a power of two


def test_autotune_choice_keeps_parity(cfg0):
    fs, am, eng, _, (f1, f2, sis, pixels) = cfg0
    res = eng.autotune(fraction=0.2, run_caps=(64, 128))
    assert res['best'] in [{'variant': t['variant'], 'run_cap': t['run_cap']} for t in res['timings']]
    assert len(res['timings']) == 6
    ns = 4
    ho, co = O.corr(fs, f1[:sis[ns]], f2[:sis[ns]], sis[:ns + 1])
    eng.run()                       # the tuned walk
    h, c = eng.histograms(0, ns)
    check_hist(h, c, ho, co, N.KERNEL_FP32_GUARDED, 'autotuned')
    eng.tuned.clear()


def test_device_neighbours_equal_reference_neighborhood():
    """The device work queue equals the reference's own quasar.neighborhood
    lists (golden vectors, tests/golden/make_neighbour_golden.py) as sets per
    first forest."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'neighbour_golden.npz'))
    for fs, tag in ((synthetic.make(0, n=400), 'cat0'), (E.edge_catalog(), 'edge')):
        off, nbr = g[f'{tag}_off'], g[f'{tag}_nbr']
        with PairEngine() as eng:
            eng.upload(fs)
            n = eng.build_pairs(float(g[f'{tag}_angmax']))
            d1, d2 = eng.get_pairs()
        assert n == len(nbr) > 0
        for f in range(fs.n):
            assert sorted(d2[d1 == f].tolist()) == sorted(nbr[off[f]:off[f + 1]].tolist()), (tag, f)
