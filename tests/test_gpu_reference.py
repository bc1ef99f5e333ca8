"""Pinning against the reference's own CUDA kernel.

oracle/_ref/libref_kernels.so is cuda_kernels.cpp of the reference tree
compiled like PyCUDA compiles it, driven like two_point_per_pixel drives it.
With w = dw = 1 its w_hist is the exact pair count per bin."""
import numpy as np
import pytest

import edge_cases as E
from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O
from oracle import ref as R

pytestmark = pytest.mark.gpu


def _need_ref():
    if not R.available():
        pytest.fail('oracle/_ref/libref_kernels.so missing: build it where the reference tree is present '
                    '(make -C oracle ref)')


def test_reference_kernel_uses_the_oracle_contraction():
    """On pairs that the three FMA contractions of cos12 bin differently, the
    compiled reference kernel agrees with contraction 0, the one the oracle and
    the library use."""
    _need_ref()
    fs, f1, f2, vb = E.cos_variant_cases(192)
    got = []
    for c in range(len(f1)):
        w, _ = R.corr_pixel(fs, [f1[c]], [[f2[c]]], weights=False)
        nz = np.nonzero(w.ravel())[0]
        got.append(int(nz[0]) if len(nz) else -1)
    got = np.array(got)
    assert np.array_equal(got, vb[:, 0])
    assert not np.array_equal(got, vb[:, 1]) and not np.array_equal(got, vb[:, 2])


def test_reference_kernel_pixel_counts_and_sums():
    """One owner pixel of the small configuration: pair counts of the reference
    kernel == oracle == every library kernel; W and DW of the reference
    (FP64 global atomics, any order) within 1e-12 of the oracle."""
    _need_ref()
    fs = synthetic.make(0)
    am = synthetic.angmax_for(fs)
    off, nbr = O.neighbours(fs, am)
    f1, f2, sis, pixels = O.items_from_csr(fs, off, nbr)
    s = 2
    firsts = np.unique(f1[sis[s]:sis[s + 1]])
    lists = [nbr[off[f]:off[f + 1]] for f in firsts]
    cref, _ = R.corr_pixel(fs, firsts, lists, weights=False)
    wref, dwref = R.corr_pixel(fs, firsts, lists, weights=True)
    ho, co = O.corr(fs, f1[sis[s]:sis[s + 1]], f2[sis[s]:sis[s + 1]], [0, sis[s + 1] - sis[s]])
    assert np.array_equal(cref.ravel().astype(np.uint64), co[0])
    np.testing.assert_allclose(wref.ravel(), ho[0, O.Q_W], rtol=1e-12, atol=0)
    assert np.all(np.abs(dwref.ravel() - ho[0, O.Q_DW]) <= 1e-12 * ho[0, O.Q_DWABS])
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        for kern in (N.KERNEL_FP32_GUARDED, N.KERNEL_FP64_DIAGONAL, N.KERNEL_FP64_PLAIN):
            eng.run(kernel=kern, slots=(s, s + 1))
            h, c = eng.histograms(s, 1)
            assert np.array_equal(c[0], cref.ravel().astype(np.uint64)), kern


# ---------------------------------------------------------------- distortion
# The reference distortion (distortion_procedures_pycuda.py:195-279) reads FP32
# copies of dc, w, delta_lambda, the unit vectors, omega and
# omega_delta_lambda2 (:71-100), bins pairs in FP32 (precompute_distances,
# cuda_kernels.cpp:67-84) and accumulates eta and D with FP32 global atomics
# (:165-278).  Its forests are padded to max_lenght = 208 pixels
# (parameters.py:59) and its scratch holds 80 neighbours (parameters.py:61), so
# the pinning catalogue keeps forests of at most 208 pixels and fewer than 80
# neighbours per first forest.
#
# Tolerances (FP32 accumulation of up to ~1e4 positive terms per bin):
#   W_B: 1e-4 relative per bin; D: 1e-4 of max|D| per entry.
# The FP32 and FP64 binnings differ on ~0.3% of pixel pairs, which moves D by
# ~7e-3 of max|D| on the pinning catalogue, so the D check tells the two
# binnings apart by a factor of ~70.
D_TOL = 1e-4
W_TOL = 1e-4


def _fp32_inputs(fs):
    """``fs`` with every value the reference distortion reads as FP32 rounded
    to FP32, so that the reference, the oracle and the library start from the
    same numbers."""
    g = fs.subset(np.arange(fs.n))
    for k in ('dc', 'w', 'dw', 'dl', 'ux', 'uy', 'uz', 'omega', 'odl2'):
        setattr(g, k, getattr(g, k).astype(np.float32).astype(np.float64))
    return g


def _pin_catalogue():
    """60 forests of 40-208 pixels with the configuration-4 sky density (3
    healpix pixels, at most 59 neighbours per first forest)."""
    fs = _fp32_inputs(synthetic.make(4, n=60, length=(40, 208)))
    return fs, synthetic.angmax_for(fs)


def _reference_distortion(fs, off, nbr):
    """The distortion.py driver loop (:101-108) over every owner pixel with
    --excluded 0 (every neighbour kept): per pixel the reference kernels' FP32
    D and W_B, summed on the host in FP64."""
    nb = 2500
    D = np.zeros((nb, nb)); W = np.zeros(nb)
    for pixel, forests in fs.pixel_groups().items():
        lists = [nbr[off[f]:off[f + 1]] for f in forests]
        Dp, Wp = R.dist_pixel(fs, forests, lists)
        D += Dp; W += Wp
    return D, W


def _d_err(D, Do):
    return float(np.abs(D - Do).max() / np.abs(Do).max())


def test_reference_distortion_bins_equal_oracle_fp32_binning():
    """Every (bin_rp, bin_rt) that the compiled precompute_distances writes
    equals the oracle's FP32 binning (contraction 0 of the FP32 cos), pixel
    pair for pixel pair, on eight first forests and all their neighbours."""
    _need_ref()
    fs, am = _pin_catalogue()
    off, nbr = O.neighbours(fs, am)
    cat = O.Catalog(fs)
    firsts = [f for f in range(fs.n) if off[f + 1] > off[f]]
    firsts = firsts[::max(1, len(firsts) // 8)][:8]
    agree = np.zeros(3, dtype=np.int64)
    total = differ64 = 0
    for f1 in firsts:
        lst = nbr[off[f1]:off[f1 + 1]]
        bp, bt = R.dist_bins(fs, f1, lst)
        for q, f2 in enumerate(lst):
            l2 = int(fs.lengths[f2])
            assert np.all(bp[:, q, l2:] == -1) and np.all(bt[:, q, l2:] == -1)
            rp, rt = bp[:, q, :l2], bt[:, q, :l2]
            for v in range(3):
                obp, obt = O.dist_bins(fs, f1, f2, cos_variant=v, bin_mode=O.BIN_FP32, cat=cat)
                agree[v] += np.count_nonzero((obp == rp) & (obt == rt))
            o64p, o64t = O.dist_bins(fs, f1, f2, bin_mode=O.BIN_FP64, cat=cat)
            differ64 += np.count_nonzero((o64p != rp) | (o64t != rt))
            total += rp.size
    assert total > 100000
    assert agree[0] == total, f'FP32 bins agreeing per contraction variant: {agree.tolist()} of {total}'
    assert differ64 > 0   # the FP32 binning is a different function from the FP64 one


def test_reference_distortion_matches_oracle_fp32_binning():
    """D and W_B of the reference kernels, driven per owner pixel like
    distortion.py, against the oracle's restatement with the reference's FP32
    binning: within FP32 accumulation tolerance, and far closer than to the
    oracle's FP64 binning."""
    _need_ref()
    fs, am = _pin_catalogue()
    off, nbr = O.neighbours(fs, am)
    f1, f2, _, _ = O.items_from_csr(fs, off, nbr)
    Dr, Wr = _reference_distortion(fs, off, nbr)
    Do, Wo = O.distortion(fs, f1, f2, bin_mode=O.BIN_FP32)
    D64, _ = O.distortion(fs, f1, f2, bin_mode=O.BIN_FP64)
    assert np.count_nonzero(Wo) > 500 and np.count_nonzero(Do) > 100000
    assert np.array_equal(Wr != 0, Wo != 0)
    np.testing.assert_allclose(Wr, Wo, rtol=W_TOL, atol=0)
    err32, err64 = _d_err(Dr, Do), _d_err(Dr, D64)
    assert err32 <= D_TOL, f'reference vs oracle (FP32 bins): {err32:.3e} of max|D|'
    assert err64 > 10 * err32, f'FP64 bins {err64:.3e} vs FP32 bins {err32:.3e}'


def test_library_distortion_matches_oracle_fp64_on_pinning_catalogue():
    """The library (FP64 binning, factored form) on the same FP32-valued
    catalogue against the oracle's FP64 binning: 1e-10 of max|D|, W 1e-12."""
    fs, am = _pin_catalogue()
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        D, W = eng.distortion()
    Do, Wo = O.distortion(fs, f1, f2, bin_mode=O.BIN_FP64)
    np.testing.assert_allclose(W, Wo, rtol=1e-12, atol=1e-12 * np.abs(Wo).max())
    assert _d_err(D, Do) <= 1e-10


def _edge_free_catalogue():
    """24 short forests (6-16 pixels) whose pixel pairs all bin the same under
    the reference's FP32 binning and the FP64 one: the weights of both pixels
    of every pair that the two binnings put in different bins (or only one of
    them in range) are set to 0, which removes those pairs from D and W_B on
    both sides.  Returns (catalogue, angmax, fraction of pixels zeroed)."""
    fs = _fp32_inputs(synthetic.make(4, n=24, length=(6, 16)))
    am = synthetic.angmax_for(fs)
    off, nbr = O.neighbours(fs, am)
    f1, f2, _, _ = O.items_from_csr(fs, off, nbr)
    cat = O.Catalog(fs)
    bad = np.zeros(fs.npix_total, dtype=bool)
    for a, b in zip(f1, f2):
        p64, t64 = O.dist_bins(fs, a, b, bin_mode=O.BIN_FP64, cat=cat)
        p32, t32 = O.dist_bins(fs, a, b, bin_mode=O.BIN_FP32, cat=cat)
        in64 = (p64 >= 0) & (p64 < 50) & (t64 >= 0) & (t64 < 50)
        in32 = (p32 >= 0) & (p32 < 50) & (t32 >= 0) & (t32 < 50)
        i, j = np.nonzero((in64 | in32) & ((p64 != p32) | (t64 != t32) | (in64 != in32)))
        bad[fs.start[a] + i] = True
        bad[fs.start[b] + j] = True
    fs.w = np.where(bad, 0.0, fs.w)
    return fs, am, float(bad.mean())


def test_library_distortion_matches_reference_directly():
    """On a catalogue with no pixel pair near a bin edge (see
    _edge_free_catalogue) the library's D and W equal the reference kernels'
    to FP32 accumulation tolerance."""
    _need_ref()
    fs, am, zeroed = _edge_free_catalogue()
    assert zeroed < 0.25
    off, nbr = O.neighbours(fs, am)
    Dr, Wr = _reference_distortion(fs, off, nbr)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        D, W = eng.distortion()
    assert np.count_nonzero(W) > 100
    np.testing.assert_allclose(Wr, W, rtol=W_TOL, atol=0)
    assert _d_err(Dr, D) <= D_TOL, f'library vs reference: {_d_err(Dr, D):.3e} of max|D|'
