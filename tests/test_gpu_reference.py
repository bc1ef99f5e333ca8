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
