"""Full-size configuration (150,000 forests): size-independent properties.

The oracle cannot bin 6e12 pixel pairs in a test, so the full-size check is:
pair counts of the FP32-guarded kernel equal the FP64 kernel's bin for bin in
every owner pixel; W agrees to 1e-6 relative; DW, RP, RT, Z agree normwise to
1e-6; the pair totals match the kernel's in-range count; a sampled pixel
matches the oracle exactly."""
import numpy as np
import pytest

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_config1_fp32_equals_fp64_everywhere():
    fs = synthetic.make(1)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        npairs = eng.build_pairs(am)
        assert npairs > 4e7
        st32 = eng.run(kernel=N.KERNEL_FP32_GUARDED)
        h32, c32 = eng.histograms()
        st64 = eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
        h64, c64 = eng.histograms()
        assert np.array_equal(c32, c64)
        assert int(c32.sum()) == int(st32['in_range_pairs']) == int(st64['in_range_pairs'])
        assert st32['evaluated_pairs'] <= st32['ref_pairs']
        W32, W64 = h32[:, N.Q_W], h64[:, N.Q_W]
        nz = W64 != 0
        assert np.max(np.abs(W32[nz] - W64[nz]) / W64[nz]) < 1e-6
        for q in (N.Q_DW, N.Q_RP, N.Q_RT, N.Q_Z):
            a, b = h32[:, q], h64[:, q]
            assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max(), q
        # one sampled owner pixel against the oracle (exact counts)
        s = len(eng.slot_pixels) // 2
        members = np.nonzero(eng.slot_of_forest == s)[0]
        f1, f2 = eng.get_pairs()
        sel = np.isin(f1, members)
        ho, co = O.corr(fs, f1[sel], f2[sel], [0, int(sel.sum())])
        assert np.array_equal(c32[s], co[0])
        np.testing.assert_allclose(W32[s], ho[0, O.Q_W], rtol=1e-6, atol=0)


def test_config3_distortion_properties():
    """Whole distortion catalogue (30,000 log-normal forests, all pairs): the
    oracle cannot restate 1.4e7 forest pairs in a test, so the check is the
    size-independent one the factored form offers.  W_B of the distortion (the
    sum of w_i w_j over the pairs of bin B, accumulated from the tensor-core
    moments) equals the FP64 correlation kernel's W histogram summed over owner
    pixels, bin for bin, to 1e-12 (the same FP64 bin formula, sums in another
    order); D is finite and symmetric to 1e-12 of its largest entry (each
    off-diagonal block is added at (A, B) and (B, A))."""
    fs = synthetic.make(3)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        assert eng.build_pairs(am) > 1e7
        D, WB = eng.distortion()
        eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
        h, c = eng.histograms()
    W = h[:, N.Q_W].sum(axis=0)
    assert np.array_equal(W != 0, WB != 0)
    nz = W != 0
    assert nz.sum() > 2000
    assert np.max(np.abs(WB[nz] - W[nz]) / np.abs(W[nz])) < 1e-12
    assert np.all(np.isfinite(D))
    assert np.abs(D - D.T).max() <= 1e-12 * np.abs(D).max()
