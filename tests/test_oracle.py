"""The CPU oracle against the reference's golden vectors and hand-computed cases."""
import numpy as np
import pytest

from helpers import forestset
from oracle import oracle as O

G_PAIRS = 'tests/golden/numba_pairs.npz'
G_PIXEL = 'tests/golden/numba_pixel.npz'
G_SWEEP = 'tests/golden/numba_sweep.npz'


def _load(name):
    import os
    return np.load(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), name))


def _pair_fs(g, c):
    keys = ('ra', 'dec', 'dc', 'w', 'dw', 'z')
    fa = {k: g[f'c{c}_a_{k}'] for k in keys}
    fb = {k: g[f'c{c}_b_{k}'] for k in keys}
    return forestset([fa, fb])


@pytest.mark.parametrize('golden', [G_PAIRS, G_SWEEP])
def test_numba_pairs_bit_exact(golden):
    """CPU-formula oracle == the reference numba pair_correlation, bit for bit
    (hand-placed pairs, and a seeded whole-sky sweep: high declinations, the
    ra = 0 / 2 pi wrap, separations around the angle cut)."""
    g = _load(golden)
    for c in range(int(g['n_cases'])):
        fs = _pair_fs(g, c)
        out, cnt = O.corr(fs, [0], [1], [0, 1], mode=O.CPU_FORMULA, angmax=float(g['angmax']))
        assert np.array_equal(out[0, O.Q_W].reshape(50, 50), g[f'c{c}_w_hist']), c
        assert np.array_equal(out[0, O.Q_DW].reshape(50, 50), g[f'c{c}_dw_hist']), c


def test_numba_pixel_bit_exact():
    """A whole pixel through the reference CPU backend (two_point_per_pixel):
    same histograms, including the per-forest-pair summation order."""
    g = _load(G_PIXEL)
    n = int(g['n'])
    forests = [dict(ra=float(g[f'f{f}_ra']), dec=float(g[f'f{f}_dec']), dc=g[f'f{f}_dc'], w=g[f'f{f}_w'],
                    dw=g[f'f{f}_dw'], z=g[f'f{f}_z']) for f in range(n)]
    fs = forestset(forests)
    f1 = np.concatenate([np.full(len(g[f'f{f}_nbr']), f) for f in range(n)]).astype(np.int32)
    f2 = np.concatenate([g[f'f{f}_nbr'] for f in range(n)]).astype(np.int32)
    out, cnt = O.corr(fs, f1, f2, [0, len(f1)], mode=O.CPU_FORMULA, angmax=float(g['angmax']))
    assert np.array_equal(out[0, O.Q_W].reshape(50, 50), g['w_hist'])
    assert np.array_equal(out[0, O.Q_DW].reshape(50, 50), g['dw_hist'])


@pytest.mark.parametrize('golden', [G_PAIRS, G_SWEEP])
def test_gpu_formula_agrees_with_cpu_formula_on_golden_cases(golden):
    """The two reference formulas differ only near bin edges; on the golden
    cases they give the same bins and sums within rounding.  The GPU kernel has
    no angle cut (the neighbour search applies it), so sweep pairs at or beyond
    angmax are left out."""
    g = _load(golden)
    angmax = float(g['angmax'])
    for c in range(int(g['n_cases'])):
        ra1, dec1, ra2, dec2 = (float(g[f'c{c}_{t}_{k}']) for t, k in (('a', 'ra'), ('a', 'dec'), ('b', 'ra'),
                                                                       ('b', 'dec')))
        cosang = np.sin(dec1) * np.sin(dec2) + np.cos(dec1) * np.cos(dec2) * np.cos(ra1 - ra2)
        if not np.arccos(min(1.0, cosang)) < angmax * (1 - 1e-9):
            continue
        fs = _pair_fs(g, c)
        oc, cc = O.corr(fs, [0], [1], [0, 1], mode=O.CPU_FORMULA, angmax=float(g['angmax']))
        og, cg = O.corr(fs, [0], [1], [0, 1], mode=O.GPU_FORMULA)
        assert np.array_equal(cc, cg)
        np.testing.assert_allclose(og[0, O.Q_W], oc[0, O.Q_W], rtol=1e-12, atol=1e-12)


def _los(ra, dec):
    return dict(ra=ra, dec=dec)


def test_kat_coincident_lines_of_sight():
    """Same direction, different quasars: cos12 = 1, rt = 0, rp = |dc1-dc2|;
    pairs exactly 4k apart land in bin k (the lower edge is inclusive)."""
    d1 = np.array([4000.0, 4004.0, 4100.0])
    d2 = np.array([4000.0, 4008.0, 4299.0, 4300.0])
    fa = dict(ra=0.5, dec=0.1, dc=d1, w=np.ones(3), dw=np.ones(3), z=np.full(3, 2.0))
    fb = dict(ra=0.5, dec=0.1, dc=d2, w=np.ones(4), dw=np.ones(4), z=np.full(4, 2.0))
    fs = forestset([fa, fb])
    out, cnt = O.corr(fs, [0], [1], [0, 1])
    expect = np.zeros(2500, dtype=np.uint64)
    for a in d1:
        for b in d2:
            k = int(np.floor(abs(a - b) * 0.25))
            if k < 50:
                expect[k * 50 + 0] += 1
    assert np.array_equal(cnt[0], expect)
    # rp = 200 exactly (4100 vs 4300) is out; 4100 vs 4299 is in bin 49
    assert expect[49 * 50] >= 1


def test_kat_rt_edge_exact():
    """sin(theta/2) = 2^-5 exactly: rt = (d1+d2)/32; d1+d2 = 6400 gives rt = 200
    (excluded), 6399.999 gives rt just below 200 (bin 49)."""
    c = 1.0 - 2.0 ** -9
    s = np.sqrt(1 - c * c)
    fa = dict(ra=0.0, dec=0.0, dc=np.array([3200.0, 3199.999]), w=np.ones(2), dw=np.ones(2), z=np.full(2, 2.0),
              ux=1.0, uy=0.0, uz=0.0)
    fb = dict(ra=0.1, dec=0.0, dc=np.array([3200.0]), w=np.ones(1), dw=np.ones(1), z=np.full(1, 2.0),
              ux=c, uy=s, uz=0.0)
    fs = forestset([fa, fb])
    out, cnt = O.corr(fs, [0], [1], [0, 1])
    assert O.cos12((1.0, 0.0, 0.0), (c, s, 0.0), 0) == c
    assert cnt[0].sum() == 1
    assert cnt[0][0 * 50 + 49] == 1


def test_cos_variant_cases_discriminate():
    import edge_cases as E
    fs, f1, f2, vb = E.cos_variant_cases(48)
    assert len(f1) == 48
    assert (vb[:, 0] != vb[:, 1]).any() and (vb[:, 0] != vb[:, 2]).any()
    # the oracle (variant 0) bins each case where the generator predicts
    for c in range(len(f1)):
        out, cnt = O.corr(fs, [f1[c]], [f2[c]], [0, 1], cos_variant=0)
        nz = np.nonzero(cnt[0])[0]
        assert (int(nz[0]) if len(nz) else -1) == vb[c, 0]


def test_adjoint_matches_finite_differences():
    """Oracle adjoint of L = sum_b g_b DW_b/W_b (bins fixed) vs central
    differences of the oracle's own histograms."""
    rng = np.random.default_rng(4)
    import edge_cases as E
    deg = np.pi / 180
    F = [E.same_grid_forest(1.0 + rng.uniform(0, 0.3) * deg, 0.2 + rng.uniform(0, 0.3) * deg,
                            int(rng.integers(0, 100)), int(rng.integers(5, 12)), rng) for _ in range(4)]
    fs = forestset(F)
    f1 = np.array([0, 0, 0, 1, 1, 2], dtype=np.int32)
    f2 = np.array([1, 2, 3, 2, 3, 3], dtype=np.int32)
    g = rng.normal(size=2500)

    def loss(fs_):
        out, _ = O.corr(fs_, f1, f2, [0, len(f1)])
        W, DW = out[0, O.Q_W], out[0, O.Q_DW]
        xi = np.divide(DW, W, out=np.zeros_like(W), where=W != 0)
        return float(np.sum(g * xi)), W, DW

    L0, W, DW = loss(fs)
    xi = np.divide(DW, W, out=np.zeros_like(W), where=W != 0)
    cdw = np.divide(g, W, out=np.zeros_like(W), where=W != 0)
    cw = -cdw * xi
    gdw, gw = O.adjoint(fs, f1, f2, cdw, cw)
    eps = 1e-6
    for p in rng.choice(fs.npix_total, 12, replace=False):
        for arr, grad in ((fs.dw, gdw), (fs.w, gw)):
            old = arr[p]
            arr[p] = old + eps
            lp = loss(fs)[0]
            arr[p] = old - eps
            lm = loss(fs)[0]
            arr[p] = old
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grad[p]) <= 1e-5 * max(1.0, abs(fd)), (p, fd, grad[p])


def _eta_form_distortion(fs, f1, f2, np_=50, nt=50):
    """Independent statement of the distortion numerator:
    D_AB = sum_{forest pairs} sum_{(i,j) in A} w_i w_j sum_{(k,l) in B} eta1_ik eta2_jl,
    eta_ik = delta_ik - w_k/Omega - dl_i w_k dl_k / sum(w dl^2)."""
    nb = np_ * nt
    D = np.zeros((nb, nb))
    WB = np.zeros(nb)
    for a, b in zip(f1, f2):
        A = fs.forest(a); B = fs.forest(b)
        c = O.cos12((fs.ux[a], fs.uy[a], fs.uz[a]), (fs.ux[b], fs.uy[b], fs.uz[b]), 0)
        ch, sh = np.sqrt(0.5 * (1 + c)), np.sqrt(0.5 * (1 - c))
        rp = np.abs(A['dc'][:, None] - B['dc'][None, :]) * ch
        rt = (A['dc'][:, None] + B['dc'][None, :]) * sh
        bp, bt = np.floor(rp * (np_ / 200.0)), np.floor(rt * (nt / 200.0))
        ok = (bp < np_) & (bt < nt)
        binm = np.where(ok, bp * nt + bt, -1).astype(int)

        def eta(F):
            w, dl = F['w'], F['dl']
            return np.eye(len(w)) - w[None, :] / w.sum() - dl[:, None] * (w * dl)[None, :] / np.sum(w * dl * dl)
        e1, e2 = eta(A), eta(B)
        ww = A['w'][:, None] * B['w'][None, :]
        for Abin in np.unique(binm[binm >= 0]):
            M = np.where(binm == Abin, ww, 0.0)
            WB[Abin] += M.sum()
            for Bbin in np.unique(binm[binm >= 0]):
                Nm = (binm == Bbin).astype(float)
                D[Abin, Bbin] += np.sum(M * (e1 @ Nm @ e2.T))
    return D, WB


@pytest.mark.parametrize('np_,nt', [(50, 50), (37, 23), (64, 16)])
def test_distortion_matches_eta_product_form(np_, nt):
    rng = np.random.default_rng(8)
    import edge_cases as E
    deg = np.pi / 180
    F = []
    for _ in range(3):
        f = E.same_grid_forest(1.0 + rng.uniform(0, 0.2) * deg, 0.2 + rng.uniform(0, 0.2) * deg,
                               int(rng.integers(0, 60)), int(rng.integers(4, 9)), rng)
        f['dl'] = np.log10((1 + f['z']) * 1215.67)
        f['dl'] = f['dl'] - np.sum(f['dl'] * f['w']) / np.sum(f['w'])
        F.append(f)
    fs = forestset(F)
    f1 = np.array([0, 0, 1], dtype=np.int32)
    f2 = np.array([1, 2, 2], dtype=np.int32)
    D, WB = O.distortion(fs, f1, f2, np_=np_, nt=nt)
    De, WBe = _eta_form_distortion(fs, f1, f2, np_, nt)
    np.testing.assert_allclose(WB, WBe, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(D, De, rtol=1e-9, atol=1e-9 * np.abs(De).max())


def test_fp32_distortion_binning_matches_numpy_float32():
    """The oracle's FP32 binning (the reference distortion's
    precompute_distances, cuda_kernels.cpp:67-84) in its uncontracted variant
    against the same arithmetic in numpy float32: FP32 unit vectors and dc,
    the half-angle argument 0.5*(1 +- cos) in FP64 rounded to FP32 before
    sqrtf, FP32 products, truncation of rp*binner and rt*binner."""
    from lya2pcf_b200 import synthetic
    fs = synthetic.make(4, n=12, length=(20, 60))
    f32 = np.float32
    for a, b in ((0, 1), (2, 5), (3, 11), (7, 4)):
        bp, bt = O.dist_bins(fs, a, b, cos_variant=2, bin_mode=O.BIN_FP32)
        u1 = [f32(fs.ux[a]), f32(fs.uy[a]), f32(fs.uz[a])]
        u2 = [f32(fs.ux[b]), f32(fs.uy[b]), f32(fs.uz[b])]
        c = (u1[0] * u2[0] + u1[1] * u2[1]) + u1[2] * u2[2]
        ch = np.sqrt(f32(0.5 * (1.0 + np.float64(c))))
        sh = np.sqrt(f32(0.5 * (1.0 - np.float64(c))))
        d1 = fs.dc[fs.start[a]:fs.start[a + 1]].astype(f32)
        d2 = fs.dc[fs.start[b]:fs.start[b + 1]].astype(f32)
        rp = np.abs(d1[:, None] - d2[None, :]) * ch
        rt = (d1[:, None] + d2[None, :]) * sh
        assert rp.dtype == f32 and rt.dtype == f32
        assert np.array_equal(bp, (rp * f32(0.25)).astype(np.int32))
        assert np.array_equal(bt, (rt * f32(0.25)).astype(np.int32))
        # the FP64 binning of the same pair is a different function
        b64p, b64t = O.dist_bins(fs, a, b, bin_mode=O.BIN_FP64)
        assert np.array_equal(b64p, np.floor(np.abs(fs.dc[fs.start[a]:fs.start[a + 1], None]
                                                    - fs.dc[None, fs.start[b]:fs.start[b + 1]])
                                             * np.sqrt(0.5 * (1.0 + O.cos12((fs.ux[a], fs.uy[a], fs.uz[a]),
                                                                            (fs.ux[b], fs.uy[b], fs.uz[b]), 0)))
                                             * 0.25).astype(np.int32))


def test_distortion_fp32_binning_differs_only_through_bins():
    """With the FP32 binning the oracle's W_B differs from the FP64 binning's
    (some pairs change bins) while its total stays within 1%."""
    from lya2pcf_b200 import synthetic
    fs = synthetic.make(4, n=14, length=(20, 80))
    off, nbr = O.neighbours(fs, synthetic.angmax_for(fs))
    f1, f2, _, _ = O.items_from_csr(fs, off, nbr)
    D64, W64 = O.distortion(fs, f1, f2, bin_mode=O.BIN_FP64)
    D32, W32 = O.distortion(fs, f1, f2, bin_mode=O.BIN_FP32)
    assert W64.sum() > 0 and not np.array_equal(W32, W64)
    np.testing.assert_allclose(W32.sum(), W64.sum(), rtol=1e-2)


def test_wdw_baseline_equals_full_oracle():
    """The W/DW-only path the CPU baseline times gives the full oracle's W and
    DW bit for bit."""
    from lya2pcf_b200 import synthetic
    fs = synthetic.make(0, scale=0.05)
    off, nbr = O.neighbours(fs, synthetic.angmax_for(fs))
    f1, f2, sis, _ = O.items_from_csr(fs, off, nbr)
    h, _ = O.corr(fs, f1, f2, sis)
    w = O.corr_wdw(fs, f1, f2, sis)
    assert np.array_equal(w[:, 0], h[:, O.Q_W]) and np.array_equal(w[:, 1], h[:, O.Q_DW])
