"""Adjoint kernel and torch.autograd.Function (no reference counterpart).

Checked against the oracle's FP64 adjoint and against central finite
differences (eps = 1e-6, float64) on the 500-forest, 10 deg^2 configuration
(forests of 100-300 pixels): tolerance 1e-5 of the gradient's largest
component.  The float32 path (float32 w and delta in, float32 gradients out)
is checked against the float64 path at the same float32-representable inputs:
1e-4 of the largest component (the float32 projection of delta rounds dw at
2^-24, and xi sums dw products of random sign, so its float32 error relative
to max |xi| is ~1e-5)."""
import numpy as np
import pytest
import torch

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.autograd import forest_index, project_delta, xi
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope='module')
def cfg4():
    fs = synthetic.make(4)
    assert fs.n == 500 and fs.lengths.min() >= 100 and fs.lengths.max() <= 300
    am = synthetic.angmax_for(fs)
    eng = PairEngine().upload(fs)
    eng.build_pairs(am)
    yield fs, am, eng
    eng.close()


def test_adjoint_matches_oracle(cfg4):
    fs, am, eng = cfg4
    eng.update_weights(fs.w, fs.dw)
    eng.run(kernel=N.KERNEL_FP64_DIAGONAL)
    hist, _ = eng.histograms()
    W, DW = hist[:, N.Q_W].sum(0), hist[:, N.Q_DW].sum(0)
    g = np.random.default_rng(3).normal(size=eng.nb)
    gdw, gw = eng.adjoint(g)
    xi_ = np.divide(DW, W, out=np.zeros_like(W), where=W != 0)
    cdw = np.divide(g, W, out=np.zeros_like(W), where=W != 0)
    f1, f2 = eng.get_pairs()
    odw, ow = O.adjoint(fs, f1, f2, cdw, -cdw * xi_)
    np.testing.assert_allclose(gdw, odw, rtol=1e-9, atol=1e-12 * np.abs(odw).max())
    np.testing.assert_allclose(gw, ow, rtol=1e-9, atol=1e-12 * np.abs(ow).max())
    # device-pointer outputs give the same (up to the order of FP64 atomics)
    tdw = torch.empty(fs.npix_total, dtype=torch.float64, device='cuda')
    tw = torch.empty_like(tdw)
    eng.adjoint(g, out_dw=tdw, out_w=tw)
    np.testing.assert_allclose(tdw.cpu().numpy(), gdw, rtol=1e-12, atol=1e-15 * np.abs(gdw).max())
    np.testing.assert_allclose(tw.cpu().numpy(), gw, rtol=1e-12, atol=1e-15 * np.abs(gw).max())


def test_autograd_matches_finite_differences(cfg4):
    fs, am, eng = cfg4
    dev = torch.device('cuda')
    fid = forest_index(fs.start, dev)
    loglam = torch.as_tensor(np.log10((1 + fs.z) * 1215.67), device=dev)
    rng = np.random.default_rng(5)
    delta0 = torch.as_tensor(rng.normal(0, 0.25, fs.npix_total), device=dev)
    w0 = torch.as_tensor(fs.w.copy(), device=dev)
    g = torch.as_tensor(rng.normal(size=eng.nb), device=dev)

    def loss(w, delta):
        dw = project_delta(w, delta, loglam, fid, fs.n)
        return torch.sum(g * xi(w, dw, eng))

    w = w0.clone().requires_grad_(True)
    delta = delta0.clone().requires_grad_(True)
    L = loss(w, delta)
    gw, gdelta = torch.autograd.grad(L, (w, delta))
    eps = 1e-6
    scale = {'delta': float(gdelta.abs().max()), 'w': float(gw.abs().max())}
    assert scale['delta'] > 0 and scale['w'] > 0
    for p in rng.choice(fs.npix_total, 8, replace=False):
        for which, grad in (('delta', gdelta), ('w', gw)):
            wp, dp = w0.clone(), delta0.clone()
            (dp if which == 'delta' else wp)[p] += eps
            lp = float(loss(wp, dp))
            wm, dm = w0.clone(), delta0.clone()
            (dm if which == 'delta' else wm)[p] -= eps
            lm = float(loss(wm, dm))
            fd = (lp - lm) / (2 * eps)
            an = float(grad[p])
            # normwise: 1e-5 of the gradient's largest component (the FP64
            # forward's rounding noise, ~1e-10 after dividing by 2 eps, sets
            # the floor for the smallest components)
            assert abs(fd - an) <= 1e-5 * max(abs(fd), scale[which]), (which, int(p), fd, an)


def test_totals_equal_summed_histograms(cfg4):
    fs, am, eng = cfg4
    eng.update_weights(fs.w, fs.dw)
    eng.run(kernel=N.KERNEL_FP32_GUARDED)
    hist, _ = eng.histograms()
    W, DW = eng.totals()
    np.testing.assert_allclose(W, hist[:, N.Q_W].sum(0), rtol=1e-13, atol=0)
    np.testing.assert_allclose(DW, hist[:, N.Q_DW].sum(0), rtol=1e-12, atol=1e-13 * np.abs(DW).max())
    tW = torch.empty(eng.nb, dtype=torch.float64, device='cuda')
    tDW = torch.empty_like(tW)
    eng.totals(out_w=tW, out_dw=tDW)
    assert np.array_equal(tW.cpu().numpy(), W) and np.array_equal(tDW.cpu().numpy(), DW)


def test_float32_path_matches_float64_path(cfg4):
    """float32 w and delta: xi and the gradients (float32) equal the float64
    path's at the same (float32-representable) inputs to 1e-4 of their
    largest component."""
    fs, am, eng = cfg4
    dev = torch.device('cuda')
    fid = forest_index(fs.start, dev)
    rng = np.random.default_rng(8)
    loglam = torch.as_tensor(np.log10((1 + fs.z) * 1215.67), device=dev)
    delta32 = torch.as_tensor(rng.normal(0, 0.25, fs.npix_total).astype(np.float32), device=dev)
    w32 = torch.as_tensor(fs.w.astype(np.float32), device=dev)
    g = torch.as_tensor(rng.normal(size=eng.nb), device=dev)
    out = {}
    for dt in (torch.float32, torch.float64):
        w = w32.to(dt).clone().requires_grad_(True)
        delta = delta32.to(dt).clone().requires_grad_(True)
        dw = project_delta(w, delta, loglam.to(dt), fid, fs.n)
        x = xi(w, dw, eng)
        L = torch.sum(g.to(dt) * x)
        gw, gd = torch.autograd.grad(L, (w, delta))
        assert x.dtype == dt and gw.dtype == dt and gd.dtype == dt
        out[dt] = (x.detach().double(), gw.double(), gd.double())
    for k in range(3):
        a, b = out[torch.float32][k], out[torch.float64][k]
        assert float((a - b).abs().max()) <= 1e-4 * float(b.abs().max()), k
