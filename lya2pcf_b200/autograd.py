"""Differentiable correlation function through the library's adjoint kernel.

No reference counterpart: the reference computes histograms only.  The loss
the adjoint serves is L = sum_b g_b xi_b with xi_b = DW_b / W_b over all owner
pixels and the pair bins held fixed (bins depend only on comoving distances and
directions, which are not differentiated).

* :func:`xi` -- ``torch.autograd.Function`` mapping per-pixel (w, dw) tensors to
  xi[np*nt]; its backward calls ``lya_corr_adjoint`` (a gather over both
  directions of every forest pair, no stored pairs).
* :func:`project_delta` -- the mean-and-slope projection of
  ``forest_class.fill_dw(project=True)`` (``forest_class.py:48-68``) in torch, so
  gradients chain from xi to the raw deltas and weights.
"""
import numpy as np
import torch

from . import _native as N


class _Xi(torch.autograd.Function):
    """Forward: the library's histograms of the given (w, dw), reduced to the
    totals W, DW on the device (lya_corr_totals) and xi = DW/W in torch.
    Backward: lya_corr_adjoint with g on the device and the gradients written
    into device tensors.  Only the library's stream and torch's current stream
    are synchronised between the two (no host copies of histograms)."""

    @staticmethod
    def forward(ctx, w, dw, engine, kernel):
        if not (w.is_cuda and dw.is_cuda):
            raise ValueError('w and dw must be CUDA tensors on the engine device')
        w64 = w.detach().to(torch.float64).contiguous()
        dw64 = dw.detach().to(torch.float64).contiguous()
        torch.cuda.current_stream(w.device).synchronize()
        engine.update_weights(w64, dw64)
        engine.run(kernel=kernel)
        W = torch.empty(engine.nb, dtype=torch.float64, device=w.device)
        DW = torch.empty_like(W)
        engine.totals(out_w=W, out_dw=DW)
        xi_ = torch.where(W != 0, DW / torch.where(W != 0, W, torch.ones_like(W)), torch.zeros_like(W))
        ctx.engine = engine
        ctx.shape = w64.shape
        ctx.device = w.device
        ctx.dtypes = (w.dtype, dw.dtype)
        return xi_.to(dtype=w.dtype)

    @staticmethod
    def backward(ctx, gxi):
        g = gxi.detach().to(torch.float64).contiguous()
        gdw = torch.empty(ctx.shape, dtype=torch.float64, device=ctx.device)
        gw = torch.empty(ctx.shape, dtype=torch.float64, device=ctx.device)
        torch.cuda.current_stream(ctx.device).synchronize()
        ctx.engine.adjoint(g, out_dw=gdw, out_w=gw)
        return gw.to(ctx.dtypes[0]), gdw.to(ctx.dtypes[1]), None, None


def xi(w, dw, engine, kernel=N.KERNEL_FP64_DIAGONAL):
    """xi_b = sum dw1 dw2 / sum w1 w2 over all pixel pairs in bin b (0 where
    empty) for the engine's catalogue and work queue, differentiable in w and dw."""
    return _Xi.apply(w, dw, engine, kernel)


def forest_index(start, device):
    """Forest id of every pixel of a CSR catalogue."""
    start = np.asarray(start)
    lens = np.diff(start)
    return torch.as_tensor(np.repeat(np.arange(len(lens)), lens), device=device)


def _segsum(v, fid, n):
    return torch.zeros(n, dtype=v.dtype, device=v.device).index_add_(0, fid, v)


def project_delta(w, delta, loglam, fid, n_forests):
    """dw = w * (delta - <delta>_w - dl <dl delta>_w / <dl^2>_w), dl = loglam - <loglam>_w,
    per forest (``forest_class.fill_dw`` with project=True), in torch."""
    sw = _segsum(w, fid, n_forests)
    mean_delta = _segsum(w * delta, fid, n_forests) / sw
    lam_avg = _segsum(w * loglam, fid, n_forests) / sw
    dl = loglam - lam_avg[fid]
    num = _segsum(w * dl * delta, fid, n_forests) / sw
    den = _segsum(w * dl * dl, fid, n_forests) / sw
    return w * (delta - mean_delta[fid] - dl * (num / den)[fid])
