"""The no-allocation entry point, lya_corr_pixel_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory (their device memory
belongs to another framework's caching allocator, they run under a fixed
device-memory budget, or allocation calls must stay out of a sequence they
record): they pass the catalogue, the pair list and the outputs in their own
device memory.  This test gives it one owner pixel of the small synthetic
catalogue in torch-owned device memory and checks two calls in a row against
the library's allocating path (lya_corr_run with the FP64 plain kernel, same
arithmetic): pair counts equal, sums within 1e-12 relative (the two paths add
in different orders).  It also checks that more bins than the fixed scratch
holds are rejected.  Collected last so that a failure here stops a run only
after every other test has run."""
import ctypes as C

import numpy as np
import pytest
import torch

from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device='cuda')


def test_noalloc_matches_allocating_path_twice():
    fs = synthetic.make(0, scale=0.1)
    am = synthetic.angmax_for(fs)
    with PairEngine() as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        s = int(eng.slot_of_forest[f1[len(f1) // 2]])
        eng.run(kernel=N.KERNEL_FP64_PLAIN, slots=(s, s + 1))
        ref_h, ref_c = eng.histograms(s, 1)
    sel = eng.slot_of_forest[f1] == s
    p1, p2 = f1[sel], f2[sel]
    nb = 2500
    t = dict(dc=_dev(fs.dc, torch.float64), w=_dev(fs.w, torch.float64), dw=_dev(fs.dw, torch.float64),
             z=_dev(fs.z, torch.float64), start=_dev(fs.start, torch.int64), ux=_dev(fs.ux, torch.float64),
             uy=_dev(fs.uy, torch.float64), uz=_dev(fs.uz, torch.float64), f1=_dev(p1, torch.int32),
             f2=_dev(p2, torch.int32))
    hist = torch.full((N.NQ * nb,), 7.0, dtype=torch.float64, device='cuda')     # garbage: must be overwritten
    cnt = torch.full((nb,), 3, dtype=torch.int64, device='cuda')
    lib = N.load()
    ptr = lambda x: C.c_void_p(x.data_ptr())  # noqa: E731
    torch.cuda.synchronize()
    for call in range(2):
        rc = lib.lya_corr_pixel_noalloc(0, ptr(t['dc']), ptr(t['w']), ptr(t['dw']), ptr(t['z']), ptr(t['start']),
                                        ptr(t['ux']), ptr(t['uy']), ptr(t['uz']), ptr(t['f1']), ptr(t['f2']),
                                        len(p1), 200.0, 200.0, 50, 50, ptr(hist), ptr(cnt), None)
        assert rc == 0, lib.lya_last_error(None)
        torch.cuda.synchronize()
        h = hist.cpu().numpy().reshape(N.NQ, nb)
        c = cnt.cpu().numpy().view(np.uint64)
        assert np.array_equal(c, ref_c[0]), f'call {call}: pair counts differ'
        np.testing.assert_allclose(h, ref_h[0], rtol=1e-12, atol=1e-12 * np.abs(ref_h[0]).max())
        assert c.sum() > 0


def test_noalloc_rejects_more_bins_than_its_scratch():
    lib = N.load()
    x = torch.zeros(8, dtype=torch.float64, device='cuda')
    i = torch.zeros(8, dtype=torch.int64, device='cuda')
    j = torch.zeros(8, dtype=torch.int32, device='cuda')
    ptr = lambda y: C.c_void_p(y.data_ptr())  # noqa: E731
    rc = lib.lya_corr_pixel_noalloc(0, ptr(x), ptr(x), ptr(x), ptr(x), ptr(i), ptr(x), ptr(x), ptr(x), ptr(j),
                                    ptr(j), 0, 200.0, 200.0, 100, 50, ptr(x), ptr(i), None)
    assert rc == 1   # LYA_ERR_ARG
    assert b'exceeds the fixed scratch' in lib.lya_last_error(None)
