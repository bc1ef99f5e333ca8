"""The no-allocation entry point, lya_corr_pixel_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory (their device memory
belongs to another framework's caching allocator, they run under a fixed
device-memory budget, or allocation calls must stay out of a sequence they
record): they pass the catalogue, the pair list and the outputs in their own
device memory.  These tests give it owner pixels in torch-owned device memory
and check two calls in a row against the CPU oracle (pair counts bit-exact,
sums within 1e-12: FP64 arithmetic added in a different order) and against
the library's allocating path (lya_corr_run with the FP64 plain kernel).  They
also cover an empty pair list (outputs zeroed), a caller's stream, the largest
binning the fixed scratch holds (64 x 64 = 4096 bins) and the rejection of
more bins than that.  Collected last so that a failure here stops a run only
after every other test has run."""
import ctypes as C

import numpy as np
import pytest
import torch

import edge_cases as E
from lya2pcf_b200 import _native as N
from lya2pcf_b200 import synthetic
from lya2pcf_b200.engine import PairEngine
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device='cuda')


def _ptr(x):
    return C.c_void_p(x.data_ptr())


class _Catalogue:
    """A catalogue and one pixel's forest pairs in torch-owned device memory."""

    def __init__(self, fs, p1, p2):
        self.t = dict(dc=_dev(fs.dc, torch.float64), w=_dev(fs.w, torch.float64), dw=_dev(fs.dw, torch.float64),
                      z=_dev(fs.z, torch.float64), start=_dev(fs.start, torch.int64),
                      ux=_dev(fs.ux, torch.float64), uy=_dev(fs.uy, torch.float64), uz=_dev(fs.uz, torch.float64),
                      f1=_dev(p1 if len(p1) else [0], torch.int32), f2=_dev(p2 if len(p2) else [0], torch.int32))
        self.n_pairs = len(p1)

    def call(self, hist, cnt, np_=50, nt=50, stream=None, n_pairs=None):
        t = self.t
        lib = N.load()
        return lib.lya_corr_pixel_noalloc(0, _ptr(t['dc']), _ptr(t['w']), _ptr(t['dw']), _ptr(t['z']),
                                          _ptr(t['start']), _ptr(t['ux']), _ptr(t['uy']), _ptr(t['uz']),
                                          _ptr(t['f1']), _ptr(t['f2']),
                                          self.n_pairs if n_pairs is None else n_pairs, 200.0, 200.0, np_, nt,
                                          _ptr(hist), _ptr(cnt), stream)


def _garbage_outputs(nb):
    hist = torch.full((N.NQ * nb,), 7.0, dtype=torch.float64, device='cuda')   # must be overwritten
    cnt = torch.full((nb,), 3, dtype=torch.int64, device='cuda')
    return hist, cnt


def _read(hist, cnt, nb):
    return hist.cpu().numpy().reshape(N.NQ, nb), cnt.cpu().numpy().view(np.uint64)


def _check_oracle(h, c, ho, co):
    """FP64 sums within 1e-12 of the oracle (DW against sum |dw1 dw2|)."""
    assert np.array_equal(c, co), 'pair counts differ from the oracle'
    assert np.all(np.abs(h[N.Q_W] - ho[O.Q_W]) <= TOL * np.abs(ho[O.Q_W]))
    assert np.all(np.abs(h[N.Q_DW] - ho[O.Q_DW]) <= TOL * ho[O.Q_DWABS])
    for q, qo in ((N.Q_RP, O.Q_RP), (N.Q_RT, O.Q_RT), (N.Q_Z, O.Q_Z)):
        assert np.all(np.abs(h[q] - ho[qo]) <= TOL * np.abs(ho[qo]) + 1e-300)


def _one_pixel(fs, am, np_=50, nt=50, pick=0.5):
    """Pairs of one owner pixel, and that pixel's histograms from the library's
    allocating path (FP64 plain kernel) at the same binning."""
    with PairEngine(np_=np_, nt=nt) as eng:
        eng.upload(fs)
        eng.build_pairs(am)
        f1, f2 = eng.get_pairs()
        s = int(eng.slot_of_forest[f1[int(len(f1) * pick)]])
        eng.run(kernel=N.KERNEL_FP64_PLAIN, slots=(s, s + 1))
        ref_h, ref_c = eng.histograms(s, 1)
        sel = eng.slot_of_forest[f1] == s
    return f1[sel], f2[sel], ref_h[0], ref_c[0]


def test_noalloc_matches_oracle_and_allocating_path_twice():
    """One owner pixel of the small configuration, two calls in a row."""
    fs = synthetic.make(0, scale=0.1)
    am = synthetic.angmax_for(fs)
    p1, p2, ref_h, ref_c = _one_pixel(fs, am)
    ho, co = O.corr(fs, p1, p2, [0, len(p1)])
    cat = _Catalogue(fs, p1, p2)
    hist, cnt = _garbage_outputs(2500)
    torch.cuda.synchronize()
    for call in range(2):
        rc = cat.call(hist, cnt)
        assert rc == 0, N.load().lya_last_error(None)
        torch.cuda.synchronize()
        h, c = _read(hist, cnt, 2500)
        _check_oracle(h, c, ho[0], co[0])
        assert np.array_equal(c, ref_c), f'call {call}: pair counts differ from lya_corr_run'
        np.testing.assert_allclose(h, ref_h, rtol=TOL, atol=TOL * np.abs(ref_h).max())
        assert c.sum() > 0


def test_noalloc_edge_catalogue_matches_oracle():
    """Every pair of the edge catalogue (coincident lines of sight, rt exactly
    200, empty and length-1 forests, twins, unsorted forests) in one call, on a
    caller's stream."""
    fs = E.edge_catalog()
    off, nbr = O.neighbours(fs, 0.05)
    f1, f2, _, _ = O.items_from_csr(fs, off, nbr)
    ho, co = O.corr(fs, f1, f2, [0, len(f1)])
    cat = _Catalogue(fs, f1, f2)
    hist, cnt = _garbage_outputs(2500)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(2):
        rc = cat.call(hist, cnt, stream=C.c_void_p(stream.cuda_stream))
        assert rc == 0, N.load().lya_last_error(None)
        stream.synchronize()
        h, c = _read(hist, cnt, 2500)
        _check_oracle(h, c, ho[0], co[0])
        assert c.sum() > 0


def test_noalloc_empty_pair_list_zeroes_outputs():
    fs = synthetic.make(0, scale=0.02)
    cat = _Catalogue(fs, np.zeros(0, np.int32), np.zeros(0, np.int32))
    hist, cnt = _garbage_outputs(2500)
    torch.cuda.synchronize()
    assert cat.call(hist, cnt) == 0
    torch.cuda.synchronize()
    h, c = _read(hist, cnt, 2500)
    assert not h.any() and not c.any()


def test_noalloc_at_its_largest_binning():
    """64 x 64 bins, the 4096 the fixed scratch holds (the largest shared-memory
    histogram of the kernel), against the oracle and lya_corr_run."""
    fs = synthetic.make(0, scale=0.1)
    am = synthetic.angmax_for(fs)
    p1, p2, ref_h, ref_c = _one_pixel(fs, am, 64, 64, pick=0.3)
    ho, co = O.corr(fs, p1, p2, [0, len(p1)], np_=64, nt=64)
    cat = _Catalogue(fs, p1, p2)
    hist, cnt = _garbage_outputs(4096)
    torch.cuda.synchronize()
    for _ in range(2):
        assert cat.call(hist, cnt, 64, 64) == 0, N.load().lya_last_error(None)
        torch.cuda.synchronize()
        h, c = _read(hist, cnt, 4096)
        _check_oracle(h, c, ho[0], co[0])
        assert np.array_equal(c, ref_c)
        assert c.sum() > 0


def test_noalloc_rejects_more_bins_than_its_scratch():
    lib = N.load()
    x = torch.zeros(8, dtype=torch.float64, device='cuda')
    i = torch.zeros(8, dtype=torch.int64, device='cuda')
    j = torch.zeros(8, dtype=torch.int32, device='cuda')
    rc = lib.lya_corr_pixel_noalloc(0, _ptr(x), _ptr(x), _ptr(x), _ptr(x), _ptr(i), _ptr(x), _ptr(x), _ptr(x),
                                    _ptr(j), _ptr(j), 0, 200.0, 200.0, 100, 50, _ptr(x), _ptr(i), None)
    assert rc == 1   # LYA_ERR_ARG
    assert b'exceeds the fixed scratch' in lib.lya_last_error(None)
